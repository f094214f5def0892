"""Batches: several solves of different shapes and precisions propagated together on one GPU give,
bit for bit, the current each gives alone (the work split and reduction order of a solve do not
depend on what runs beside it)."""
import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu


def _solves(pyswe):
    import tbgen

    base = dict(nr3=1, tmax=1.5, dt=0.02197, intensity=1.5e12, tmax_field=80.0, phi_vec=np.zeros(3),
                **{"lambda": 3000.0})
    specs = [("haldane", 24, [0.0, 1.0, 0.0], "fp64"), ("tmd6_s1", 10, [0.6, 0.8, 0.0], "fp64"),
             ("tmd11_s7", 12, [0.0, 1.0, 0.0], "fp64"), ("tmd11_s2", 8, [0.8, 0.6, 0.0], "mixed"),
             ("haldane", 16, [1.0, 0.0, 0.0], "mixed"), ("tmd12_s3", 6, [0.0, 1.0, 0.0], "mixed")]
    out = []
    for model, n, pol, prec in specs:
        p = dict(base, path_tb=tbgen.model_path(model), nr1=n, nr2=n, pol_vec=np.array(pol))
        out.append(pyswe.SWE(pyswe.Settings(p), precision=prec))
    return out


def test_batch_equals_solo_bit_for_bit():
    from pySWE import pyswe

    solves = _solves(pyswe)
    solo = []
    for s in solves:
        s.reset()
        s.run_simulation()
        solo.append(s.get_current()[1:])
    batch = pyswe.SWEBatch(solves)
    for rep in range(2):  # first run captures the graph, second replays it
        batch.run()
        for s, J in zip(solves, solo):
            assert np.array_equal(s.get_current()[1:], J), rep
    assert batch.last_ms() > 0
    batch.delete()
    for s in solves:
        s.delete()


def test_batch_recaptures_after_reinit():
    from pySWE import pyswe

    meta, param, _, J_ref = load_golden("tmd11_10")
    a = pyswe.SWE(pyswe.Settings(dict(param)))
    meta2, param2, _, J_ref2 = load_golden("haldane_12_pol")
    b = pyswe.SWE(pyswe.Settings(dict(param2)))
    batch = pyswe.SWEBatch([a, b])
    batch.run()
    a.restart()  # new device buffers: the batch must notice
    batch.run()
    for s, J in ((a, J_ref), (b, J_ref2)):
        got = s.get_current()[1:]
        assert rel_l2(got[1], J[1]) < 1e-10
    batch.delete()
    a.delete()
    b.delete()
