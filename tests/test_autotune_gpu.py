"""Autotuned tile shapes: the tuner picks among shapes that give the same propagation (results differ
only by the rounding of the current's k-sum order), and the choice is cached per solve shape, so
solves of one shape share tiles and batches stay bit-identical to solo runs."""
import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu


def _param(model, n, tmax, pol):
    import tbgen

    return {"path_tb": tbgen.model_path(model), "nr1": n, "nr2": n, "nr3": 1, "tmax": tmax, "dt": 0.02197,
            "intensity": 1.5e12, "lambda": 3000.0, "tmax_field": 80.0, "pol_vec": np.array(pol), "phi_vec": np.zeros(3)}


@pytest.mark.parametrize("model,n,prec", [("tmd11_s7", 30, "mixed"), ("tmd6_s1", 24, "fp64"), ("haldane", 160, "fp64")])
def test_autotuned_matches_default(model, n, prec):
    from pySWE import pyswe

    p = _param(model, n, 3.0, [0.6, 0.8, 0.0])
    out = []
    for tune in (False, True):
        s = pyswe.SWE(pyswe.Settings(p), precision=prec, autotune=tune)
        s.run_simulation()
        out.append((s.get_current()[1:], s.launch_shape()))
        s.delete()
    (J0, _), (J1, shape1) = out
    for a in range(2):
        assert rel_l2(J1[a], J0[a]) < (1e-11 if prec == "fp64" else 1e-6), (a, shape1)
    # a second solve of the same shape reuses the cached choice
    s = pyswe.SWE(pyswe.Settings(dict(p, intensity=0.7e12)), precision=prec, autotune=True)
    assert s.launch_shape() == shape1
    s.delete()


def test_autotuned_batch_equals_solo():
    from pySWE import pyswe

    specs = [(_param("tmd11_s2", 20, 1.0, [0.0, 1.0, 0.0]), "mixed"), (_param("tmd6_s3", 16, 1.0, [1.0, 0.0, 0.0]), "fp64")]
    solves = [pyswe.SWE(pyswe.Settings(p), precision=prec, autotune=True) for p, prec in specs]
    solo = []
    for s in solves:
        s.reset()
        s.run_simulation()
        solo.append(s.get_current()[1:])
    b = pyswe.SWEBatch(solves)
    b.run()
    for s, J in zip(solves, solo):
        assert np.array_equal(s.get_current()[1:], J)
    b.delete()
    for s in solves:
        s.delete()
