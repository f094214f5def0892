"""Serving with continuous batching (SWEServer): requests that arrive while others run are admitted
by device-memory footprint, advance together in chunks of RK4 steps, and each result equals, bit for
bit, the current the same solve gives alone (plain FP64 and mixed precision alike)."""
import threading
import time

import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu

BASE = dict(nr3=1, tmax=1.2, dt=0.02197, tmax_field=80.0, phi_vec=np.zeros(3), **{"lambda": 3000.0})
SPECS = [("haldane", 24, 0.0, 1.5e12, "fp64"), ("tmd11_s2", 10, 30.0, 1e12, "mixed"),
         ("tmd6_s1", 12, 75.0, 2e12, "fp64"), ("haldane", 16, 120.0, 0.5e12, "mixed"),
         ("tmd12_s3", 8, 160.0, 1e12, "mixed"), ("tmd6_s2", 14, 10.0, 3e11, "mixed"),
         ("tmd11_s7", 8, 90.0, 1e12, "fp64")]


def _settings(pyswe, model, n, ang, inten):
    import tbgen

    a = np.radians(ang)
    p = dict(BASE, path_tb=tbgen.model_path(model), nr1=n, nr2=n, intensity=inten,
             pol_vec=np.array([np.sin(a), np.cos(a), 0.0]))
    return pyswe.Settings(p)


def _solo(pyswe, specs=SPECS):
    out = []
    for model, n, ang, inten, prec in specs:
        s = pyswe.SWE(_settings(pyswe, model, n, ang, inten), precision=prec)
        s.run_simulation()
        out.append(s.get_current()[1:])
        s.delete()
    return out


@pytest.mark.parametrize("chunk", [20, 33, 256])  # 33: chunks that start on odd steps
def test_each_result_is_the_same_alone_and_in_the_mix(chunk):
    from pySWE import pyswe

    solo = _solo(pyswe)
    srv = pyswe.SWEServer(device=0, max_active=4, chunk_steps=chunk)
    reqs = [pyswe.SWE(_settings(pyswe, m, n, a, i), precision=p, defer_init=True) for m, n, a, i, p in SPECS]
    tickets = []

    def arrive():  # staggered arrivals: later requests join while earlier ones run
        for r in reqs:
            tickets.append(srv.submit(r))
            time.sleep(0.003)

    th = threading.Thread(target=arrive)
    th.start()
    th.join()
    for tk in tickets:
        assert srv.wait(tk, timeout=120.0)
    for r, J, tk in zip(reqs, solo, tickets):
        assert np.array_equal(r.get_current()[1:], J), (tk, srv.times(tk))
        tm = srv.times(tk)
        assert tm["submit"] <= tm["admit"] <= tm["start"] <= tm["done"]
    st = srv.stats()
    assert st["completed"] == len(SPECS) and st["failed"] == 0
    assert 1 <= st["peak_running"] <= 4
    srv.close()
    for r in reqs:
        r.delete()


def test_admission_respects_the_memory_budget():
    from pySWE import pyswe

    specs = SPECS[:3]
    solo = _solo(pyswe, specs)
    # A budget of a few MiB admits one or two of these solves at a time.
    srv = pyswe.SWEServer(device=0, hbm_budget=24 << 20, max_active=8, chunk_steps=16)
    reqs = [pyswe.SWE(_settings(pyswe, m, n, a, i), precision=p, defer_init=True) for m, n, a, i, p in specs]
    tickets = [srv.submit(r) for r in reqs]
    for tk in tickets:
        assert srv.wait(tk, timeout=120.0)
    st = srv.stats()
    assert st["peak_bytes"] <= st["budget_bytes"] or st["peak_running"] == 1
    for r, J in zip(reqs, solo):
        assert np.array_equal(r.get_current()[1:], J)
    srv.close()


def test_a_failing_request_does_not_disturb_the_others(tmp_path):
    from pySWE import pyswe

    _, param, _, J_ref = load_golden("haldane_12_pol")
    srv = pyswe.SWEServer(device=0, chunk_steps=64)
    good = pyswe.SWE(pyswe.Settings(dict(param)), defer_init=True)
    bad = pyswe.SWE(pyswe.Settings(dict(param, path_tb=str(tmp_path / "missing_tb.dat"))), defer_init=True)
    odd = pyswe.SWE(pyswe.Settings(dict(param, nr1=13)), defer_init=True)
    t_good, t_bad, t_odd = srv.submit(good), srv.submit(bad), srv.submit(odd)
    with pytest.raises(pyswe.SWEError, match="tb file"):
        srv.wait(t_bad, timeout=60.0)
    with pytest.raises(pyswe.SWEError, match="even"):
        srv.wait(t_odd, timeout=60.0)
    assert srv.wait(t_good, timeout=60.0)
    assert rel_l2(good.get_current()[2], J_ref[1]) < 1e-10  # the golden pulse, served in 64-step chunks
    assert srv.stats()["failed"] == 2
    srv.close()
    # A served SWESim can be set up again and run alone.
    good.init()
    good.run_simulation()
    assert rel_l2(good.get_current()[2], J_ref[1]) < 1e-10
