"""The reference's k-space solver (src/solver_kspace.cpp) on the GPU: SWE(..., solver="kspace")
against the CPU oracle's restatement of it (itself pinned to the reference's compiled solver by the
ks_* golden fixtures, checked in test_gpu_parity.py), in plain FP64 and mixed precision, alone and
served in chunks beside other solves."""
import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu


def _param(model, n, tmax, pol, intensity=1.5e12, lam=3000.0):
    import tbgen

    return {"path_tb": tbgen.model_path(model), "nr1": n, "nr2": n, "nr3": 1, "tmax": tmax, "dt": 0.02197,
            "intensity": intensity, "lambda": lam, "tmax_field": 80.0, "pol_vec": np.array(pol), "phi_vec": np.zeros(3)}


CASES = [("haldane", 20, 3.0, [0.6, 0.8, 0.0]),    # thread-per-k-point kernel
         ("haldane", 14, 2.0, [1.0, 0.0, 0.0]),
         ("tmd6_s2", 10, 1.0, [0.0, 1.0, 0.0]),    # element-group kernel
         ("tmd12_s3", 8, 0.6, [0.5, 0.5, 0.0]),
         ("tmd5_s4", 12, 0.8, [0.8, 0.6, 0.0])]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}_{c[1]}")
def test_kspace_fp64_matches_oracle(oracle_mod, case):
    from pySWE import pyswe

    p = _param(*case)
    _, J_ref = oracle_mod.run_kspace(p["path_tb"], p)
    s = pyswe.SWE(pyswe.Settings(p), solver="kspace")
    s.run_simulation()
    J = s.get_current()[1:]
    s.delete()
    for a in range(2):
        assert rel_l2(J[a], J_ref[a]) < 1e-10, (a, rel_l2(J[a], J_ref[a]))


@pytest.mark.parametrize("name", ["ks_tmd11_10", "ks_c0"])
def test_kspace_mixed_error_against_fp64(name):
    from pySWE import pyswe

    _, param, _, J_ref = load_golden(name)
    s = pyswe.SWE(pyswe.Settings(dict(param)), solver="kspace", precision="mixed")
    s.run_simulation()
    J = s.get_current()[1:]
    s.delete()
    err = np.linalg.norm(J - J_ref) / np.linalg.norm(J_ref)
    assert err < 1e-5, err


def test_kspace_chunked_and_served_equals_alone():
    from pySWE import pyswe

    specs = [(_param("haldane", 16, 1.5, [0.0, 1.0, 0.0]), "fp64"), (_param("tmd6_s1", 8, 1.0, [0.6, 0.8, 0.0]), "fp64"),
             (_param("tmd11_s2", 8, 0.6, [1.0, 0.0, 0.0]), "mixed")]
    solo = []
    for p, prec in specs:
        s = pyswe.SWE(pyswe.Settings(p), solver="kspace", precision=prec)
        s.run_simulation()
        solo.append(s.get_current()[1:])
        s.delete()
    srv = pyswe.SWEServer(device=0, max_active=3, chunk_steps=7)
    reqs = [pyswe.SWE(pyswe.Settings(p), solver="kspace", precision=prec, defer_init=True) for p, prec in specs]
    # one real-space solve in the mix as well
    rs = pyswe.SWE(pyswe.Settings(_param("haldane", 12, 1.5, [0.0, 1.0, 0.0])), defer_init=True)
    tickets = [srv.submit(r) for r in reqs] + [srv.submit(rs)]
    for tk in tickets:
        assert srv.wait(tk, timeout=120.0)
    for r, J in zip(reqs, solo):
        assert np.array_equal(r.get_current()[1:], J)
    srv.close()
