"""Edge cases against the CPU oracle: the largest supported orbital count (16), a single orbital,
a large grid (512 x 512, four column tiles per column), non-square grids on the element-group
kernel, the shortest pulse (nt = 2) and a prime step count."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _param(model, n1, n2, tmax, pol=(0.6, 0.8, 0.0)):
    import tbgen

    return {"path_tb": tbgen.model_path(model), "nr1": n1, "nr2": n2, "nr3": 1, "tmax": tmax, "dt": 0.02197,
            "intensity": 2e12, "lambda": 3000.0, "tmax_field": 80.0, "pol_vec": np.array(pol), "phi_vec": np.zeros(3)}


CASES = [("tmd16_s1", 6, 6, 0.3), ("tmd1_s2", 8, 8, 1.0), ("haldane", 512, 512, 0.2), ("tmd6_s2", 10, 14, 0.6),
         ("tmd11_s7", 6, 8, 0.05), ("haldane", 16, 16, 0.05), ("tmd6_s1", 8, 8, 0.0221 * 31)]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}_{c[1]}x{c[2]}_t{c[3]}")
def test_edge_case_matches_oracle(oracle_mod, case):
    from pySWE import pyswe

    model, n1, n2, tmax = case
    p = _param(model, n1, n2, tmax)
    _, J_ref = oracle_mod.run(p["path_tb"], p)
    s = pyswe.SWE(pyswe.Settings(p))
    s.run_simulation()
    J = s.get_current()[1:]
    nt = s.settings.nt
    s.delete()
    assert J.shape[1] == nt >= 2
    for a in range(2):
        if np.abs(J_ref[a]).max() == 0:
            assert np.abs(J[a]).max() < 1e-14  # a current the oracle finds exactly zero (one orbital)
        else:
            # Relative 1e-10, or an absolute floor of 1e-12: with the field barely on (nt = 2, or 0.2 fs
            # into the pulse) the current is 1e-7 or less of the O(1) terms the k-sum cancels, and its
            # rounding (about sqrt(Nk) x 1e-16 of those terms) is all that is left to compare.
            err = np.linalg.norm(J[a] - J_ref[a])
            assert err < 1e-10 * np.linalg.norm(J_ref[a]) or err < 1e-12, (a, rel_l2(J[a], J_ref[a]), err)
    if model != "haldane" or n1 < 100:
        m = pyswe.SWE(pyswe.Settings(p), precision="mixed")
        m.run_simulation()
        Jm = m.get_current()[1:]
        m.delete()
        err = np.linalg.norm(Jm - J_ref)
        assert err < 1e-5 * np.linalg.norm(J_ref) or err < 1e-12
