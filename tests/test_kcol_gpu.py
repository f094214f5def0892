"""The column-tile kernel (2-orbital models, FP64): forced onto grids where the planner would pick
the thread-per-k-point kernel, it must reproduce the reference's goldens (both solvers) and stay
bit-identical when run in chunks beside other solves."""
import os

import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture
def force_kcol():
    old = os.environ.get("HHG_KERNEL")
    os.environ["HHG_KERNEL"] = "kcol"
    yield
    if old is None:
        del os.environ["HHG_KERNEL"]
    else:
        os.environ["HHG_KERNEL"] = old


@pytest.mark.parametrize("name", ["haldane_8_y", "haldane_12_pol", "haldane_16_rect", "c0", "ks_haldane_12_pol",
                                  "ks_c0"])
def test_kcol_matches_golden(force_kcol, name):
    from pySWE import pyswe

    _, param, t_ref, J_ref = load_golden(name)
    s = pyswe.SWE(pyswe.Settings(dict(param)), solver=param.get("solver", "rspace"))
    assert s.launch_shape()["kernel_name"] == "propagate_kcol_kernel"
    s.run_simulation()
    J = s.get_current()[1:]
    s.delete()
    for a in range(3):
        if np.abs(J_ref[a]).max() == 0:
            assert np.abs(J[a]).max() == 0
        else:
            assert rel_l2(J[a], J_ref[a]) < 1e-10, (name, a, rel_l2(J[a], J_ref[a]))


@pytest.mark.parametrize("name", ["haldane_12_pol", "ks_haldane_12_pol"])
def test_kcol_full_box_form_matches_golden(force_kcol, name):
    """HHG_KCOL_FULLBOX=1 sums every box row instead of the Hermitian-halved ones."""
    from pySWE import pyswe

    _, param, t_ref, J_ref = load_golden(name)
    os.environ["HHG_KCOL_FULLBOX"] = "1"
    try:
        s = pyswe.SWE(pyswe.Settings(dict(param)), solver=param.get("solver", "rspace"))
        assert s.launch_shape()["kernel_name"] == "propagate_kcol_kernel"
        s.run_simulation()
        J = s.get_current()[1:]
        s.delete()
    finally:
        del os.environ["HHG_KCOL_FULLBOX"]
    for a in range(3):
        if np.abs(J_ref[a]).max() > 0:
            assert rel_l2(J[a], J_ref[a]) < 1e-10, (name, a, rel_l2(J[a], J_ref[a]))


def test_kcol_tile_split_does_not_change_the_result(force_kcol):
    from pySWE import pyswe

    _, param, _, _ = load_golden("c0")
    param = dict(param, tmax=3.0)
    out = []
    for parts in ("1", "3"):
        os.environ["HHG_KCOL_PARTS"] = parts
        s = pyswe.SWE(pyswe.Settings(dict(param)))
        s.run_simulation()
        out.append(s.get_current()[1:])
        s.delete()
    del os.environ["HHG_KCOL_PARTS"]
    assert rel_l2(out[0][1], out[1][1]) < 1e-11  # the k-sum is grouped differently: rounding only


def test_kcol_served_in_chunks_equals_alone(force_kcol):
    from pySWE import pyswe

    _, param, _, _ = load_golden("haldane_12_pol")
    solo = pyswe.SWE(pyswe.Settings(dict(param)))
    solo.run_simulation()
    J = solo.get_current()[1:]
    solo.delete()
    srv = pyswe.SWEServer(device=0, chunk_steps=13)
    r = pyswe.SWE(pyswe.Settings(dict(param)), defer_init=True)
    tk = srv.submit(r)
    assert srv.wait(tk, timeout=60.0)
    assert np.array_equal(r.get_current()[1:], J)
    srv.close()
