"""The element-group variants a solve can run on a Hermitian 7x7 cell box (the compiled box, k-point
pairs with 2x2 register tiles for the commutator, precomputed inner Wannier sums) against each other
and against the golden J(t) made by the reference build: precomputed sums give the same bits as the
in-kernel sums, and every variant stays within the parity bar (FP64 1e-10 per axis, mixed 1e-6).

The HHG_GROUP_* variables only remove variants from the planner's list; they are read when a solve is
set up."""
import os

import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu

FLAGS = ("HHG_GROUP_NOPRE", "HHG_GROUP_NOPAIR", "HHG_GROUP_ANYBOX")
NAMES = ["tmd6_8", "tmd11_10", "tmd12_6", "c2_prefix", "ks_tmd11_10"]


def run(param, precision, env):
    from pySWE import pyswe

    saved = {k: os.environ.pop(k, None) for k in FLAGS}
    os.environ.update({k: "1" for k in env})
    try:
        s = pyswe.SWE(pyswe.Settings(dict(param)), precision=precision, solver=param.get("solver", "rspace"))
        s.run_simulation()
        J = np.stack(s.get_current()[1:])
        launches = s.last_launches()
        shape = s.launch_shape()
        s.delete()
    finally:
        for k in FLAGS:
            os.environ.pop(k, None)
        os.environ.update({k: v for k, v in saved.items() if v is not None})
    return J, launches, (shape["threads"], shape["k_per_cta"], shape["ctas"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["tmd6_8", "tmd11_10", "c2_prefix", "ks_tmd11_10"])  # grids of at least 7x7: a 7x7 box
def test_precomputed_sums_are_bit_identical(name, precision):
    _, param, _, _ = load_golden(name)
    J_pre, n_pre, shape_pre = run(param, precision, [])
    J_in, n_in, shape_in = run(param, precision, ["HHG_GROUP_NOPRE"])
    nt = J_pre.shape[1]
    # Precomputed: one (sums, propagation) launch pair per 64 steps; in-kernel: one propagation.
    # (Only the k-space solver's 11- and 12-orbital shapes have them among its compiled shapes.)
    if param.get("solver") == "kspace" and "tmd11" not in name:
        pytest.skip("no precomputed-sum shape")
    assert n_pre == 2 * ((nt + 63) // 64) + 1, (n_pre, nt)
    assert n_in == 2
    if shape_pre == shape_in:
        assert np.array_equal(J_pre, J_in)
    else:
        # FP64 shapes with precomputed sums hold more k-points per CTA (they need fewer registers),
        # which changes only the order of the final k-sum.
        assert precision == "fp64" and rel_l2(J_pre, J_in) < 1e-13, (shape_pre, shape_in, rel_l2(J_pre, J_in))


@pytest.mark.parametrize("env", [[], ["HHG_GROUP_NOPRE"], ["HHG_GROUP_NOPAIR"], ["HHG_GROUP_NOPRE", "HHG_GROUP_NOPAIR"],
                                 ["HHG_GROUP_ANYBOX"]])
@pytest.mark.parametrize("name", NAMES)
def test_every_variant_within_the_parity_bar(name, env):
    _, param, _, J_ref = load_golden(name)
    J64, _, _ = run(param, "fp64", env)
    for a in range(3):
        if np.abs(J_ref[a]).max() == 0:
            assert np.abs(J64[a]).max() == 0, (name, env, a)
        else:
            assert rel_l2(J64[a], J_ref[a]) < 1e-10, (name, env, a, rel_l2(J64[a], J_ref[a]))
    Jm, _, _ = run(param, "mixed", env)
    assert rel_l2(Jm, J_ref) < 1e-6, (name, env, rel_l2(Jm, J_ref))
