"""The element-group variants a solve can run on a Hermitian 7x7 cell box (the compiled box, k-point
pairs with 2x2 register tiles for the commutator, precomputed inner Wannier sums) against each other
and against the golden J(t) made by the reference build: precomputed sums give the same bits as the
in-kernel sums, and every variant stays within the parity bar (FP64 1e-10 per axis, mixed 1e-6).

The HHG_GROUP_* variables only remove variants from the planner's list; they are read when a solve is
set up.  The plain form of 11- and 12-orbital models on a 7x7 box runs the FP64 tensor-core fragment
kernel (sbe_dfrag.cuh) before any of them, and their mixed form the tile kernel (sbe_mtile.cuh);
HHG_DFRAG=0 and HHG_MTILE=0 remove them, so the element-group variants are compared with them off.
The mixed-form tensor-core fragment kernel (sbe_frag.cuh) is opt-in (HHG_FRAG=1) and checked against
its own measured accuracy."""
import os

import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu

FLAGS = ("HHG_GROUP_NOPRE", "HHG_GROUP_NOPAIR", "HHG_GROUP_ANYBOX", "HHG_FRAG", "HHG_FRAG_KPC", "HHG_DFRAG", "HHG_MTILE")
NAMES = ["tmd6_8", "tmd11_10", "tmd12_6", "c2_prefix", "ks_tmd11_10"]


def run(param, precision, env):
    from pySWE import pyswe

    saved = {k: os.environ.pop(k, None) for k in FLAGS}
    os.environ.update({k: "1" for k in env if "=" not in k})
    os.environ.update(dict(k.split("=") for k in env if "=" in k))
    try:
        s = pyswe.SWE(pyswe.Settings(dict(param)), precision=precision, solver=param.get("solver", "rspace"))
        s.run_simulation()
        J = np.stack(s.get_current()[1:])
        launches = s.last_launches()
        shape = s.launch_shape()
        name = shape["kernel_name"]
        s.delete()
    finally:
        for k in FLAGS:
            os.environ.pop(k, None)
        os.environ.update({k: v for k, v in saved.items() if v is not None})
    return J, launches, (shape["threads"], shape["k_per_cta"], shape["ctas"], name)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["tmd6_8", "tmd11_10", "c2_prefix", "ks_tmd11_10"])  # grids of at least 7x7: a 7x7 box
def test_precomputed_sums_are_bit_identical(name, precision):
    _, param, _, _ = load_golden(name)
    J_pre, n_pre, shape_pre = run(param, precision, ["HHG_DFRAG=0", "HHG_MTILE=0"])
    J_in, n_in, shape_in = run(param, precision, ["HHG_GROUP_NOPRE", "HHG_DFRAG=0", "HHG_MTILE=0"])
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


@pytest.mark.parametrize("env", [[], ["HHG_DFRAG=0", "HHG_MTILE=0"], ["HHG_GROUP_NOPRE", "HHG_DFRAG=0", "HHG_MTILE=0"],
                                 ["HHG_GROUP_NOPAIR", "HHG_MTILE=0"],
                                 ["HHG_GROUP_NOPRE", "HHG_GROUP_NOPAIR", "HHG_DFRAG=0", "HHG_MTILE=0"],
                                 ["HHG_GROUP_ANYBOX", "HHG_MTILE=0"]])
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


# Measured accuracy of the opt-in fragment kernel (round-toward-zero tensor-core accumulation, see
# sbe_frag.cuh): within the mixed form's 1e-6 on short runs, 2e-5 on the full pulse.
FRAG_TOL = {"tmd11_10": 1e-6, "c2_prefix": 1e-6, "tmd11_12_full": 2e-5}


@pytest.mark.parametrize("name", sorted(FRAG_TOL))
def test_fragment_kernel_against_element_groups(name):
    """The opt-in tensor-core fragment kernel (split-TF32 mma for the outer Wannier sums and the
    commutator) against the reference's current and the element-group kernel's."""
    _, param, _, J_ref = load_golden(name)
    J_frag, n_frag, shape = run(param, "mixed", ["HHG_FRAG=1"])
    assert shape[3] == "propagate_frag_kernel", shape
    J_grp, _, shape_grp = run(param, "mixed", ["HHG_MTILE=0"])
    assert shape_grp[3].startswith("propagate_group_kernel"), shape_grp
    nt = J_frag.shape[1]
    assert n_frag == 2 * ((nt + 63) // 64) + 1
    assert rel_l2(J_frag, J_ref) < FRAG_TOL[name], rel_l2(J_frag, J_ref)
    assert rel_l2(J_frag, J_grp) < FRAG_TOL[name], rel_l2(J_frag, J_grp)


@pytest.mark.parametrize("kpc", [16, 8])
def test_fragment_kernel_tile_shapes_and_ragged_columns(kpc):
    """16 and 8 k-points per CTA on grids whose columns do not divide into whole tiles (10 rows: a tile
    of 16 holds 10 k-points, tiles of 8 leave 2), on a non-square grid, and on a row slab."""
    import tbgen

    for n1, n2 in ((10, 10), (14, 8)):
        p = {"path_tb": tbgen.model_path("tmd11_s7"), "nr1": n1, "nr2": n2, "nr3": 1, "tmax": 3.0, "dt": 0.02197,
             "intensity": 2e12, "lambda": 3000.0, "tmax_field": 80.0, "pol_vec": np.array([0.6, 0.8, 0.0]),
             "phi_vec": np.zeros(3)}
        Jf, _, shape = run(p, "mixed", ["HHG_FRAG=1", f"HHG_FRAG_KPC={kpc}"])
        J64, _, _ = run(p, "fp64", [])
        assert shape[1] == kpc and shape[3] == "propagate_frag_kernel", shape
        assert rel_l2(Jf, J64) < 1e-6, (n1, n2, rel_l2(Jf, J64))
    # rows [3, 12) of a 14 x 8 grid: the slab's partial current against the FP64 slab's
    from pySWE import pyswe

    os.environ["HHG_FRAG"], os.environ["HHG_FRAG_KPC"] = "1", str(kpc)
    try:
        out = []
        for precision in ("mixed", "fp64"):
            s = pyswe.SWE(pyswe.Settings(dict(p)), precision=precision, k_rows=(3, 12))
            s.run_simulation()
            out.append(np.stack(s.get_current()[1:]))
            s.delete()
    finally:
        os.environ.pop("HHG_FRAG", None)
        os.environ.pop("HHG_FRAG_KPC", None)
    assert rel_l2(out[0], out[1]) < 1e-6, rel_l2(out[0], out[1])


@pytest.mark.parametrize("name", ["tmd11_10", "c2_prefix", "tmd11_12_full", "tmd12_12_full", "tmd12_6", "ks_tmd11_10"])
def test_fp64_fragment_kernel_against_element_groups(name):
    """The FP64 tensor-core fragment kernel (mma.m8n8k4.f64 for the outer Wannier sums and the
    commutator) is the plain form's kernel for 11 and 12 orbitals on a Hermitian 7x7 box: within the
    parity bar of the reference's current (1e-10 per axis) and within FP64 rounding of the
    element-group kernel.  (On the 6 x 6 and 12-orbital 12 x 12 grids the placement folds the model's
    cells into another box or a non-Hermitian table, and the element-group kernel runs.)"""
    _, param, _, J_ref = load_golden(name)
    J_d, n_d, shape = run(param, "fp64", [])
    J_g, _, shape_g = run(param, "fp64", ["HHG_DFRAG=0"])
    assert shape_g[3] != "propagate_dfrag_kernel"
    if name in ("tmd11_10", "c2_prefix", "tmd11_12_full", "ks_tmd11_10"):
        assert shape[3] == "propagate_dfrag_kernel", shape
        nt = J_d.shape[1]
        assert n_d == 2 * ((nt + 63) // 64) + 1
    for a in range(3):
        if np.abs(J_ref[a]).max() == 0:
            assert np.abs(J_d[a]).max() == 0
        else:
            assert rel_l2(J_d[a], J_ref[a]) < 1e-10, (a, rel_l2(J_d[a], J_ref[a]))
            assert rel_l2(J_d[a], J_g[a]) < 1e-11, (a, rel_l2(J_d[a], J_g[a]))


def test_fp64_fragment_kernel_ragged_columns_and_slabs():
    """Columns that do not divide into whole tiles of 8 k-points (10 and 14 rows), non-square grids, both
    polarisation layouts (one and two field axes), 11 and 12 orbitals, and a row slab, against the
    element-group kernel."""
    import tbgen
    from pySWE import pyswe

    ran12 = False
    for model, (n1, n2), pol in (("tmd11_s7", (10, 10), [0.0, 1.0, 0.0]), ("tmd11_s7", (14, 8), [0.6, 0.8, 0.0]),
                                 ("tmd12_s1", (20, 20), [0.8, 0.6, 0.0]), ("tmd12_s1", (30, 30), [0.0, 1.0, 0.0]),
                                 ("tmd12_s3", (18, 24), [0.0, 1.0, 0.0])):
        p = {"path_tb": tbgen.model_path(model), "nr1": n1, "nr2": n2, "nr3": 1, "tmax": 2.0, "dt": 0.02197,
             "intensity": 2e12, "lambda": 3000.0, "tmax_field": 80.0, "pol_vec": np.array(pol),
             "phi_vec": np.zeros(3)}
        Jd, _, shape = run(p, "fp64", [])
        Jg, _, _ = run(p, "fp64", ["HHG_DFRAG=0"])
        if model.startswith("tmd11"):
            assert shape[3] == "propagate_dfrag_kernel", (model, n1, n2, shape)
        ran12 = ran12 or (model.startswith("tmd12") and shape[3] == "propagate_dfrag_kernel")
        assert rel_l2(Jd, Jg) < 1e-11, (model, n1, n2, rel_l2(Jd, Jg))
    assert ran12
    p = dict(p, path_tb=tbgen.model_path("tmd11_s7"), nr1=14, nr2=8)
    out = []
    for env in ([], ["HHG_DFRAG=0"]):
        saved = os.environ.pop("HHG_DFRAG", None)
        os.environ.update(dict(k.split("=") for k in env))
        try:
            s = pyswe.SWE(pyswe.Settings(dict(p)), k_rows=(3, 9))
            s.run_simulation()
            out.append(np.stack(s.get_current()[1:]))
            s.delete()
        finally:
            os.environ.pop("HHG_DFRAG", None)
            if saved is not None:
                os.environ["HHG_DFRAG"] = saved
    assert rel_l2(out[0], out[1]) < 1e-11, rel_l2(out[0], out[1])


def test_fp64_fragment_kernel_kspace_solver():
    """The k-space solver's form of the FP64 fragment kernel (evaluation points t, t + dt/2, t + dt of
    the interpolation tables, the point t carried between steps, a constant window) against the
    element-group kernel on square grids, one and two field axes, a whole 64-step chunk and a ragged
    last chunk."""
    import tbgen

    for n, pol, tmax in ((10, [0.0, 1.0, 0.0], 3.0), (14, [0.6, 0.8, 0.0], 2.0)):
        p = {"path_tb": tbgen.model_path("tmd11_s7"), "nr1": n, "nr2": n, "nr3": 1, "tmax": tmax, "dt": 0.02197,
             "intensity": 2e12, "lambda": 3000.0, "tmax_field": 80.0, "pol_vec": np.array(pol),
             "phi_vec": np.zeros(3), "solver": "kspace"}
        Jd, _, shape = run(p, "fp64", [])
        Jg, _, _ = run(p, "fp64", ["HHG_DFRAG=0"])
        assert shape[3] == "propagate_dfrag_kernel", shape
        assert rel_l2(Jd, Jg) < 1e-11, (n, rel_l2(Jd, Jg))


@pytest.mark.parametrize("name", ["tmd11_10", "c2_prefix", "tmd11_12_full", "tmd12_12_full"])
def test_tile_kernel_against_element_groups_and_golden(name):
    """The mixed form's default kernel for 11- and 12-orbital models on a 7x7 box (half a warp per
    k-point, 3x3 register tiles) against the reference's current and the element-group kernel's, within
    the mixed form's 1e-6 (full pulses of 4096 steps included)."""
    _, param, _, J_ref = load_golden(name)
    Jt, n_t, shape = run(param, "mixed", [])
    assert shape[3] == "propagate_mtile_kernel", shape
    Jg, _, shape_g = run(param, "mixed", ["HHG_MTILE=0"])
    assert shape_g[3].startswith("propagate_group_kernel"), shape_g
    nt = Jt.shape[1]
    assert n_t == 2 * ((nt + 63) // 64) + 1
    assert rel_l2(Jt, J_ref) < 1e-6, rel_l2(Jt, J_ref)
    assert rel_l2(Jt, Jg) < 1e-6, rel_l2(Jt, Jg)


def test_tile_kernel_ragged_columns_two_axes_and_slabs():
    """Columns that do not divide into 8-k-point tiles (10 and 22 rows), non-square grids, two field
    axes (polarisation in the plane) with 11 and 12 orbitals, and a row slab, against the FP64 solve of
    the same case."""
    import tbgen
    from pySWE import pyswe

    for model, n1, n2 in (("tmd11_s7", 10, 10), ("tmd11_s7", 14, 8), ("tmd11_s7", 22, 10), ("tmd12_s3", 10, 12)):
        p = {"path_tb": tbgen.model_path(model), "nr1": n1, "nr2": n2, "nr3": 1, "tmax": 3.0, "dt": 0.02197,
             "intensity": 2e12, "lambda": 3000.0, "tmax_field": 80.0, "pol_vec": np.array([0.6, 0.8, 0.0]),
             "phi_vec": np.zeros(3)}
        Jt, _, shape = run(p, "mixed", [])
        J64, _, _ = run(p, "fp64", [])
        assert shape[1] == 8 and shape[3] == "propagate_mtile_kernel", shape
        assert rel_l2(Jt, J64) < 1e-6, (model, n1, n2, rel_l2(Jt, J64))
    # rows [3, 12) of a 14 x 8 grid: the slab's partial current against the FP64 slab's
    p = dict(p, nr1=14, nr2=8)
    out = []
    for precision in ("mixed", "fp64"):
        s = pyswe.SWE(pyswe.Settings(dict(p)), precision=precision, k_rows=(3, 12))
        if precision == "mixed":
            assert s.launch_shape()["kernel_name"] == "propagate_mtile_kernel"
        s.run_simulation()
        out.append(np.stack(s.get_current()[1:]))
        s.delete()
    assert rel_l2(out[0], out[1]) < 1e-6, rel_l2(out[0], out[1])


def test_tile_kernel_kspace_solver():
    """The k-space solver's form of the tile kernel (outer sums at t + dt/2 and t + dt per step, those
    at t carried from the previous step, a constant window) against the reference's current and the
    element-group kernel's; a pulse served in chunks that start on odd steps gives the same bits; two
    field axes and 12 orbitals (two CTAs per SM) against the FP64 solve."""
    import tbgen
    from pySWE import pyswe

    _, param, _, J_ref = load_golden("ks_tmd11_10")
    Jt, _, shape = run(param, "mixed", [])
    assert shape[3] == "propagate_mtile_kernel", shape
    Jg, _, shape_g = run(param, "mixed", ["HHG_MTILE=0"])
    assert shape_g[3].startswith("propagate_group_kernel"), shape_g
    assert rel_l2(Jt, J_ref) < 1e-6, rel_l2(Jt, J_ref)
    assert rel_l2(Jt, Jg) < 1e-6, rel_l2(Jt, Jg)
    p = {"path_tb": tbgen.model_path("tmd11_s7"), "nr1": 10, "nr2": 10, "nr3": 1, "tmax": 3.0, "dt": 0.02197,
         "intensity": 2e12, "lambda": 3000.0, "tmax_field": 80.0, "pol_vec": np.array([0.0, 1.0, 0.0]),
         "phi_vec": np.zeros(3), "solver": "kspace"}
    Jt, n_t, shape = run(p, "mixed", [])
    J64, _, _ = run(p, "fp64", [])
    assert shape[3] == "propagate_mtile_kernel", shape
    assert n_t == 2 * ((Jt.shape[1] + 63) // 64) + 1
    assert rel_l2(Jt, J64) < 1e-6, rel_l2(Jt, J64)
    srv = pyswe.SWEServer(device=0, chunk_steps=33)
    r = pyswe.SWE(pyswe.Settings(dict(p)), precision="mixed", solver="kspace", defer_init=True)
    tk = srv.submit(r)
    assert srv.wait(tk, timeout=120.0)
    assert np.array_equal(np.stack(r.get_current()[1:]), Jt)
    srv.close()
    for model, pol in (("tmd11_s7", [0.6, 0.8, 0.0]), ("tmd12_s3", [0.0, 1.0, 0.0]), ("tmd12_s3", [0.6, 0.8, 0.0])):
        p2 = dict(p, path_tb=tbgen.model_path(model), pol_vec=np.array(pol))
        J2, _, shape2 = run(p2, "mixed", [])
        J64, _, _ = run(p2, "fp64", [])
        assert shape2[3] == "propagate_mtile_kernel", (model, pol, shape2)
        assert rel_l2(J2, J64) < 1e-6, (model, pol, rel_l2(J2, J64))


@pytest.mark.parametrize("name", ["tmd6_8", "ks_tmd6_8"])
def test_tile_kernel_six_orbitals_against_golden(name):
    """The 6 x 6 frame of the tile kernel (4 lanes per k-point, 32 k-points per CTA) against the
    reference's current and the element-group kernel's (two field axes; the k-space solver's form)."""
    _, param, _, J_ref = load_golden(name)
    Jt, _, shape = run(param, "mixed", [])
    assert shape[3] == "propagate_mtile_kernel" and shape[1] == 32, shape
    Jg, _, shape_g = run(param, "mixed", ["HHG_MTILE=0"])
    assert shape_g[3].startswith("propagate_group_kernel"), shape_g
    assert rel_l2(Jt, J_ref) < 1e-6, rel_l2(Jt, J_ref)
    assert rel_l2(Jt, Jg) < 1e-6, rel_l2(Jt, Jg)


def test_tile_kernel_six_orbitals_ragged_columns_and_chunks():
    """Columns of 40 and 10 rows (tiles of 32 k-points: 32 + 8 and 10), one and two field axes, against
    the FP64 solve; a pulse served in chunks that start on odd steps gives the same bits."""
    import tbgen
    from pySWE import pyswe

    for n1, n2, pol in ((40, 8, [0.0, 1.0, 0.0]), (10, 12, [0.6, 0.8, 0.0])):
        p = {"path_tb": tbgen.model_path("tmd6_s1"), "nr1": n1, "nr2": n2, "nr3": 1, "tmax": 3.0, "dt": 0.02197,
             "intensity": 2e12, "lambda": 3000.0, "tmax_field": 80.0, "pol_vec": np.array(pol),
             "phi_vec": np.zeros(3)}
        Jt, n_t, shape = run(p, "mixed", [])
        J64, _, _ = run(p, "fp64", [])
        assert shape[3] == "propagate_mtile_kernel", shape
        assert n_t == 2 * ((Jt.shape[1] + 63) // 64) + 1
        assert rel_l2(Jt, J64) < 1e-6, (n1, n2, rel_l2(Jt, J64))
    srv = pyswe.SWEServer(device=0, chunk_steps=33)
    r = pyswe.SWE(pyswe.Settings(dict(p)), precision="mixed", defer_init=True)
    tk = srv.submit(r)
    assert srv.wait(tk, timeout=120.0)
    assert np.array_equal(np.stack(r.get_current()[1:]), Jt)
    srv.close()
