"""Host-side checks that need no GPU: the C-ABI library loads and exports every declared entry
point, fails loudly (no CPU fallback) without a device, and reports bad input as errors."""
import ctypes as ct
import os
import re

import numpy as np
import pytest

from conftest import REPO, REFERENCE_CHECKOUT, gpu_available, load_golden

LIB = os.path.join(REPO, "hhg-solids_b200", "lib", "libhhg_b200.so")
HEADER = os.path.join(REPO, "include", "hhg_swe.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(\w+)\s*\([^;{]*\)\s*;", text)))


def test_library_exports_every_declared_symbol():
    L = ct.CDLL(LIB)
    names = declared_functions()
    assert "SWESim_run_simulation" in names and "Settings_set_phi_vec" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing


def test_reference_surface_is_complete():
    """The 20 functions of the reference's src/cwrapper.cpp:7-27 are all declared."""
    ref = ["SWESim_new", "SWESim_run_simulation", "SWESim_test_files", "SWESim_set_path_tb", "SWESim_set_settings",
           "SWESim_init", "SWESim_restart", "SWESim_get_current", "SWESim_delete", "Settings_new",
           "Settings_set_nr1", "Settings_set_nr2", "Settings_set_nr3", "Settings_set_tmax", "Settings_set_dt",
           "Settings_set_intensity", "Settings_set_lambda", "Settings_set_tmax_field", "Settings_set_pol_vec",
           "Settings_set_phi_vec"]
    assert set(ref) <= set(declared_functions())
    if os.path.isdir(os.path.join(REFERENCE_CHECKOUT, "src")):
        text = open(os.path.join(REFERENCE_CHECKOUT, "src", "cwrapper.cpp")).read()
        text = "\n".join(l for l in text.splitlines() if not l.strip().startswith("//"))
        found = set(re.findall(r"\b((?:SWESim|Settings)_\w+)\s*\(", text))
        assert found == set(ref)


def _param(**over):
    _, param, _, _ = load_golden("haldane_8_y")
    param.update(over)
    return param


def test_missing_tb_file_raises_instead_of_aborting():
    from pySWE import pyswe

    with pytest.raises(pyswe.SWEError, match="tb file"):
        pyswe.SWE(pyswe.Settings(_param(path_tb="/nonexistent/model_tb.dat")))


@pytest.mark.parametrize("over,msg", [(dict(nr1=7), "even"), (dict(nr2=2), "even"), (dict(nr3=2), "2D"),
                                      (dict(tmax=0.01), "time steps")])
def test_bad_settings_raise(over, msg):
    from pySWE import pyswe

    with pytest.raises(pyswe.SWEError, match=msg):
        pyswe.SWE(pyswe.Settings(_param(**over)))


def test_malformed_tb_file_raises(tmp_path):
    from pySWE import pyswe

    bad = tmp_path / "bad_tb.dat"
    src = open(_param()["path_tb"]).read().splitlines()
    bad.write_text("\n".join(src[:40]) + "\n")
    with pytest.raises(pyswe.SWEError, match="TB file"):
        pyswe.SWE(pyswe.Settings(_param(path_tb=str(bad))))


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU behaviour")
def test_no_gpu_fails_loudly():
    from pySWE import pyswe

    with pytest.raises(pyswe.SWEError, match="no CUDA device"):
        pyswe.SWE(pyswe.Settings(_param()))


def test_null_and_uninitialised_objects_do_not_crash():
    L = ct.CDLL(LIB)
    L.SWESim_new.restype = ct.c_void_p
    L.SWESim_last_error.restype = ct.c_char_p
    L.SWESim_last_error.argtypes = [ct.c_void_p]
    L.HHG_last_error.restype = ct.c_char_p
    for name in ("SWESim_run_simulation", "SWESim_test_files", "SWESim_init", "SWESim_restart", "SWESim_delete",
                 "SWESim_reset"):
        getattr(L, name).argtypes = [ct.c_void_p]
    L.SWESim_run_simulation(None)
    assert b"null" in L.HHG_last_error()
    sim = L.SWESim_new()
    L.SWESim_run_simulation(sim)
    assert b"SWESim_init" in L.SWESim_last_error(sim)
    L.SWESim_init(sim)  # no settings
    assert b"settings" in L.SWESim_last_error(sim)
    L.SWESim_delete(sim)


def test_wrapper_drives_the_reference_build_too(oracle_mod):
    """The same Python classes run the reference's own library (same C ABI): drop-in both ways."""
    if not oracle_mod.have_ref():
        pytest.skip("reference build not present")
    from pySWE import pyswe

    from conftest import rel_l2

    meta, param, t_ref, J_ref = load_golden("haldane_8_y")
    param["path_lib"] = oracle_mod.ref_paths()[0]
    swe = pyswe.SWE(pyswe.Settings(param))
    swe.run_simulation()
    t, jx, jy, jz = swe.get_current()
    swe.delete()
    assert np.array_equal(np.real(t), t_ref)
    assert rel_l2(jy, J_ref[1]) < 1e-12


def test_reference_wrapper_binds_this_library():
    """The reference's unmodified pySWE/pyswe.py loads this library and binds every call
    (here without a GPU the calls report errors through SWESim_last_error, never abort)."""
    path = os.path.join(REFERENCE_CHECKOUT, "pySWE", "pyswe.py")
    if not os.path.exists(path):
        pytest.skip("reference checkout not present")
    import importlib.util

    spec = importlib.util.spec_from_file_location("reference_pyswe", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    param = _param(path_lib=LIB)
    settings = mod.Settings(param)
    swe = mod.SWE(settings)
    if not gpu_available():
        swe.run_simulation()
        t, jx, jy, jz = swe.get_current()
        assert np.all(t == 0)
    swe.delete()


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU behaviour")
def test_server_without_gpu_fails_loudly():
    from pySWE import pyswe

    with pytest.raises(pyswe.SWEError, match="no CUDA device"):
        pyswe.SWEServer()


def test_deferred_request_holds_no_device_state():
    """A request built for the server (defer_init) only records its settings: no device call."""
    from pySWE import pyswe

    swe = pyswe.SWE(pyswe.Settings(_param()), precision="mixed", defer_init=True)
    with pytest.raises(pyswe.SWEError, match="SWESim_init"):
        swe.get_current()
    swe.delete()


def test_kspace_solver_rejects_non_square_grids():
    from pySWE import pyswe

    with pytest.raises(pyswe.SWEError, match="nr1 == nr2"):
        pyswe.SWE(pyswe.Settings(_param(nr1=8, nr2=10)), solver="kspace")
    with pytest.raises(pyswe.SWEError, match="solver must be"):
        pyswe.SWE(pyswe.Settings(_param()), solver="fft")


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU behaviour")
def test_spectrum_without_gpu_fails_loudly():
    from pySWE import pyswe

    with pytest.raises(pyswe.SWEError, match="no CUDA device"):
        pyswe.spectrum(np.zeros((3, 16), dtype=complex), 0.1)


def test_wrapper_trace_is_the_reference_wrappers_traffic():
    """The committed wrapper traces are what the reference's pySWE/pyswe.py declares and calls today."""
    if not os.path.exists(os.path.join(REFERENCE_CHECKOUT, "pySWE", "pyswe.py")):
        pytest.skip("reference checkout not present")
    import json
    import sys

    sys.path.insert(0, os.path.join(REPO, "tests", "golden"))
    import make_wrapper_trace

    for name in make_wrapper_trace.CASES:
        with open(os.path.join(REPO, "tests", "golden", "wrapper_trace", f"{name}.json")) as f:
            committed = json.load(f)
        assert make_wrapper_trace.record(REFERENCE_CHECKOUT, name) == committed, name


def test_wrapper_trace_replay_reproduces_golden_on_reference_build(oracle_mod):
    """Replaying a recorded wrapper trace against the reference's own build gives its golden current:
    the replay is faithful, so the same replay against this library on a GPU is a drop-in check."""
    if not oracle_mod.have_ref():
        pytest.skip("reference build not present")
    import json

    from test_zy_reference_wrapper_gpu import TRACES, replay

    from conftest import rel_l2

    for name in ("tmd6_8", "haldane_12_pol"):
        with open(os.path.join(TRACES, f"{name}.json")) as f:
            trace = json.load(f)
        meta, param, t_ref, J_ref = load_golden(name)
        t, jx, jy, jz = replay(trace, oracle_mod.ref_paths()[0], param["path_tb"])
        assert np.array_equal(t, t_ref)
        for a, j in enumerate((jx, jy)):
            assert rel_l2(j, J_ref[a]) < 1e-12, (name, a)
