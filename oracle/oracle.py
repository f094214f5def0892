"""ctypes access to the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``liboracle.so`` (the plain-C restatement in ``sbe_oracle.c``) and, when present, the
reference build ``_ref/libwannier.so`` / ``_ref/libref_probe.so`` made by ``oracle/Makefile``.
Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import this
module, and only as the checker.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
_probe = None


class OracleSettings(ct.Structure):
    _fields_ = [
        ("nr1", ct.c_int), ("nr2", ct.c_int), ("nr3", ct.c_int),
        ("tmax", ct.c_double), ("dt", ct.c_double), ("intensity", ct.c_double),
        ("lambda_nm", ct.c_double), ("tmax_field", ct.c_double),
        ("pol", ct.c_double * 3), ("phi", ct.c_double * 3),
        ("tb_flags", ct.c_int),
    ]


def settings(param: dict) -> OracleSettings:
    """Build the C settings struct from a pySWE-style parameter dict."""
    s = OracleSettings()
    s.nr1, s.nr2, s.nr3 = int(param["nr1"]), int(param["nr2"]), int(param.get("nr3", 1))
    s.tmax, s.dt = float(param["tmax"]), float(param["dt"])
    s.intensity, s.lambda_nm = float(param["intensity"]), float(param["lambda"])
    s.tmax_field = float(param["tmax_field"])
    for i in range(3):
        s.pol[i] = float(param["pol_vec"][i])
        s.phi[i] = float(param["phi_vec"][i])
    s.tb_flags = {"reference": 0, "faithful": 3}[param.get("tb_convention", "reference")]
    return s


def build() -> None:
    """Compile liboracle.so (and the reference build when its sources are present)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ct.CDLL(path)
        P = ct.POINTER(OracleSettings)
        dp = ct.POINTER(ct.c_double)
        L.oracle_nt.argtypes = [P]
        L.oracle_model_info.argtypes = [ct.c_char_p, ct.POINTER(ct.c_int), ct.POINTER(ct.c_int)]
        L.oracle_fields.argtypes = [ct.c_char_p, P, dp, dp, dp]
        L.oracle_place.argtypes = [ct.c_char_p, P, dp, dp]
        L.oracle_velocity_window.argtypes = [ct.c_char_p, P, dp]
        L.oracle_rho0.argtypes = [ct.c_char_p, P, dp]
        L.oracle_run.argtypes = [ct.c_char_p, P, ct.c_int, ct.c_int, dp, dp]
        L.oracle_run_steps.argtypes = [ct.c_char_p, P, ct.c_int, ct.c_int, ct.c_int, dp, dp]
        L.oracle_run_kspace_steps.argtypes = [ct.c_char_p, P, ct.c_int, dp, dp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ct.POINTER(ct.c_double))


def model_info(tb: str):
    nw, ns = ct.c_int(), ct.c_int()
    if lib().oracle_model_info(tb.encode(), ct.byref(nw), ct.byref(ns)) != 0:
        raise FileNotFoundError(tb)
    return nw.value, ns.value


def nt(param: dict) -> int:
    s = settings(param)
    return lib().oracle_nt(ct.byref(s))


def fields(tb: str, param: dict):
    s = settings(param)
    n = lib().oracle_nt(ct.byref(s))
    t = np.zeros(n)
    E = np.zeros((3, n))
    A = np.zeros((3, n))
    if lib().oracle_fields(tb.encode(), ct.byref(s), _dp(t), _dp(E), _dp(A)) != n:
        raise ValueError("oracle_fields failed")
    return t, E, A


def place(tb: str, param: dict):
    s = settings(param)
    nw, _ = model_info(tb)
    nk = s.nr1 * s.nr2
    H = np.zeros((nk, nw * nw), dtype=np.complex128)
    r3 = np.zeros((3, nk, nw * nw), dtype=np.complex128)
    if lib().oracle_place(tb.encode(), ct.byref(s), _dp(H), _dp(r3)) != nw:
        raise ValueError("oracle_place failed")
    return H, r3


def velocity_window(tb: str, param: dict):
    s = settings(param)
    nw, _ = model_info(tb)
    v = np.zeros((3, 16, nw * nw), dtype=np.complex128)
    if lib().oracle_velocity_window(tb.encode(), ct.byref(s), _dp(v)) != nw:
        raise ValueError("oracle_velocity_window failed")
    return v


def rho0(tb: str, param: dict):
    s = settings(param)
    nw, _ = model_info(tb)
    rho = np.zeros((s.nr1 * s.nr2, nw * nw), dtype=np.complex128)
    if lib().oracle_rho0(tb.encode(), ct.byref(s), _dp(rho)) != nw:
        raise ValueError("oracle_rho0 failed")
    return rho


def run(tb: str, param: dict, k_begin: int = 0, k_end: int | None = None, nsteps: int = -1):
    """Propagate; returns (t, J[3, nt]) with J the (partial, if a k-range is given) current.

    ``nsteps`` >= 0 stops after that many steps (the later samples stay zero)."""
    s = settings(param)
    n = lib().oracle_nt(ct.byref(s))
    if k_end is None:
        k_end = s.nr1 * s.nr2
    t = np.zeros(n)
    J = np.zeros((3, n), dtype=np.complex128)
    got = lib().oracle_run_steps(tb.encode(), ct.byref(s), int(k_begin), int(k_end), int(nsteps), _dp(t), _dp(J))
    if got != n:
        raise ValueError(f"oracle_run failed ({got})")
    return t, J


def run_kspace(tb: str, param: dict, nsteps: int = -1):
    """The reference's k-space solver (src/solver_kspace.cpp) restated; returns (t, J[3, nt])."""
    s = settings(param)
    n = lib().oracle_nt(ct.byref(s))
    t = np.zeros(n)
    J = np.zeros((3, n), dtype=np.complex128)
    got = lib().oracle_run_kspace_steps(tb.encode(), ct.byref(s), int(nsteps), _dp(t), _dp(J))
    if got != n:
        raise ValueError(f"oracle_run_kspace_steps failed ({got})")
    return t, J


# ---------------------------------------------------------------- the reference's own build


def ref_paths():
    return os.path.join(HERE, "_ref", "libwannier.so"), os.path.join(HERE, "_ref", "libref_probe.so")


def have_ref() -> bool:
    return all(os.path.exists(p) for p in ref_paths())


def probe():
    global _probe
    if _probe is None:
        P = ct.CDLL(ref_paths()[1])
        dp = ct.POINTER(ct.c_double)
        P.probe_nt.argtypes = [ct.c_double, ct.c_double]
        P.probe_fields.argtypes = [ct.c_char_p, ct.c_int, ct.c_int] + [ct.c_double] * 5 + [dp] * 5
        P.probe_operators.argtypes = [ct.c_char_p, ct.c_int, ct.c_int, dp, dp, dp]
        P.probe_rho0.argtypes = [ct.c_char_p, ct.c_int, ct.c_int, dp, dp]
        P.probe_kspace_run.argtypes = [ct.c_char_p, ct.c_int, ct.c_int] + [ct.c_double] * 5 + [dp, dp, ct.c_int,
                                                                                              dp, dp]
        _probe = P
    return _probe


def ref_fields(tb: str, param: dict):
    P = probe()
    n = P.probe_nt(float(param["tmax"]), float(param["dt"]))
    t = np.zeros(n)
    E = np.zeros((3, n))
    A = np.zeros((3, n))
    pol = np.ascontiguousarray(param["pol_vec"], dtype=np.float64)
    phi = np.ascontiguousarray(param["phi_vec"], dtype=np.float64)
    P.probe_fields(tb.encode(), int(param["nr1"]), int(param["nr2"]), float(param["tmax"]), float(param["dt"]),
                   float(param["intensity"]), float(param["lambda"]), float(param["tmax_field"]), _dp(pol),
                   _dp(phi), _dp(t), _dp(E), _dp(A))
    return t, E, A


def ref_operators(tb: str, n1: int, n2: int):
    nw, _ = model_info(tb)
    nk = n1 * n2
    H = np.zeros((nk, nw * nw), dtype=np.complex128)
    r3 = np.zeros((3, nk, nw * nw), dtype=np.complex128)
    v3 = np.zeros((3, nk, nw * nw), dtype=np.complex128)
    probe().probe_operators(tb.encode(), n1, n2, _dp(H), _dp(r3), _dp(v3))
    return H, r3, v3


def ref_rho0(tb: str, n1: int, n2: int):
    nw, _ = model_info(tb)
    rho = np.zeros((n1 * n2, nw * nw), dtype=np.complex128)
    Hk = np.zeros((n1 * n2, nw * nw), dtype=np.complex128)
    probe().probe_rho0(tb.encode(), n1, n2, _dp(rho), _dp(Hk))
    return rho, Hk


def window_cells(n1: int, n2: int):
    """Flattened grid indices of the 4x4 current window, window order w = (n1+2)*4 + (n2+2)."""
    return [(n1 // 2 + a) * n2 + (n2 // 2 + b) for a in range(-2, 2) for b in range(-2, 2)]


def ref_run(tb: str, param: dict, lib_path: str | None = None):
    """Run the reference's own build through its C ABI (src/cwrapper.cpp:5-28); returns (t, J[3, nt])."""
    L = ct.CDLL(lib_path or ref_paths()[0])
    vp = ct.c_void_p
    L.SWESim_new.restype = vp
    L.Settings_new.restype = vp
    for name in ["SWESim_run_simulation", "SWESim_init", "SWESim_delete"]:
        getattr(L, name).argtypes = [vp]
    L.SWESim_set_path_tb.argtypes = [vp, ct.c_char_p]
    L.SWESim_set_settings.argtypes = [vp, vp]
    dp = ct.POINTER(ct.c_double)
    L.SWESim_get_current.argtypes = [vp, dp, dp, dp, dp]
    for name in ["nr1", "nr2", "nr3"]:
        getattr(L, f"Settings_set_{name}").argtypes = [vp, ct.c_int]
    for name in ["tmax", "dt", "intensity", "lambda", "tmax_field"]:
        getattr(L, f"Settings_set_{name}").argtypes = [vp, ct.c_double]
    L.Settings_set_pol_vec.argtypes = [vp, dp]
    L.Settings_set_phi_vec.argtypes = [vp, dp]
    s = L.Settings_new()
    L.Settings_set_nr1(s, int(param["nr1"]))
    L.Settings_set_nr2(s, int(param["nr2"]))
    L.Settings_set_nr3(s, int(param.get("nr3", 1)))
    for name, key in [("tmax", "tmax"), ("dt", "dt"), ("intensity", "intensity"), ("lambda", "lambda"),
                      ("tmax_field", "tmax_field")]:
        getattr(L, f"Settings_set_{name}")(s, float(param[key]))
    pol = np.ascontiguousarray(param["pol_vec"], dtype=np.float64)
    phi = np.ascontiguousarray(param["phi_vec"], dtype=np.float64)
    L.Settings_set_pol_vec(s, _dp(pol))
    L.Settings_set_phi_vec(s, _dp(phi))
    sim = L.SWESim_new()
    L.SWESim_set_path_tb(sim, tb.encode())
    L.SWESim_set_settings(sim, s)
    L.SWESim_init(sim)
    L.SWESim_run_simulation(sim)
    n = int(float(param["tmax"]) / float(param["dt"]))
    t = np.zeros(n)
    J = np.zeros((3, n), dtype=np.complex128)
    L.SWESim_get_current(sim, _dp(t), _dp(J[0]), _dp(J[1]), _dp(J[2]))
    L.SWESim_delete(sim)
    return t, J


def ref_kspace_run(tb: str, param: dict, nsteps: int = -1):
    """The reference's own Solver_kspace, driven step by step (ref_probe.cpp); returns (t, J[3, nt])."""
    P = probe()
    n = P.probe_nt(float(param["tmax"]), float(param["dt"]))
    t = np.zeros(n)
    J = np.zeros((3, n), dtype=np.complex128)
    pol = np.ascontiguousarray(param["pol_vec"], dtype=np.float64)
    phi = np.ascontiguousarray(param["phi_vec"], dtype=np.float64)
    got = P.probe_kspace_run(tb.encode(), int(param["nr1"]), int(param["nr2"]), float(param["tmax"]),
                             float(param["dt"]), float(param["intensity"]), float(param["lambda"]),
                             float(param["tmax_field"]), _dp(pol), _dp(phi), int(nsteps), _dp(t), _dp(J))
    if got != n:
        raise ValueError(f"probe_kspace_run failed ({got})")
    return t, J
