"""Python API over ``libhhg_b200.so`` with the classes and parameter dict of the reference's
``pySWE/pyswe.py`` (rodrigomarher/HHG-Solids): ``Settings(param)`` and ``SWE(settings)`` with
``run_simulation``, ``get_current``, ``test_files``, ``restart``, ``delete``.

``param`` keys, as in the reference: ``path_lib``, ``path_tb``, ``nr1``, ``nr2``, ``nr3``, ``tmax``
(fs), ``dt`` (fs), ``intensity`` (W/cm^2), ``lambda`` (nm), ``tmax_field`` (fs), ``pol_vec`` and
``phi_vec`` (3 floats each).  ``path_lib`` may be omitted to use this package's library; any
library with the reference's C ABI works, including the reference's own build.

Error behaviour: the reference aborts the process on a bad TB path or settings (an exception
thrown through extern "C").  Here every call checks the library's last-error message and raises
:class:`SWEError` instead.  Against a library without ``SWESim_last_error`` (the reference's own
build) no check is possible and calls behave as in the reference.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_PKG = os.path.dirname(_HERE)

ND_POINTER_1_double = np.ctypeslib.ndpointer(dtype=np.float64, ndim=1, flags="C")
ND_POINTER_1_complex = np.ctypeslib.ndpointer(dtype=np.complex128, ndim=1, flags="C")
_libs: dict = {}


class SWEError(RuntimeError):
    """A call into the propagator library failed; the message is the library's."""


def default_library() -> str:
    return os.path.join(_PKG, "lib", "libhhg_b200.so")


def _load(path: str):
    path = os.path.abspath(path)
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise SWEError(f"propagator library not found: {path} (build it with `make -C hhg-solids_b200`)")
    L = ct.CDLL(path)
    vp = ct.c_void_p
    L.SWESim_new.argtypes = []
    L.SWESim_new.restype = vp
    for name in ("SWESim_run_simulation", "SWESim_test_files", "SWESim_init", "SWESim_restart", "SWESim_delete"):
        getattr(L, name).argtypes = [vp]
        getattr(L, name).restype = None
    L.SWESim_set_path_tb.argtypes = [vp, ct.c_char_p]
    L.SWESim_set_settings.argtypes = [vp, vp]
    L.SWESim_get_current.argtypes = [vp, ND_POINTER_1_double, ND_POINTER_1_complex, ND_POINTER_1_complex,
                                     ND_POINTER_1_complex]
    L.Settings_new.argtypes = []
    L.Settings_new.restype = vp
    for name in ("nr1", "nr2", "nr3"):
        getattr(L, f"Settings_set_{name}").argtypes = [vp, ct.c_int]
    for name in ("tmax", "dt", "intensity", "lambda", "tmax_field"):
        getattr(L, f"Settings_set_{name}").argtypes = [vp, ct.c_double]
    L.Settings_set_pol_vec.argtypes = [vp, ND_POINTER_1_double]
    L.Settings_set_phi_vec.argtypes = [vp, ND_POINTER_1_double]
    ext = hasattr(L, "SWESim_last_error")
    if ext:
        L.SWESim_last_error.argtypes = [vp]
        L.SWESim_last_error.restype = ct.c_char_p
        L.Settings_delete.argtypes = [vp]
        L.SWESim_get_nt.argtypes = [vp]
        L.SWESim_get_num_orb.argtypes = [vp]
        L.SWESim_set_device.argtypes = [vp, ct.c_int]
        L.SWESim_last_kernel_ms.argtypes = [vp]
        L.SWESim_last_kernel_ms.restype = ct.c_double
        L.SWESim_last_launches.argtypes = [vp]
        L.SWESim_last_propagate_ms.argtypes = [vp]
        L.SWESim_last_propagate_ms.restype = ct.c_double
        L.SWESim_h2d_bytes.argtypes = [vp]
        L.SWESim_h2d_bytes.restype = ct.c_longlong
        L.SWESim_launch_shape.argtypes = [vp] + [ct.POINTER(ct.c_int)] * 3 + [ct.POINTER(ct.c_longlong)]
        L.SWESim_reset.argtypes = [vp]
        L.SWESim_set_k_rows.argtypes = [vp, ct.c_int, ct.c_int]
        L.SWESim_set_precision.argtypes = [vp, ct.c_int]
        L.SWESim_set_solver.argtypes = [vp, ct.c_int]
        L.SWESim_set_tb_convention.argtypes = [vp, ct.c_int]
        L.SWESim_set_autotune.argtypes = [vp, ct.c_int]
        L.SWEBatch_new.restype = vp
        L.SWEBatch_add.argtypes = [vp, vp]
        L.SWEBatch_run.argtypes = [vp]
        L.SWEBatch_last_ms.argtypes = [vp]
        L.SWEBatch_last_ms.restype = ct.c_double
        L.SWEBatch_last_error.argtypes = [vp]
        L.SWEBatch_last_error.restype = ct.c_char_p
        L.SWEBatch_delete.argtypes = [vp]
        L.SWEServer_new.argtypes = [ct.c_int, ct.c_longlong, ct.c_int, ct.c_int]
        L.SWEServer_new.restype = vp
        L.SWEServer_submit.argtypes = [vp, vp]
        L.SWEServer_submit.restype = ct.c_longlong
        L.SWEServer_wait.argtypes = [vp, ct.c_longlong, ct.c_double]
        L.SWEServer_status.argtypes = [vp, ct.c_longlong]
        L.SWEServer_times.argtypes = [vp, ct.c_longlong, ND_POINTER_1_double]
        L.SWEServer_ticket_error.argtypes = [vp, ct.c_longlong]
        L.SWEServer_ticket_error.restype = ct.c_char_p
        L.SWEServer_stats.argtypes = [vp, ND_POINTER_1_double, ct.c_int]
        L.SWEServer_delete.argtypes = [vp]
        L.SWESim_get_spectrum.argtypes = [vp, ct.c_double, ND_POINTER_1_complex, ND_POINTER_1_complex,
                                           ND_POINTER_1_complex]
        L.HHG_spectrum.argtypes = [ND_POINTER_1_complex, ct.c_int, ct.c_int, ct.c_double, ND_POINTER_1_complex]
        L.HHG_harmonic_intensities.argtypes = [ND_POINTER_1_complex, ct.c_int, ct.c_int, ct.c_double, ct.c_double,
                                               ct.c_int, ND_POINTER_1_double]
        L.HHG_last_error.argtypes = []
        L.HHG_last_error.restype = ct.c_char_p
        L.SWESim_get_rho_k.argtypes = [vp, ND_POINTER_1_complex]
        L.SWESim_get_fields.argtypes = [vp, ND_POINTER_1_double, ND_POINTER_1_double, ND_POINTER_1_double]
    _libs[path] = (L, ext)
    return _libs[path]


class Settings:
    """Simulation parameters (include/settings.h of the reference); owns a C ``Settings``."""

    def __init__(self, param):
        self.path_lib = param.get("path_lib") or default_library()
        self.path_tb = param["path_tb"]
        self.nt = int(param["tmax"] / param["dt"])
        self.param = dict(param)
        self.settings_swe, self._ext = _load(self.path_lib)
        L = self.settings_swe
        self.ptr = L.Settings_new()
        L.Settings_set_nr1(self.ptr, int(param["nr1"]))
        L.Settings_set_nr2(self.ptr, int(param["nr2"]))
        L.Settings_set_nr3(self.ptr, int(param.get("nr3", 1)))
        L.Settings_set_tmax(self.ptr, float(param["tmax"]))
        L.Settings_set_dt(self.ptr, float(param["dt"]))
        L.Settings_set_intensity(self.ptr, float(param["intensity"]))
        L.Settings_set_lambda(self.ptr, float(param["lambda"]))
        L.Settings_set_tmax_field(self.ptr, float(param["tmax_field"]))
        L.Settings_set_pol_vec(self.ptr, np.ascontiguousarray(param["pol_vec"], dtype=np.float64))
        L.Settings_set_phi_vec(self.ptr, np.ascontiguousarray(param["phi_vec"], dtype=np.float64))

    def __del__(self):
        try:
            if self._ext and self.ptr:
                self.settings_swe.Settings_delete(self.ptr)
                self.ptr = None
        except Exception:
            pass


class SWE:
    """One propagation: setup on construction (SWESim_init), then run_simulation / get_current.
    ``defer_init=True`` skips the setup (for a request handed to :class:`SWEServer`).
    ``solver="kspace"`` selects the reference's k-space solver (src/solver_kspace.cpp) instead of
    its real-space one.  ``tb_convention="faithful"`` reads the TB file as Wannier90 defines it
    (degeneracy weights applied, orbital order kept) instead of as the reference does.
    ``autotune=True`` times a few tile shapes at setup and keeps the fastest."""

    _TB = {"reference": 0, "faithful": 3, "degeneracy": 1, "untransposed": 2}

    def __init__(self, settings: Settings, device: int | None = None, k_rows: tuple | None = None,
                 precision: str = "fp64", defer_init: bool = False, solver: str = "rspace",
                 tb_convention: str = "reference", autotune: bool = False):
        self.settings = settings
        self.swe_cpp, self._ext = _load(settings.path_lib)
        self.ptr = self.swe_cpp.SWESim_new()
        if not self.ptr:
            raise SWEError("SWESim_new failed")
        if device is not None:
            self._call("SWESim_set_device", int(device))
        if k_rows is not None:
            self._call("SWESim_set_k_rows", int(k_rows[0]), int(k_rows[1]))
        if precision not in ("fp64", "mixed"):
            raise SWEError(f"precision must be 'fp64' or 'mixed', not {precision!r}")
        if precision == "mixed":
            self._call("SWESim_set_precision", 1)
        if solver not in ("rspace", "kspace"):
            raise SWEError(f"solver must be 'rspace' or 'kspace', not {solver!r}")
        if solver == "kspace":
            self._call("SWESim_set_solver", 1)
        if tb_convention not in self._TB:
            raise SWEError(f"tb_convention must be one of {sorted(self._TB)}, not {tb_convention!r}")
        if self._TB[tb_convention]:
            self._call("SWESim_set_tb_convention", self._TB[tb_convention])
        if autotune:
            self._call("SWESim_set_autotune", 1)
        self.set_path_tb(settings.path_tb.encode("UTF-8"))
        self.set_settings(settings.ptr)
        if not defer_init:
            self.init()

    def _call(self, name, *args):
        if self.ptr is None:
            raise SWEError(f"{name}: SWE object already deleted")
        out = getattr(self.swe_cpp, name)(self.ptr, *args)
        if self._ext:
            msg = self.swe_cpp.SWESim_last_error(self.ptr)
            if msg:
                raise SWEError(msg.decode())
        return out

    # --- the reference's methods (pySWE/pyswe.py:37-57) ---
    def run_simulation(self):
        self._call("SWESim_run_simulation")

    def test_files(self):
        self._call("SWESim_test_files")

    def set_path_tb(self, val):
        self._call("SWESim_set_path_tb", val)

    def set_settings(self, val):
        self._call("SWESim_set_settings", val)

    def init(self):
        self._call("SWESim_init")

    def restart(self):
        self._call("SWESim_restart")

    def delete(self):
        if self.ptr is not None:
            self.swe_cpp.SWESim_delete(self.ptr)
            self.ptr = None

    def get_current(self):
        n = self.settings.nt
        t = np.zeros(n, dtype=np.float64)
        jx = np.zeros(n, dtype=np.complex128)
        jy = np.zeros(n, dtype=np.complex128)
        jz = np.zeros(n, dtype=np.complex128)
        self._call("SWESim_get_current", t, jx, jy, jz)
        return np.array([t, jx, jy, jz])

    # --- additions ---
    def reset(self):
        """Back to rho0 with an empty current record, keeping the setup."""
        self._call("SWESim_reset")

    def last_kernel_ms(self) -> float:
        return float(self.swe_cpp.SWESim_last_kernel_ms(self.ptr))

    def last_propagate_ms(self) -> float:
        return float(self.swe_cpp.SWESim_last_propagate_ms(self.ptr))

    def h2d_bytes(self) -> int:
        return int(self.swe_cpp.SWESim_h2d_bytes(self.ptr))

    def launch_shape(self) -> dict:
        c, t, k = ct.c_int(), ct.c_int(), ct.c_int()
        s = ct.c_longlong()
        kind = int(self.swe_cpp.SWESim_launch_shape(self.ptr, ct.byref(c), ct.byref(t), ct.byref(k), ct.byref(s)))
        names = {0: "propagate_kpt_kernel", 1: "propagate_group_kernel<double>", 2: "propagate_group_kernel<float>",
                 3: "propagate_kcol_kernel", 4: "propagate_frag_kernel", 5: "propagate_dfrag_kernel",
                 6: "propagate_mtile_kernel"}
        return {"ctas": c.value, "threads": t.value, "k_per_cta": k.value, "smem_bytes": s.value,
                "kernel_name": names.get(kind, "none")}

    def last_launches(self) -> int:
        return int(self.swe_cpp.SWESim_last_launches(self.ptr))

    def num_orb(self) -> int:
        return int(self.swe_cpp.SWESim_get_num_orb(self.ptr))

    def get_rho_k(self):
        nk = int(self.settings.param["nr1"]) * int(self.settings.param["nr2"])
        nw = self.num_orb()
        out = np.zeros(nk * nw * nw, dtype=np.complex128)
        self._call("SWESim_get_rho_k", out)
        return out.reshape(nk, nw * nw)

    def get_spectrum(self, spacing: float | None = None):
        """(hhg_x, hhg_y, hhg_z) = fftshift(fft(ifftshift(gradient(J, dt)))) per axis, computed on the
        GPU: the spectra of the reference's scripts/pol_scan.py:34-40 (dt = the settings' dt in fs)."""
        n = self.settings.nt
        out = [np.zeros(n, dtype=np.complex128) for _ in range(3)]
        self._call("SWESim_get_spectrum", float(spacing or 0.0), out[0], out[1], out[2])
        return out

    def get_fields(self):
        n = self.settings.nt
        t = np.zeros(n)
        E = np.zeros(3 * n)
        A = np.zeros(3 * n)
        self._call("SWESim_get_fields", t, E, A)
        return t, E.reshape(3, n), A.reshape(3, n)

    def __del__(self):
        try:
            self.delete()
        except Exception:
            pass


class SWEBatch:
    """Several SWE solves propagated together on one GPU (each from its equilibrium); every solve's
    current is then read with its own get_current() and equals, bit for bit, what it gives alone."""

    def __init__(self, solves):
        self.solves = list(solves)
        if not self.solves:
            raise SWEError("SWEBatch needs at least one solve")
        self.lib = self.solves[0].swe_cpp
        self.ptr = self.lib.SWEBatch_new()
        for s in self.solves:
            if self.lib.SWEBatch_add(self.ptr, s.ptr) < 0:
                raise SWEError("SWEBatch_add failed")

    def run(self):
        if self.lib.SWEBatch_run(self.ptr) != 0:
            msg = self.lib.SWEBatch_last_error(self.ptr)
            raise SWEError(msg.decode() if msg else "SWEBatch_run failed")

    def last_ms(self) -> float:
        return float(self.lib.SWEBatch_last_ms(self.ptr))

    def delete(self):
        if self.ptr is not None:
            self.lib.SWEBatch_delete(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.delete()
        except Exception:
            pass


class SWEServer:
    """Request loop with continuous batching on one GPU (``SWEServer_*`` of the library).

    ``submit(swe)`` queues a :class:`SWE` (built with ``defer_init=True``, or already set up) and
    returns a ticket; the server admits requests by device-memory footprint, runs the admitted ones
    together in chunks of ``chunk_steps`` RK4 steps, and completes each ticket when its pulse ends.
    ``wait(ticket)`` blocks until then; the solve's current is read with its own ``get_current()``.
    ``hbm_budget=0`` takes 80 % of the free device memory."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, max_active: int = 32, chunk_steps: int = 256,
                 path_lib: str | None = None):
        self.ptr = None
        self.lib, ext = _load(path_lib or default_library())
        if not ext:
            raise SWEError("SWEServer needs this package's library")
        self.ptr = self.lib.SWEServer_new(int(device), int(hbm_budget), int(max_active), int(chunk_steps))
        if not self.ptr:
            msg = self.lib.HHG_last_error()
            raise SWEError(msg.decode() if msg else "SWEServer_new failed")
        self._held = {}

    def submit(self, swe: SWE) -> int:
        t = int(self.lib.SWEServer_submit(self.ptr, swe.ptr))
        if t < 0:
            msg = self.lib.HHG_last_error()
            raise SWEError(msg.decode() if msg else "SWEServer_submit failed")
        self._held[t] = swe  # the SWESim and its Settings must outlive the request
        return t

    def wait(self, ticket: int, timeout: float | None = None) -> bool:
        """True when done, False on timeout; raises SWEError if the request failed."""
        rc = int(self.lib.SWEServer_wait(self.ptr, int(ticket), -1.0 if timeout is None else float(timeout)))
        if rc == 1:
            self._held.pop(ticket, None)
            return True
        if rc == 0:
            return False
        if rc == -2:
            raise SWEError(f"unknown ticket {ticket}")
        msg = self.lib.SWEServer_ticket_error(self.ptr, int(ticket))
        self._held.pop(ticket, None)
        raise SWEError(msg.decode() if msg else "request failed")

    _STATES = {0: "queued", 1: "setting up", 2: "running", 3: "done", -1: "failed", -2: "unknown"}

    def status(self, ticket: int) -> str:
        return self._STATES[int(self.lib.SWEServer_status(self.ptr, int(ticket)))]

    def times(self, ticket: int) -> dict:
        out = np.zeros(4)
        self.lib.SWEServer_times(self.ptr, int(ticket), out)
        return {"submit": out[0], "admit": out[1], "start": out[2], "done": out[3]}

    def stats(self) -> dict:
        out = np.zeros(12)
        self.lib.SWEServer_stats(self.ptr, out, 12)
        keys = ("completed", "failed", "chunks", "gpu_ms", "peak_running", "peak_bytes", "budget_bytes", "queued",
                "admitted", "gap_ms", "setup_ms", "finish_ms")
        return {k: (float(v) if k.endswith("_ms") else int(v)) for k, v in zip(keys, out)}

    def close(self):
        """Serves everything submitted, then stops the server."""
        if self.ptr is not None:
            self.lib.SWEServer_delete(self.ptr)
            self.ptr = None
            self._held.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _check(lib, rc, name):
    if rc != 0:
        msg = lib.HHG_last_error()
        raise SWEError(msg.decode() if msg else f"{name} failed")


def spectrum(J, spacing: float, path_lib: str | None = None):
    """fftshift(fft(ifftshift(gradient(J, spacing)))) along the last axis of J, on the GPU."""
    lib, _ = _load(path_lib or default_library())
    J = np.ascontiguousarray(J, dtype=np.complex128)
    shape = J.shape
    flat = J.reshape(-1, shape[-1])
    out = np.zeros_like(flat)
    _check(lib, lib.HHG_spectrum(flat.reshape(-1), flat.shape[1], flat.shape[0], float(spacing), out.reshape(-1)),
           "HHG_spectrum")
    return out.reshape(shape)


def harmonic_intensities(S, tmax: float, lam: float, n_harmonics: int, path_lib: str | None = None):
    """|S|^2 summed over the odd harmonic orders 1, 3, ..., 2 n - 1 (windows of +-1/2 on pol_scan's
    order axis), on the GPU; returns [..., n_harmonics]."""
    lib, _ = _load(path_lib or default_library())
    S = np.ascontiguousarray(S, dtype=np.complex128)
    flat = S.reshape(-1, S.shape[-1])
    out = np.zeros((flat.shape[0], int(n_harmonics)))
    _check(lib, lib.HHG_harmonic_intensities(flat.reshape(-1), flat.shape[1], flat.shape[0], float(tmax), float(lam),
                                             int(n_harmonics), out.reshape(-1)), "HHG_harmonic_intensities")
    return out.reshape(S.shape[:-1] + (int(n_harmonics),))
