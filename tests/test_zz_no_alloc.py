"""SWESim_run_simulation_noalloc: the propagation for callers that must not allocate GPU memory
(their device memory belongs to another framework's pool, or a cudaFree's device-wide
synchronisation would stall their other streams).  It keeps its scratch in a fixed 32 MiB device
array owned by the library, so the caller passes only the state and the result buffers.

Checked here through the C ABI: two calls in a row give the current of the allocating entry point
(SWESim_run_simulation), for each of the three propagation kernels, and a solve that needs more
scratch than the array holds is refused with a message.  This file is collected last on purpose."""
import ctypes as ct

import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-10  # the relative L2 bar of the other parity tests


def _lib():
    from pySWE import pyswe

    L = ct.CDLL(pyswe.default_library())
    L.SWESim_run_simulation_noalloc.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    L.SWESim_run_simulation_noalloc.restype = ct.c_int
    L.SWESim_last_error.argtypes = [ct.c_void_p]
    L.SWESim_last_error.restype = ct.c_char_p
    return L


# (golden case, tmax override, HHG_KERNEL, expected kernel): the thread-per-k-point kernel, the
# element-group kernel (precomputed-sum shape), the column-tile kernel on the 200 x 200 2-orbital grid
# it is chosen for (a short pulse, within the scratch limit), and the column-tile kernel forced on a
# small grid.
CASES = [("haldane_12_pol", None, None, "propagate_kpt_kernel"),
         ("tmd11_10", None, None, "propagate_"),
         ("c1", 2.2, None, "propagate_kcol_kernel"),
         ("haldane_12_pol", None, "kcol", "propagate_kcol_kernel")]


@pytest.mark.parametrize("name,tmax,kernel,expect", CASES)
def test_two_calls_match_the_allocating_entry_point(name, tmax, kernel, expect, monkeypatch):
    import torch
    from pySWE import pyswe

    meta, param, _, _ = load_golden(name)
    if tmax:
        param = dict(param, tmax=tmax)
    if kernel:
        monkeypatch.setenv("HHG_KERNEL", kernel)  # read at SWESim_init
    swe = pyswe.SWE(pyswe.Settings(param), device=0)
    monkeypatch.delenv("HHG_KERNEL", raising=False)
    assert swe.launch_shape()["kernel_name"].startswith(expect), swe.launch_shape()
    rho0 = swe.get_rho_k()  # equilibrium, before any propagation
    swe.run_simulation()
    J_alloc = swe.get_current()[1:]
    nt = swe.settings.nt
    L = _lib()
    stream = torch.cuda.current_stream(torch.device("cuda", 0))
    for call in range(2):
        rho = torch.from_numpy(rho0.copy()).to("cuda:0")
        cur = torch.full((3, nt), complex(float("nan"), float("nan")), dtype=torch.complex128, device="cuda:0")
        rc = L.SWESim_run_simulation_noalloc(swe.ptr, rho.data_ptr(), cur.data_ptr(), stream.cuda_stream)
        assert rc == 0, L.SWESim_last_error(swe.ptr)
        torch.cuda.synchronize()
        J = cur.cpu().numpy()
        for a in range(3):
            if np.abs(J_alloc[a]).max() == 0:
                assert np.abs(J[a]).max() == 0, (call, a)
            else:
                assert rel_l2(J[a], J_alloc[a]) < TOL, (call, a, rel_l2(J[a], J_alloc[a]))
    swe.delete()


def test_refuses_a_solve_beyond_its_scratch():
    import torch
    from pySWE import pyswe

    _, param, _, _ = load_golden("haldane_8_y")
    param = dict(param, nr1=100, nr2=100, tmax=176.0)  # about 100 CTAs x 8010 steps x 48 B > 32 MiB
    swe = pyswe.SWE(pyswe.Settings(param), device=0)
    nt = swe.settings.nt
    rho = torch.zeros((100 * 100, 4), dtype=torch.complex128, device="cuda:0")
    cur = torch.zeros((3, nt), dtype=torch.complex128, device="cuda:0")
    L = _lib()
    rc = L.SWESim_run_simulation_noalloc(swe.ptr, rho.data_ptr(), cur.data_ptr(), None)
    assert rc == -1
    assert b"scratch" in L.SWESim_last_error(swe.ptr)
    swe.delete()
