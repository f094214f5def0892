"""HHG spectra on the device against the reference's own recipe, run in numpy
(scripts/pol_scan.py:34-40: fftshift(fft(ifftshift(gradient(J, dt))))) and its order axis
(scripts/pol_scan.py:50-57)."""
import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu


def numpy_spectrum(J, dt):
    return np.fft.fftshift(np.fft.fft(np.fft.ifftshift(np.gradient(J, dt, axis=-1), axes=-1), axis=-1), axes=-1)


def numpy_harmonics(S, tmax, lam, nh):
    n = S.shape[-1]
    dw = 2.0 * np.pi / tmax
    order = np.linspace(-n * dw / 2.0, n * dw / 2.0, n) / (2.0 * np.pi * 300 / lam)
    out = np.zeros(S.shape[:-1] + (nh,))
    for k in range(nh):
        h = 2 * k + 1
        win = (order > h - 0.5) & (order < h + 0.5)
        out[..., k] = (np.abs(S[..., win]) ** 2).sum(axis=-1)
    return out


@pytest.mark.parametrize("n", [2, 5, 54, 97, 182, 1000, 4095, 4096])
def test_spectrum_matches_numpy_any_length(n):
    from pySWE import pyswe

    rng = np.random.default_rng(n)
    J = rng.standard_normal((3, n)) + 1j * rng.standard_normal((3, n))
    S = pyswe.spectrum(J, 0.02197)
    ref = numpy_spectrum(J, 0.02197)
    for a in range(3):
        assert rel_l2(S[a], ref[a]) < 1e-13, (n, a, rel_l2(S[a], ref[a]))


@pytest.mark.parametrize("name", ["c0", "haldane_12_pol", "ks_c0"])
def test_solve_spectrum_and_harmonics(name):
    from pySWE import pyswe

    _, param, _, J_ref = load_golden(name)
    s = pyswe.SWE(pyswe.Settings(dict(param)), solver=param.get("solver", "rspace"))
    s.run_simulation()
    J = s.get_current()[1:]
    spec = np.array(s.get_spectrum())
    s.delete()
    ref = numpy_spectrum(J, param["dt"])
    for a in range(2):
        assert rel_l2(spec[a], ref[a]) < 1e-13
    assert np.abs(spec[2]).max() == 0
    # against the reference's own current: the spectrum parity of the propagation itself
    ref_spec = numpy_spectrum(J_ref, param["dt"])
    axis = int(np.argmax(np.linalg.norm(J_ref, axis=1)))
    assert rel_l2(spec[axis], ref_spec[axis]) < 1e-10
    I = pyswe.harmonic_intensities(spec[:2], param["tmax"], param["lambda"], 20)
    I_ref = numpy_harmonics(ref[:2], param["tmax"], param["lambda"], 20)
    assert I.shape == I_ref.shape
    nz = I_ref > 0
    assert np.all(np.abs(I[nz] - I_ref[nz]) <= 1e-12 * I_ref[nz] + 1e-300)
    assert np.array_equal(I[~nz], I_ref[~nz])
