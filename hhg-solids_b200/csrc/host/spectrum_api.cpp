// HHG spectra on the device (the post-processing of the reference's scripts/pol_scan.py:34-40),
// for a solve's recorded current or for caller-supplied currents.
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "swe_sim.hpp"

using hhg::check_cuda;
using hhg::DevBuf;

namespace {

// S = fftshift(fft(ifftshift(gradient(J, h)))) for `count` host signals of length n.
void spectrum_host(const double2* J, int n, int count, double h, double2* S, cudaStream_t stream) {
  if (n < 2) throw std::runtime_error("spectrum: a signal needs at least 2 samples");
  if (count < 1) throw std::runtime_error("spectrum: no signals");
  if (!(h > 0.0)) throw std::runtime_error("spectrum: the sample spacing must be positive");
  const size_t total = (size_t)n * count;
  DevBuf<double2> dJ, dS, dT;
  dJ.alloc(total);
  dS.alloc(total);
  dT.alloc(total);
  check_cuda(cudaMemcpyAsync(dJ.p, J, sizeof(double2) * total, cudaMemcpyHostToDevice, stream), "H2D");
  if (hhg::spectrum_device(dJ.p, n, count, h, dS.p, dT.p, stream) < 0)
    throw std::runtime_error("spectrum: launch failed: " + std::string(cudaGetErrorString(cudaGetLastError())));
  check_cuda(cudaMemcpyAsync(S, dS.p, sizeof(double2) * total, cudaMemcpyDeviceToHost, stream), "D2H");
  check_cuda(cudaStreamSynchronize(stream), "spectrum");
}

int no_device_check(const char* name) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    throw std::runtime_error(std::string(name) + ": no CUDA device (this library has no CPU path)");
  return ndev;
}

}  // namespace

extern "C" {

int HHG_spectrum(const hhg_cdouble* J, int n, int count, double spacing, hhg_cdouble* S) {
  try {
    no_device_check("HHG_spectrum");
    if (!J || !S) throw std::runtime_error("HHG_spectrum: null buffer");
    spectrum_host(reinterpret_cast<const double2*>(J), n, count, spacing, reinterpret_cast<double2*>(S), nullptr);
    return 0;
  } catch (const std::exception& e) {
    hhg::set_thread_error(e.what());
    return -1;
  }
}

int HHG_harmonic_intensities(const hhg_cdouble* S, int n, int count, double tmax_fs, double lambda_nm, int nh,
                             double* I) {
  try {
    no_device_check("HHG_harmonic_intensities");
    if (!S || !I) throw std::runtime_error("HHG_harmonic_intensities: null buffer");
    if (n < 2 || count < 1 || nh < 1) throw std::runtime_error("HHG_harmonic_intensities: empty input");
    if (!(tmax_fs > 0.0) || !(lambda_nm > 0.0))
      throw std::runtime_error("HHG_harmonic_intensities: tmax and lambda must be positive");
    const size_t total = (size_t)n * count;
    DevBuf<double2> dS;
    DevBuf<double> dI;
    dS.alloc(total);
    dI.alloc((size_t)count * nh);
    check_cuda(cudaMemcpy(dS.p, S, sizeof(double2) * total, cudaMemcpyHostToDevice), "H2D");
    if (hhg::harmonics_device(dS.p, n, count, tmax_fs, lambda_nm, nh, dI.p, nullptr) != 0)
      throw std::runtime_error("HHG_harmonic_intensities: launch failed");
    check_cuda(cudaMemcpy(I, dI.p, sizeof(double) * (size_t)count * nh, cudaMemcpyDeviceToHost), "D2H");
    return 0;
  } catch (const std::exception& e) {
    hhg::set_thread_error(e.what());
    return -1;
  }
}

void SWESim_get_spectrum(SWESim* swe, double spacing, hhg_cdouble* sx, hhg_cdouble* sy, hhg_cdouble* sz) {
  try {
    if (!swe) throw std::runtime_error("SWESim_get_spectrum: null SWESim");
    swe->has_err = false;
    if (!swe->ready && !swe->served) throw std::runtime_error("SWESim_get_spectrum: SWESim_init has not succeeded");
    if ((int)swe->Jhist[0].size() < swe->nt)
      throw std::runtime_error("SWESim_get_spectrum: run_simulation has not been called");
    const int n = swe->nt;
    const double h = spacing > 0.0 ? spacing : swe->settings->dt;  // scripts/pol_scan.py:34 uses param["dt"]
    std::vector<double2> J((size_t)3 * n), S((size_t)3 * n);
    for (int a = 0; a < 3; ++a)
      for (int i = 0; i < n; ++i) J[(size_t)a * n + i] = make_double2(swe->Jhist[a][i].real(), swe->Jhist[a][i].imag());
    if (swe->device >= 0) check_cuda(cudaSetDevice(swe->device), "cudaSetDevice");
    spectrum_host(J.data(), n, 3, h, S.data(), swe->ready ? swe->stream : nullptr);
    hhg_cdouble* out[3] = {sx, sy, sz};
    for (int a = 0; a < 3; ++a)
      if (out[a])
        for (int i = 0; i < n; ++i) out[a][i] = hhg_cdouble{S[(size_t)a * n + i].x, S[(size_t)a * n + i].y};
  } catch (const std::exception& e) {
    hhg::set_thread_error(e.what());
    if (swe) {
      swe->err = e.what();
      swe->has_err = true;
    }
  }
}

}  // extern "C"
