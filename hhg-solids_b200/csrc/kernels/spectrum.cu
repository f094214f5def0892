// HHG spectrum of a current on the device: the recipe of the reference's scripts/pol_scan.py:34-40,
//   S = fftshift(fft(ifftshift(gradient(J, h))))      (numpy semantics, h = sample spacing)
// and the harmonic intensities of its order axis (scripts/pol_scan.py:50-57):
//   order_i = linspace(-wmax, wmax, n)_i / w0,  wmax = n pi / tmax,  w0 = 2 pi 300 / lambda_nm,
//   I_h = sum over order_i in (h - 1/2, h + 1/2) of |S_i|^2   for odd h.
//
// The FFT is a batched mixed-radix Stockham transform (autosorting, so no bit reversal): n is
// factored into radices 4, 2, 3, 5 and any remaining prime, and each pass reads the previous pass's
// buffer and writes the other.  For a pass of radix R after a product Ns of earlier radices, thread
// j (of n/R) takes the R inputs j + r n/R, multiplies input r by e^{-2 pi i r (j mod Ns) / (Ns R)},
// forms their length-R DFT and writes output q to (j div Ns) Ns R + (j mod Ns) + q Ns.  The first pass
// reads the gradient of the current through the ifftshift, the last one writes through the fftshift.
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "sbe_device.h"

namespace hhg {
namespace {

__device__ __forceinline__ double2 sp_mul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

// e^{-2 pi i num / den} for 0 <= num < den.
__device__ __forceinline__ double2 sp_twiddle(long long num, long long den) {
  double s, c;
  sincospi(-2.0 * (double)num / (double)den, &s, &c);
  return make_double2(c, s);
}

// numpy.gradient (second-order central differences inside, first-order at the ends, the same
// divisions as numpy) of a signal at index i, read through ifftshift: element i of ifftshift(g) is
// g[(i + n/2) mod n].
__device__ __forceinline__ double2 sp_grad_shifted(const double2* J, int n, int i, double h) {
  const int g = (i + n / 2) % n;
  if (g == 0) return make_double2((J[1].x - J[0].x) / h, (J[1].y - J[0].y) / h);
  if (g == n - 1) return make_double2((J[n - 1].x - J[n - 2].x) / h, (J[n - 1].y - J[n - 2].y) / h);
  const double h2 = 2.0 * h;
  return make_double2((J[g + 1].x - J[g - 1].x) / h2, (J[g + 1].y - J[g - 1].y) / h2);
}

__device__ __forceinline__ double2 sp_fma(double2 a, double2 w, double2 acc) {
  return make_double2(fma(a.x, w.x, fma(-a.y, w.y, acc.x)), fma(a.x, w.y, fma(a.y, w.x, acc.y)));
}

// One Stockham pass of radix R over `count` signals of length n.  first: read gradients of J
// through the ifftshift; last: write through the fftshift.
__global__ void stockham_pass_kernel(const double2* in, double2* out, const double2* J, int n, int count, int R,
                                     int Ns, int first, int last, double h) {
  const long long total = (long long)count * (n / R);
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= total) return;
  const int b = (int)(gid / (n / R)), j = (int)(gid % (n / R));
  const double2* src = first ? nullptr : in + (size_t)b * n;
  const double2* Jb = J + (size_t)b * n;
  double2* dst = out + (size_t)b * n;
  const int k = j % Ns, stride = n / R;
  const int base = (j / Ns) * Ns * R + k;
  const long long span = (long long)Ns * R;
  auto input = [&](int r) {
    const double2 x = first ? sp_grad_shifted(Jb, n, j + r * stride, h) : src[j + r * stride];
    return r == 0 ? x : sp_mul(x, sp_twiddle((long long)r * k % span, span));
  };
  auto store = [&](int q, double2 acc) {
    const int o = base + q * Ns;
    dst[last ? (o + n / 2) % n : o] = acc;  // fftshift: element i of the result is X[(i - n/2) mod n]
  };
  constexpr int kMaxReg = 8;
  if (R <= kMaxReg) {
    double2 v[kMaxReg];
    for (int r = 0; r < R; ++r) v[r] = input(r);
    for (int q = 0; q < R; ++q) {
      double2 acc = v[0];
      for (int r = 1; r < R; ++r) acc = sp_fma(v[r], sp_twiddle((long long)r * q % R, R), acc);
      store(q, acc);
    }
  } else {
    // Large prime radix: direct DFT, inputs re-read for every output.
    for (int q = 0; q < R; ++q) {
      double2 acc = make_double2(0.0, 0.0);
      for (int r = 0; r < R; ++r) acc = sp_fma(input(r), sp_twiddle((long long)r * q % R, R), acc);
      store(q, acc);
    }
  }
}

// I[b][h'] for odd harmonics h = 2 h' + 1: sum of |S|^2 over order in (h - 1/2, h + 1/2).
__global__ void harmonics_kernel(const double2* S, int n, int count, double tmax, double w0, int nh, double* I) {
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= count * nh) return;
  const int b = gid / nh, hh = gid % nh;
  const double h = 2.0 * hh + 1.0;
  const double wmax = n * (2.0 * M_PI / tmax) / 2.0;
  const double step = n > 1 ? 2.0 * wmax / (double)(n - 1) : 0.0;
  double acc = 0.0;
  for (int i = 0; i < n; ++i) {
    const double order = (-wmax + step * i) / w0;
    if (order > h - 0.5 && order < h + 0.5) {
      const double2 s = S[(size_t)b * n + i];
      acc += s.x * s.x + s.y * s.y;
    }
  }
  I[gid] = acc;
}

std::vector<int> factor_radices(int n) {
  std::vector<int> f;
  while (n % 4 == 0) {
    f.push_back(4);
    n /= 4;
  }
  for (int p : {2, 3, 5}) {
    while (n % p == 0) {
      f.push_back(p);
      n /= p;
    }
  }
  for (int p = 7; (long long)p * p <= n; p += 2)
    while (n % p == 0) {
      f.push_back(p);
      n /= p;
    }
  if (n > 1) f.push_back(n);
  return f;
}

}  // namespace

int spectrum_device(const double2* J, int n, int count, double h, double2* S, double2* scratch, cudaStream_t stream) {
  if (n < 2 || count < 1 || h <= 0.0) return -1;
  const std::vector<int> rad = factor_radices(n);
  // Ping-pong between S and scratch so that the last pass lands in S.
  const int passes = (int)rad.size();
  double2* bufs[2] = {S, scratch};
  int cur = passes % 2 == 1 ? 0 : 1;  // buffer written by the first pass
  int Ns = 1;
  const double2* prev = nullptr;
  for (int p = 0; p < passes; ++p) {
    const int R = rad[p];
    const long long threads = (long long)count * (n / R);
    const int block = 128;
    const int grid = (int)((threads + block - 1) / block);
    stockham_pass_kernel<<<grid, block, 0, stream>>>(prev, bufs[cur], J, n, count, R, Ns, p == 0, p == passes - 1, h);
    prev = bufs[cur];
    cur ^= 1;
    Ns *= R;
  }
  return cudaGetLastError() == cudaSuccess ? passes : -1;
}

int harmonics_device(const double2* S, int n, int count, double tmax, double lambda_nm, int nh, double* I,
                     cudaStream_t stream) {
  if (n < 2 || count < 1 || nh < 1 || tmax <= 0.0 || lambda_nm <= 0.0) return -1;
  const double w0 = 2.0 * M_PI * 300.0 / lambda_nm;
  const int total = count * nh;
  harmonics_kernel<<<(total + 127) / 128, 128, 0, stream>>>(S, n, count, tmax, w0, nh, I);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace hhg
