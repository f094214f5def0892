// Warp reductions of the current partials.
#pragma once

#include <cuda_runtime.h>

namespace hhg {

// Sums four values over the 32 lanes of a warp with 12 shuffles instead of 4 x 10: at each of the
// first two levels every lane keeps half of its values and sends the other half to its partner, so
// afterwards each lane carries one of the four partial sums, reduced over the remaining three levels.
// Lane 8c (c < 4) returns the sum of value c; the other lanes return partial sums.
__device__ __forceinline__ double warp_sum4(double v0, double v1, double v2, double v3, int lane) {
  const bool hi = (lane & 16) != 0, h8 = (lane & 8) != 0;
  double a = hi ? v2 : v0, b = hi ? v3 : v1;
  const double sa = hi ? v0 : v2, sb = hi ? v1 : v3;
  a += __shfl_xor_sync(0xffffffffu, sa, 16);
  b += __shfl_xor_sync(0xffffffffu, sb, 16);
  double c = h8 ? b : a;
  const double sc = h8 ? a : b;
  c += __shfl_xor_sync(0xffffffffu, sc, 8);
  c += __shfl_xor_sync(0xffffffffu, c, 4);
  c += __shfl_xor_sync(0xffffffffu, c, 2);
  c += __shfl_xor_sync(0xffffffffu, c, 1);
  return c;
}

// The real and imaginary parts of up to three current axes (re[a], im[a], a < nj), summed over the
// warp and stored by the lanes that hold them at dst[2a] and dst[2a + 1].
__device__ __forceinline__ void warp_store_current(const double* re, const double* im, int nj, int lane, double* dst) {
  const double s0 = warp_sum4(re[0], im[0], nj > 1 ? re[1] : 0.0, nj > 1 ? im[1] : 0.0, lane);
  if ((lane & 7) == 0 && (lane >> 3) < 2 * nj) dst[lane >> 3] = s0;
  if (nj > 2) {
    const double s1 = warp_sum4(re[2], im[2], 0.0, 0.0, lane);
    if ((lane & 7) == 0 && (lane >> 3) < 2) dst[4 + (lane >> 3)] = s1;
  }
}

}  // namespace hhg
