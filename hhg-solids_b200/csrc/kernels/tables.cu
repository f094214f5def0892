// Per-step factor tables built on the device at SWESim_init (they are nt x cells sin/cos
// evaluations, the largest host cost of the setup otherwise):
//   real-space solver: Q[ti][c] = e^{i A(t_i).R_c} for the listed cells (src/swe.cpp:225-233) and the
//     separable powers P[ti][d][n] = e^{i n A(t_i).a_d};
//   k-space solver: P[j][d][n] = C_d(n) = sum_{a=-1..2} w_a(t_d) e^{-2 pi i (o_d + a) n / N} (the
//     Catmull-Rom stencil of src/interpolation.cpp acting on cell n; o_d + t_d = -N u_d(A_j), the
//     offsets computed on the host from the reference's Cramer solve) and Q[j][c] = C_1(n1') C_2(n2')
//     for the cells, 1 for the window cells.
#include <cuda_runtime.h>

#include "sbe_device.h"

namespace hhg {
namespace {

__global__ void peierls_q_kernel(const double* A, const double* Rc, int nt, int ncw, double2* Q) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)nt * ncw) return;
  const int ti = (int)(idx / ncw), c = (int)(idx % ncw);
  const double th = A[ti] * Rc[3 * c] + A[nt + ti] * Rc[3 * c + 1] + A[2 * (size_t)nt + ti] * Rc[3 * c + 2];
  double s, co;
  sincos(th, &s, &co);
  Q[idx] = make_double2(co, s);
}

__global__ void peierls_p_kernel(const double* A, double a0x, double a0y, double a0z, double a1x, double a1y,
                                 double a1z, int nt, int np, double2* P) {
  const int npw = 2 * np + 1;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)nt * 2 * npw) return;
  const int ti = (int)(idx / (2 * npw)), d = (int)(idx / npw % 2), n = (int)(idx % npw) - np;
  const double ax = A[ti], ay = A[nt + ti], az = A[2 * (size_t)nt + ti];
  const double th = d == 0 ? ax * a0x + ay * a0y + az * a0z : ax * a1x + ay * a1y + az * a1z;
  double s, co;
  sincos(n * th, &s, &co);
  P[idx] = make_double2(co, s);
}

__global__ void interp_factor_kernel(const double* x0, int N, int np, int npts, double2* P) {
  const int npw = 2 * np + 1;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)npts * 2 * npw) return;
  const int j = (int)(idx / (2 * npw)), d = (int)(idx / npw % 2), n = (int)(idx % npw) - np;
  const double x = x0[2 * j + d];
  const double o = floor(x), tt = x - o;
  const double w[4] = {((-0.5 * tt + 1.0) * tt - 0.5) * tt, (1.5 * tt - 2.5) * tt * tt + 1.0,
                       ((-1.5 * tt + 2.0) * tt + 0.5) * tt, (0.5 * tt - 0.5) * tt * tt};
  const long long ox = (long long)o;
  double re = 0.0, im = 0.0;
#pragma unroll
  for (int a = -1; a <= 2; ++a) {
    long long m = ((ox + a) * (long long)n) % N;
    if (m < 0) m += N;
    double s, co;
    sincospi(2.0 * (double)m / (double)N, &s, &co);
    re += w[a + 1] * co;
    im -= w[a + 1] * s;
  }
  P[idx] = make_double2(re, im);
}

__global__ void interp_q_kernel(const double2* P, const int2* cellp, int ncell, int ncw, int np, int npts, double2* Q) {
  const int npw = 2 * np + 1;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)npts * ncw) return;
  const int j = (int)(idx / ncw), c = (int)(idx % ncw);
  if (c >= ncell) {
    Q[idx] = make_double2(1.0, 0.0);
    return;
  }
  const double2 cx = P[((size_t)j * 2 + 0) * npw + cellp[c].x + np];
  const double2 cy = P[((size_t)j * 2 + 1) * npw + cellp[c].y + np];
  Q[idx] = make_double2(cx.x * cy.x - cx.y * cy.y, cx.x * cy.y + cx.y * cy.x);
}

__global__ void to_float2_kernel(const double2* in, size_t n, float2* out) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < n) out[idx] = make_float2((float)in[idx].x, (float)in[idx].y);
}

inline int blocks(long long n) { return (int)((n + 255) / 256); }

}  // namespace

void launch_peierls_tables(const double* A, const double* Rc, const double lat[2][3], int nt, int ncw, int np,
                           double2* Q, double2* P, cudaStream_t stream) {
  peierls_q_kernel<<<blocks((long long)nt * ncw), 256, 0, stream>>>(A, Rc, nt, ncw, Q);
  peierls_p_kernel<<<blocks((long long)nt * 2 * (2 * np + 1)), 256, 0, stream>>>(
      A, lat[0][0], lat[0][1], lat[0][2], lat[1][0], lat[1][1], lat[1][2], nt, np, P);
}

void launch_interp_tables(const double* x0, int N, int np, int npts, const int2* cellp, int ncell, int ncw, double2* P,
                          double2* Q, cudaStream_t stream) {
  interp_factor_kernel<<<blocks((long long)npts * 2 * (2 * np + 1)), 256, 0, stream>>>(x0, N, np, npts, P);
  interp_q_kernel<<<blocks((long long)npts * ncw), 256, 0, stream>>>(P, cellp, ncell, ncw, np, npts, Q);
}

void launch_to_float2(const double2* in, size_t n, float2* out, cudaStream_t stream) {
  if (n) to_float2_kernel<<<blocks((long long)n), 256, 0, stream>>>(in, n, out);
}

}  // namespace hhg
