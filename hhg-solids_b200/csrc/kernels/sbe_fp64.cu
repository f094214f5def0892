// FP64 SBE propagation kernels for sm_100a.
//
// The reference (rodrigomarher/HHG-Solids) advances rho(R) in real space and forms every RK4
// stage commutator as an FFT convolution (src/solver.cpp:1428-1726): FFT of e^{iA.R} H_eff(R) and
// of rho(R) + c k_{n-1}(R), a per-k commutator, an inverse FFT.  Because the four stages are
// linear in rho and the Peierls phase is fixed for the step (src/swe.cpp:192-196), the same
// propagation runs with rho resident in k space:
//   H_s(k)  = sum_cells e^{-ik.R} e^{iA(t_i).R} (H0_cell + E_s . r_cell)
//   k_n     = -i [H_s(k), rho(k) + c_n k_{n-1}],  c = 0, dt/2, dt/2, dt
//   rho    += 0.1666666666666 dt (k1 + 2 k2 + 2 k3 + k4)                       (src/solver.cpp:170-180)
//   J_a(t_i) = (1/Nk) sum_k sum_ij W_a,ij(k) conj(rho_ij(k)),  W_a = sum_{n in 4x4} e^{-ik.R_n} e^{iA.R_n} v_a(n)
// (the 4x4 real-space window of src/observable.cpp:16-30 in Parseval form).  Every k-point is
// independent for the whole pulse, so each kernel keeps its k-points' matrices on chip for all nt
// steps: no per-step FFT, no HBM round trip of rho, one launch per solve.  The field table comes in
// and the current partials go out through a kRing-step shared-memory ring.
//
// propagate_kpt_kernel<NW>  (nw <= 2, Hermitian placement): one thread per k-point, the whole
//   state in registers; per-cell phases e^{-ik.R_c} (per thread, fixed) x e^{iA.R_c} (per step).
// propagate_group_kernel    (any nw <= 16, FP64 or mixed precision): in sbe_group.cu.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "sbe_device.h"
#include "sbe_herm2.cuh"

namespace hhg {
namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// c + a * b
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
  c.x = fma(a.x, b.x, c.x);
  c.x = fma(-a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y);
  c.y = fma(a.y, b.x, c.y);
  return c;
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ int wrap_mod(long long x, int n) {
  int r = (int)(x % n);
  return r < 0 ? r + n : r;
}

// Adds the ring of per-warp current partials of `nsteps` steps into a virtual CTA's Jpart row.
__device__ __forceinline__ void flush_current(const SolveTables& t, const double* sJ, int nwarps, int ti0, int nsteps,
                                              double2* Jpart) {
  const int nj = t.nj;
  for (int idx = threadIdx.x; idx < nsteps * nj; idx += blockDim.x) {
    const int s = idx / nj, a = idx % nj;
    double re = 0.0, im = 0.0;
    for (int w = 0; w < nwarps; ++w) {
      re += sJ[(s * nwarps + w) * 2 * nj + 2 * a];
      im += sJ[(s * nwarps + w) * 2 * nj + 2 * a + 1];
    }
    double2* dst = Jpart + ((size_t)ti0 + s) * 3 + t.j_id[a];
    const double2 old = *dst;
    *dst = make_double2(old.x + re, old.y + im);
  }
}

// ------------------------------------------------------------------ thread per k-point (nw <= 2)

constexpr int kKptMaxThreads = 288;

// NAXc, NJc: field axes and current axes fixed at compile time (0: read from t).
template <int NW, int NAXc, int NJc, bool KM>
__global__ void __launch_bounds__(kKptMaxThreads) propagate_kpt_kernel(SolveTables t, int vctas, double2* rho,
                                                                       double2* Jpart) {
  constexpr int NW2 = NW * NW;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nc = t.ncell, nwn = t.nwin, ncw = nc + nwn, nax = NAXc ? NAXc : t.nax, nj = NJc ? NJc : t.nj;
  const int nthr = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = nthr >> 5;
  double2* sH = reinterpret_cast<double2*>(smraw);  // [nc][NW2]
  double2* sR = sH + nc * NW2;                      // [nax][nc][NW2]
  double2* sV = sR + nax * nc * NW2;                // [nj][nwn][NW2]
  double2* sTk = sV + nj * nwn * NW2;               // [ncw][nthr]
  double2* sQ = sTk + ncw * nthr;                   // [kRing (k-space solver: 2 kRing + 1)][ncw]
  double* sE = reinterpret_cast<double*>(sQ + (t.kmode ? 2 * kRing + 1 : kRing) * ncw);  // [kRing][9]
  double* sJ = sE + kRing * 9;                      // [kRing][nwarps][2 nj]

  for (int idx = tid; idx < nc * NW2; idx += nthr) sH[idx] = t.H0[idx];
  for (int idx = tid; idx < nax * nc * NW2; idx += nthr) sR[idx] = t.R[idx];
  for (int idx = tid; idx < nj * nwn * NW2; idx += nthr) sV[idx] = t.V[idx];

  const double dt = t.dt;
  const double prefac = 0.1666666666666 * dt;
  const int kbeg = t.row0 * t.N2, kend = t.row1 * t.N2;
  const int ntiles = (kend - kbeg + nthr - 1) / nthr;
  // Virtual CTA v owns tiles v, v + vctas, ... and its own row of current partials, so the result
  // does not depend on how many physical CTAs share the work.
  for (int v = blockIdx.x; v < vctas; v += gridDim.x)
  for (int tile = v; tile < ntiles; tile += vctas) {
    const int k = kbeg + tile * nthr + tid;
    const bool kval = k < kend;
    double2 r[NW2];
#pragma unroll
    for (int e = 0; e < NW2; ++e) r[e] = kval ? rho[(size_t)k * NW2 + e] : make_double2(0.0, 0.0);
    const int m1 = kval ? k / t.N2 : 0, m2 = kval ? k % t.N2 : 0;
    for (int c = 0; c < ncw; ++c) {
      const int2 n = c < nc ? t.cell_n[c] : t.win_n[c - nc];
      sTk[c * nthr + tid] = cmul(t.T1[wrap_mod((long long)m1 * n.x, t.N1)], t.T2[wrap_mod((long long)m2 * n.y, t.N2)]);
    }

    constexpr bool km = KM;
    // Hermitian parts of the Wannier sums of one evaluation point: diagonal real, upper triangle
    // complex.  q = the point's row of per-cell factors.
    double hd[NW], rd[3][NW];
    double2 hu[NW2], ru[3][NW2], w[3][NW2];
    auto box_sums = [&](const double2* q) {
#pragma unroll
      for (int i = 0; i < NW; ++i) {
        hd[i] = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a) rd[a][i] = 0.0;
      }
#pragma unroll
      for (int e = 0; e < NW2; ++e) {
        hu[e] = make_double2(0.0, 0.0);
#pragma unroll
        for (int a = 0; a < 3; ++a) ru[a][e] = make_double2(0.0, 0.0);
      }
#pragma unroll 4
      for (int c = 0; c < nc; ++c) {
        const double2 ph = cmul(sTk[c * nthr + tid], q[c]);
        const double2* hc = sH + c * NW2;
#pragma unroll
        for (int i = 0; i < NW; ++i) {
          hd[i] = fma(ph.x, hc[i * NW + i].x, fma(-ph.y, hc[i * NW + i].y, hd[i]));
#pragma unroll
          for (int j = i + 1; j < NW; ++j) hu[i * NW + j] = cfma(ph, hc[i * NW + j], hu[i * NW + j]);
        }
#pragma unroll
        for (int a = 0; a < 3; ++a)
          if (a < nax) {
            const double2* rc = sR + (a * nc + c) * NW2;
#pragma unroll
            for (int i = 0; i < NW; ++i) {
              rd[a][i] = fma(ph.x, rc[i * NW + i].x, fma(-ph.y, rc[i * NW + i].y, rd[a][i]));
#pragma unroll
              for (int j = i + 1; j < NW; ++j) ru[a][i * NW + j] = cfma(ph, rc[i * NW + j], ru[a][i * NW + j]);
            }
          }
      }
    };
    // Window velocity W_a(k): q = the point's factors (Peierls), or none (k-space solver).
    auto window_sums = [&](const double2* q) {
#pragma unroll
      for (int e = 0; e < NW2; ++e)
#pragma unroll
        for (int a = 0; a < 3; ++a) w[a][e] = make_double2(0.0, 0.0);
#pragma unroll 4
      for (int c = 0; c < nwn; ++c) {
        double2 ph;
        if constexpr (KM)
          ph = sTk[(nc + c) * nthr + tid];
        else
          ph = cmul(sTk[(nc + c) * nthr + tid], q[nc + c]);
#pragma unroll
        for (int a = 0; a < 3; ++a)
          if (a < nj) {
            const double2* vc = sV + (a * nwn + c) * NW2;
#pragma unroll
            for (int e = 0; e < NW2; ++e) w[a][e] = cfma(ph, vc[e], w[a][e]);
          }
      }
    };
    if (km) window_sums(nullptr);

    const int ppr = km ? 2 : 1;  // evaluation points per step
    for (int ti0 = t.step0; ti0 < t.step1; ti0 += kRing) {
      const int nsteps = min(kRing, t.step1 - ti0);
      const int nrows = km ? 2 * nsteps + 1 : nsteps;
      __syncthreads();
      for (int idx = tid; idx < nrows * ncw; idx += nthr) sQ[idx] = t.Q[(size_t)ppr * ti0 * ncw + idx];
      for (int idx = tid; idx < nsteps * 9; idx += nthr) sE[idx] = t.es[(size_t)ti0 * 9 + idx];
      __syncthreads();
      for (int s = 0; s < nsteps; ++s) {
        if (!km) {
          box_sums(sQ + s * ncw);
          window_sums(sQ + s * ncw);
        } else if (s == 0) {
          box_sums(sQ);  // point t of the chunk's first step; later steps carry it from stage 4
        }

        if constexpr (NW == 2) {
          herm2_rk4_step<NAXc>(r, hd, hu, rd, ru, nax, t.ax_id, sE + s * 9, dt, prefac, [&](int fpt) {
            if (km) box_sums(sQ + (2 * s + fpt) * ncw);  // the k-space solver's points t + dt/2, t + dt
          });
        } else {
          // Four RK4 stages (src/solver.cpp:157-163), fields at t, t+dt/2, t+dt/2, t+dt.
          double2 K[NW2], S[NW2];
#pragma unroll
          for (int st = 0; st < 4; ++st) {
            const int f = st == 0 ? 0 : (st == 3 ? 2 : 1);
            const double* es = sE + s * 9 + f * 3;
            if (km && st > 0 && st != 2) box_sums(sQ + (2 * s + f) * ncw);  // points t + dt/2, t + dt
            double2 H[NW2], X[NW2];
#pragma unroll
            for (int i = 0; i < NW; ++i) {
              double d = hd[i];
#pragma unroll
              for (int a = 0; a < 3; ++a)
                if (a < nax) d = fma(es[t.ax_id[a]], rd[a][i], d);
              H[i * NW + i] = make_double2(d, 0.0);
#pragma unroll
              for (int j = i + 1; j < NW; ++j) {
                double2 u = hu[i * NW + j];
#pragma unroll
                for (int a = 0; a < 3; ++a)
                  if (a < nax) {
                    const double ea = es[t.ax_id[a]];
                    u.x = fma(ea, ru[a][i * NW + j].x, u.x);
                    u.y = fma(ea, ru[a][i * NW + j].y, u.y);
                  }
                H[i * NW + j] = u;
                H[j * NW + i] = cconj(u);
              }
            }
            const double cs = (st == 3 ? 1.0 : 0.5) * dt;
#pragma unroll
            for (int e = 0; e < NW2; ++e)
              X[e] = st == 0 ? r[e] : make_double2(r[e].x + cs * K[e].x, r[e].y + cs * K[e].y);
            double2 HX[NW2];
#pragma unroll
            for (int i = 0; i < NW; ++i)
#pragma unroll
              for (int j = 0; j < NW; ++j) {
                double2 acc = make_double2(0.0, 0.0);
#pragma unroll
                for (int l = 0; l < NW; ++l) acc = cfma(H[i * NW + l], X[l * NW + j], acc);
                HX[i * NW + j] = acc;
              }
#pragma unroll
            for (int i = 0; i < NW; ++i)
#pragma unroll
              for (int j = 0; j < NW; ++j) {
                // k = -i (HX - (HX)^+)
                const double cx = HX[i * NW + j].x - HX[j * NW + i].x, cy = HX[i * NW + j].y + HX[j * NW + i].y;
                K[i * NW + j] = make_double2(cy, -cx);
              }
            const double wgt = st == 3 ? 1.0 : 2.0;
#pragma unroll
            for (int e = 0; e < NW2; ++e)
              S[e] = st == 0 ? K[e] : make_double2(S[e].x + wgt * K[e].x, S[e].y + wgt * K[e].y);
          }
#pragma unroll
          for (int e = 0; e < NW2; ++e) r[e] = make_double2(r[e].x + prefac * S[e].x, r[e].y + prefac * S[e].y);
        }

        // Current partials.
#pragma unroll
        for (int a = 0; a < 3; ++a)
          if (a < nj) {
            double re = 0.0, im = 0.0;
            if (kval) {
#pragma unroll
              for (int e = 0; e < NW2; ++e) {
                re = fma(w[a][e].x, r[e].x, fma(w[a][e].y, r[e].y, re));
                im = fma(w[a][e].y, r[e].x, fma(-w[a][e].x, r[e].y, im));
              }
            }
            re = warp_sum(re);
            im = warp_sum(im);
            if (lane == 0) {
              sJ[(s * nwarps + warp) * 2 * nj + 2 * a] = re;
              sJ[(s * nwarps + warp) * 2 * nj + 2 * a + 1] = im;
            }
          }
      }
      __syncthreads();
      flush_current(t, sJ, nwarps, ti0, nsteps, Jpart + (size_t)v * t.nt * 3);
    }
    if (kval) {
#pragma unroll
      for (int e = 0; e < NW2; ++e) rho[(size_t)k * NW2 + e] = r[e];
    }
  }
}

// J[a][ti] = (1/Nk) sum_v Jpart[v][ti][a], summed in virtual-CTA order.
__global__ void reduce_current_kernel(const double2* Jpart, int ctas, int nt, double inv_nk, double2* J) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 3 * nt) return;
  const int ti = idx / 3, a = idx % 3;
  double2 acc = make_double2(0.0, 0.0);
  for (int c = 0; c < ctas; ++c) {
    const double2 v = Jpart[((size_t)c * nt + ti) * 3 + a];
    acc.x += v.x;
    acc.y += v.y;
  }
  J[(size_t)a * nt + ti] = make_double2(acc.x * inv_nk, acc.y * inv_nk);
}

// rho0(k) = U f U^+ for H(k) = sum_cells e^{-ik.R} H0 (no field): the equilibrium of
// src/rdm.cpp:23-38 taken back to the W gauge (src/swe.cpp:80-90).  U diagonalises the Hermitian
// matrix read from the lower triangle (zheevd 'L', src/hamiltonian.cpp:83-91) by cyclic complex
// Jacobi rotations; f_n = [Re (U^+ H U)_nn < 0] with the full H, as the reference rotates H
// (src/operator.cpp:165-221) before reading its diagonal.  One warp per k-point, matrices in shared
// memory, lanes over rows / columns; the rotation order is fixed, so results are deterministic.
constexpr int kRho0Warps = 8;

__global__ void __launch_bounds__(kRho0Warps * 32) rho0_fp64_kernel(SolveTables t, double2* rho) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nw = t.nw, nw2 = t.nw2;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int k = blockIdx.x * kRho0Warps + warp;
  if (k >= t.Nk) return;  // whole warps exit together
  double2* A = reinterpret_cast<double2*>(smraw) + (size_t)warp * 3 * nw2;
  double2* B = A + nw2;
  double2* V = B + nw2;
  __shared__ double w[kRho0Warps][kMaxOrb];
  const int m1 = k / t.N2, m2 = k % t.N2;
  for (int o = lane; o < nw2; o += 32) {
    double2 acc = make_double2(0.0, 0.0);
    for (int c = 0; c < t.ncell; ++c) {
      const int2 n = t.cell_n[c];
      const double2 p = cmul(t.T1[wrap_mod((long long)m1 * n.x, t.N1)], t.T2[wrap_mod((long long)m2 * n.y, t.N2)]);
      acc = cfma(p, t.H0[(size_t)c * nw2 + o], acc);
    }
    A[o] = acc;
  }
  __syncwarp();
  for (int o = lane; o < nw2; o += 32) {
    const int i = o / nw, j = o % nw;
    B[o] = i == j ? make_double2(A[o].x, 0.0) : (i > j ? A[o] : cconj(A[j * nw + i]));
    V[o] = make_double2(i == j ? 1.0 : 0.0, 0.0);
  }
  __syncwarp();
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int o = lane; o < nw2; o += 32) {
      const double a2 = B[o].x * B[o].x + B[o].y * B[o].y;
      tot += a2;
      if (o / nw != o % nw) off += a2;
    }
    off = warp_sum(off);
    tot = warp_sum(tot);
    if (off == 0.0 || off <= 1e-32 * tot) break;
    for (int p = 0; p < nw - 1; ++p)
      for (int q = p + 1; q < nw; ++q) {
        const double2 apq = B[p * nw + q];
        const double mag = hypot(apq.x, apq.y);
        if (mag == 0.0) continue;  // uniform over the warp
        const double2 ph = make_double2(apq.x / mag, apq.y / mag);
        const double tau = (B[q * nw + q].x - B[p * nw + p].x) / (2.0 * mag);
        const double tt = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        const double c = 1.0 / sqrt(1.0 + tt * tt), s = tt * c;
        const double2 se = make_double2(s * ph.x, s * ph.y), sec = make_double2(s * ph.x, -s * ph.y);
        __syncwarp();
        // B <- J^+ B J with J = [[c, s e], [-s conj(e), c]] on (p, q): columns, then rows.
        if (lane < nw) {
          const double2 akp = B[lane * nw + p], akq = B[lane * nw + q];
          const double2 t1 = cmul(sec, akq), t2 = cmul(se, akp);
          B[lane * nw + p] = make_double2(c * akp.x - t1.x, c * akp.y - t1.y);
          B[lane * nw + q] = make_double2(t2.x + c * akq.x, t2.y + c * akq.y);
        }
        __syncwarp();
        if (lane < nw) {
          const double2 apk = B[p * nw + lane], aqk = B[q * nw + lane];
          const double2 t1 = cmul(se, aqk), t2 = cmul(sec, apk);
          B[p * nw + lane] = make_double2(c * apk.x - t1.x, c * apk.y - t1.y);
          B[q * nw + lane] = make_double2(t2.x + c * aqk.x, t2.y + c * aqk.y);
          const double2 vkp = V[lane * nw + p], vkq = V[lane * nw + q];
          const double2 t3 = cmul(sec, vkq), t4 = cmul(se, vkp);
          V[lane * nw + p] = make_double2(c * vkp.x - t3.x, c * vkp.y - t3.y);
          V[lane * nw + q] = make_double2(t4.x + c * vkq.x, t4.y + c * vkq.y);
        }
        __syncwarp();
        if (lane == 0) {
          B[p * nw + q] = make_double2(0.0, 0.0);
          B[q * nw + p] = make_double2(0.0, 0.0);
        }
        __syncwarp();
      }
  }
  // Occupations from the full H.
  if (lane < nw) {
    const int n = lane;
    double d = 0.0;
    for (int p = 0; p < nw; ++p) {
      double2 hv = make_double2(0.0, 0.0);
      for (int q = 0; q < nw; ++q) hv = cfma(A[p * nw + q], V[q * nw + n], hv);
      const double2 u = V[p * nw + n];
      d += u.x * hv.x + u.y * hv.y;
    }
    w[warp][n] = d;
  }
  __syncwarp();
  for (int o = lane; o < nw2; o += 32) {
    const int p = o / nw, q = o % nw;
    double2 acc = make_double2(0.0, 0.0);
    for (int n = 0; n < nw; ++n)
      if (w[warp][n] < 0.0) acc = cfma(V[p * nw + n], cconj(V[q * nw + n]), acc);
    rho[(size_t)k * nw2 + o] = acc;
  }
}

template <typename T>
__global__ void fma_chain_kernel(T* out, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) x[q] = (T)(threadIdx.x + q);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int q = 0; q < 8; ++q) x[q] = fma(x[q], a, b);
  }
  T s = 0;
#pragma unroll
  for (int q = 0; q < 8; ++q) s += x[q];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <typename T>
double time_fma(int sms) {
  const int blocks = sms * 8, threads = 256, iters = 4096, reps = 10;
  T* d = nullptr;
  if (cudaMalloc(&d, sizeof(T) * blocks * threads) != cudaSuccess) return -1.0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int w = 0; w < 3; ++w) fma_chain_kernel<T><<<blocks, threads>>>(d, iters, (T)0.999999, (T)1e-7);
  cudaEventRecord(e0);
  for (int r = 0; r < reps; ++r) fma_chain_kernel<T><<<blocks, threads>>>(d, iters, (T)0.999999, (T)1e-7);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  const double flops = 2.0 * 8 * (double)iters * blocks * threads * reps;
  return flops / (ms * 1e-3) / 1e12;
}

size_t kpt_smem(const SolveTables& t, int threads) {
  const int ncw = t.ncell + t.nwin, qrows = t.kmode ? 2 * kRing + 1 : kRing;
  const size_t n2 = (size_t)(t.ncell * t.nw2 * (1 + t.nax) + t.nj * t.nwin * t.nw2 + ncw * threads + qrows * ncw);
  return n2 * sizeof(double2) + sizeof(double) * (kRing * 9 + kRing * (threads / 32) * 2 * t.nj);
}

using KptKernel = void (*)(SolveTables, int, double2*, double2*);
template <bool KM>
KptKernel kpt_kernel_t(const SolveTables& t) {
  if (t.nw == 2 && t.nj == 2) {
    if (t.nax == 1) return propagate_kpt_kernel<2, 1, 2, KM>;
    if (t.nax == 2) return propagate_kpt_kernel<2, 2, 2, KM>;
  }
  return t.nw == 1 ? propagate_kpt_kernel<1, 0, 0, KM> : propagate_kpt_kernel<2, 0, 0, KM>;
}
KptKernel kpt_kernel_for(const SolveTables& t) { return t.kmode ? kpt_kernel_t<true>(t) : kpt_kernel_t<false>(t); }

bool plan_kpt(const SolveTables& t, int sm_count, LaunchShape* out, size_t smem_max) {
  KptKernel kern = kpt_kernel_for(t);
  const long nk_local = (long)(t.row1 - t.row0) * t.N2;
  int threads = (int)((nk_local + sm_count - 1) / sm_count);
  threads = (threads + 31) / 32 * 32;
  threads = threads < 64 ? 64 : (threads > kKptMaxThreads ? kKptMaxThreads : threads);
  while (threads > 64 && kpt_smem(t, threads) > smem_max) threads -= 32;
  if (kpt_smem(t, threads) > smem_max) return false;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kpt_smem(t, threads));
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, kpt_smem(t, threads));
  if (occ < 1) return false;
  const long slots = (long)occ * sm_count;
  long ntiles = (nk_local + threads - 1) / threads;
  const long rounds = (ntiles + slots - 1) / slots;
  int balanced = (int)((nk_local + rounds * slots - 1) / (rounds * slots));
  balanced = (balanced + 31) / 32 * 32;
  if (balanced >= 64 && balanced < threads) threads = balanced;
  ntiles = (nk_local + threads - 1) / threads;
  out->kernel = 0;
  out->kmode = t.kmode;
  out->k_per_cta = threads;
  out->group = 1;
  out->threads = threads;
  out->ntiles = (int)ntiles;
  out->ctas = (int)(ntiles < slots ? ntiles : slots);
  out->vctas = out->ctas;
  out->box_sm = out->win_sm = 0;
  out->ept = 1;
  out->variant = -1;
  out->smem = kpt_smem(t, threads);
  return true;
}

}  // namespace

bool plan_propagate(const SolveTables& t, int precision, int sm_count, LaunchShape* out, char* why, int why_len,
                    int tile_hint) {
  const size_t kSmemMax = 220 * 1024;
  if (t.nw < 1 || t.nw > kMaxOrb) {
    snprintf(why, why_len, "num_orb=%d outside the supported range 1..%d", t.nw, kMaxOrb);
    return false;
  }
  // Tuning override: HHG_KERNEL=group / kpt / kcol forces that kernel where a thread-per-k-point one
  // would be chosen.
  const char* force = std::getenv("HHG_KERNEL");
  const bool force_group = force && std::strcmp(force, "group") == 0;
  const bool force_kpt = force && std::strcmp(force, "kpt") == 0;
  const bool force_kcol = force && std::strcmp(force, "kcol") == 0;
  // nw <= 2 runs the FP64 thread-per-k-point kernels in both precisions: with 2x2 matrices the FP32
  // element-group kernel is several times slower, so the mixed form gains nothing there.
  if (!force_group && t.hermitian && t.nw <= 2) {
    // Column tiles when there are enough columns to fill the GPU, else one k-point per thread in
    // consecutive-k tiles.
    LaunchShape kc{};
    if (!force_kpt && plan_kcol(t, sm_count, &kc, kSmemMax, tile_hint) && (force_kcol || kc.ntiles >= sm_count)) {
      *out = kc;
      return true;
    }
    if (plan_kpt(t, sm_count, out, kSmemMax)) return true;
  }
  return plan_group(t, precision, sm_count, out, why, why_len, tile_hint);
}

int launch_propagate_steps(const SolveTables& t, const GroupTables& gt, const LaunchShape& s, double2* rho,
                           double2* Jpart, cudaStream_t stream) {
  if (t.step0 >= t.step1) return 0;
  if (s.kernel == 0) {
    KptKernel kern = kpt_kernel_for(t);
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem);
    kern<<<s.ctas, s.threads, s.smem, stream>>>(t, s.vctas, rho, Jpart);
    return 1;
  }
  if (s.kernel == 3) {
    launch_kcol(t, gt, s, rho, Jpart, stream);
    return 1;
  }
  return launch_group(t, gt, s, rho, Jpart, stream);
}

cudaError_t record_event(cudaEvent_t ev, cudaStream_t stream) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  const cudaError_t e = cudaStreamIsCapturing(stream, &st);
  if (e != cudaSuccess) return e;
  // Inside a capture an external record becomes a graph node that records the event when the graph
  // runs; outside one the flag is not accepted.
  return st == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(ev, stream, cudaEventRecordExternal)
                                             : cudaEventRecord(ev, stream);
}

int launch_propagate(const SolveTables& t, const GroupTables& gt, const LaunchShape& s, double2* rho, double2* Jpart,
                     double2* J, cudaStream_t stream, cudaEvent_t after_propagate) {
  const int launches = launch_propagate_steps(t, gt, s, rho, Jpart, stream);
  if (after_propagate) record_event(after_propagate, stream);
  const int n = 3 * t.nt;
  reduce_current_kernel<<<(n + 255) / 256, 256, 0, stream>>>(Jpart, s.vctas, t.nt, 1.0 / (double)t.Nk, J);
  return launches + 1;
}

void launch_reduce_current(const double2* Jpart, int vctas, int nt, int Nk, double2* J, cudaStream_t stream) {
  const int n = 3 * nt;
  reduce_current_kernel<<<(n + 255) / 256, 256, 0, stream>>>(Jpart, vctas, nt, 1.0 / (double)Nk, J);
}

int launch_rho0_fp64(const SolveTables& t, double2* rho, cudaStream_t stream) {
  const size_t smem = (size_t)kRho0Warps * 3 * t.nw2 * sizeof(double2);
  cudaFuncSetAttribute(rho0_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  rho0_fp64_kernel<<<(t.Nk + kRho0Warps - 1) / kRho0Warps, kRho0Warps * 32, smem, stream>>>(t, rho);
  return 1;
}

int measure_fma_peaks(double* fp64_tflops, double* fp32_tflops) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  *fp64_tflops = time_fma<double>(sms);
  *fp32_tflops = time_fma<float>(sms);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace hhg
