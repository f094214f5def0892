// FP64 SBE propagation kernels for sm_100a.
//
// The reference (rodrigomarher/HHG-Solids) advances rho(R) in real space and forms every RK4
// stage commutator as an FFT convolution (src/solver.cpp:1428-1726): FFT of e^{iA.R} H_eff(R) and
// of rho(R) + c k_{n-1}(R), a per-k commutator, an inverse FFT.  Because the four stages are
// linear in rho and the Peierls phase is fixed for the step (src/swe.cpp:192-196), the same
// propagation runs with rho resident in k space:
//   H_s(k)  = sum_cells u1^{n1} u2^{n2} (H0_cell + E_s . r_cell),  u_a = e^{-2 pi i m_a/N_a} e^{i A(t_i).a_a}
//   k_n     = -i [H_s(k), rho(k) + c_n k_{n-1}],  c = 0, dt/2, dt/2, dt
//   rho    += 0.1666666666666 dt (k1 + 2 k2 + 2 k3 + k4)                       (src/solver.cpp:170-180)
//   J_a(t_i) = (1/Nk) sum_k sum_ij W_a,ij(k) conj(rho_ij(k)),  W_a = sum_{n in 4x4} u1^{n1} u2^{n2} v_a(n)
// (the 4x4 real-space window of src/observable.cpp:16-30 in Parseval form).  Every k-point is
// independent for the whole pulse, so one persistent kernel keeps each k-point's matrices on chip
// for all nt steps: no per-step FFT, no HBM round trip of rho, one launch per solve.
//
// Thread layout: a k-point is a group of G threads, thread e of the group owns matrix element
// e = i*nw + j.  G is the next power of two >= nw^2 when nw^2 <= 32 (several k-points per warp,
// __syncwarp between phases) or nw^2 rounded up to whole warps (one named barrier per group).
// The commutator uses [H, X] = HX - (HX)^+ for Hermitian H, X: one nw^3 product per stage.
#include <cstdio>
#include <cstring>

#include "sbe_device.h"

namespace hhg {
namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
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
// u^n for |u| = 1 (u^{-1} = conj(u)).
__device__ __forceinline__ double2 cpow_unit(double2 u, int n) {
  const double2 b = n >= 0 ? u : cconj(u);
  const int m = n >= 0 ? n : -n;
  double2 r = make_double2(1.0, 0.0);
  for (int q = 0; q < m; ++q) r = cmul(r, b);
  return r;
}

__device__ __forceinline__ void group_sync(int g, int G) {
  if (G <= 32) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(G) : "memory");
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

constexpr int kMaxThreads = 512;

__global__ void __launch_bounds__(kMaxThreads) propagate_fp64_kernel(SolveTables t, int kpc, int G, double2* rho,
                                                                     double2* Jpart) {
  extern __shared__ double2 sm[];
  const int nw = t.nw, nw2 = t.nw2, nt = t.nt;
  const int tid = threadIdx.x;
  const int g = tid / G, e = tid % G;
  const bool act = e < nw2;
  const int i = act ? e / nw : 0, j = act ? e % nw : 0;
  const int per = 3 * nw2 + t.ncell + kWindow;
  double2* Hs = sm + g * per;
  double2* Xs = Hs + nw2;
  double2* HXs = Xs + nw2;
  double2* ph = HXs + nw2;
  double2* phw = ph + t.ncell;
  const int nwarps = blockDim.x >> 5, warp = tid >> 5, lane = tid & 31;
  double2* Jw = sm + kpc * per;  // [2][nwarps][3]
  const double2 zero = make_double2(0.0, 0.0);
  const double dt = t.dt;
  const double prefac = 0.1666666666666 * dt;
  const int ntiles = (t.Nk + kpc - 1) / kpc;

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int k = tile * kpc + g;
    const bool kval = k < t.Nk;
    const bool own = act && kval;
    double2 r = own ? rho[(size_t)k * nw2 + e] : zero;
    const int m1 = kval ? k / t.N2 : 0, m2 = kval ? k % t.N2 : 0;
    const double2 T1 = t.T1[m1], T2 = t.T2[m2];

    for (int ti = 0; ti < nt; ++ti) {
      const StepParams* sp = t.steps + ti;
      const double2 u1 = cmul(T1, sp->p1), u2 = cmul(T2, sp->p2);
      for (int c = e; c < t.ncell; c += G) {
        const int2 n = t.cell_n[c];
        ph[c] = cmul(cpow_unit(u1, n.x), cpow_unit(u2, n.y));
      }
      for (int w = e; w < kWindow; w += G) phw[w] = cmul(cpow_unit(u1, (w >> 2) - 2), cpow_unit(u2, (w & 3) - 2));
      group_sync(g, G);

      // Wannier sums: H0(k - A), r_a(k - A) and the windowed velocity W_a(k).
      double2 h0 = zero;
      double2 rk[3] = {zero, zero, zero};
      double2 wk[3] = {zero, zero, zero};
      if (act) {
        for (int c = 0; c < t.ncell; ++c) {
          const double2 p = ph[c];
          h0 = cfma(p, t.H0[(size_t)c * nw2 + e], h0);
#pragma unroll
          for (int a = 0; a < 3; ++a)
            if (a < t.nax) rk[a] = cfma(p, t.R[((size_t)a * t.ncell + c) * nw2 + e], rk[a]);
        }
        for (int w = 0; w < kWindow; ++w) {
          const double2 p = phw[w];
#pragma unroll
          for (int a = 0; a < 3; ++a)
            if (a < t.nj) wk[a] = cfma(p, t.V[((size_t)a * kWindow + w) * nw2 + e], wk[a]);
        }
      }

      // Four RK4 stages (src/solver.cpp:157-163): fields at t, t+dt/2, t+dt/2, t+dt.
      double2 K = zero, S = zero;
#pragma unroll 1
      for (int s = 0; s < 4; ++s) {
        const int f = s == 0 ? 0 : (s == 3 ? 2 : 1);
        double2 hs = h0;
#pragma unroll
        for (int a = 0; a < 3; ++a)
          if (a < t.nax) {
            const double ea = sp->es[f][t.ax_id[a]];
            hs.x = fma(ea, rk[a].x, hs.x);
            hs.y = fma(ea, rk[a].y, hs.y);
          }
        double2 x = r;
        if (s > 0) {
          const double cs = (s == 3 ? 1.0 : 0.5) * dt;
          x.x = r.x + cs * K.x;
          x.y = r.y + cs * K.y;
        }
        if (act) {
          Hs[e] = hs;
          Xs[e] = x;
        }
        group_sync(g, G);
        double2 hx = zero;
        if (t.hermitian) {
          if (act) {
            for (int l = 0; l < nw; ++l) hx = cfma(Hs[i * nw + l], Xs[l * nw + j], hx);
            HXs[e] = hx;
          }
          group_sync(g, G);
          if (act) {
            const double2 ht = HXs[j * nw + i];
            // k = -i (HX - (HX)^+)
            const double cx = hx.x - ht.x, cy = hx.y + ht.y;
            K = make_double2(cy, -cx);
          }
        } else {
          // Placed operators not Hermitian-symmetric on the grid: full HX - XH.
          double2 xh = zero;
          if (act) {
            for (int l = 0; l < nw; ++l) {
              hx = cfma(Hs[i * nw + l], Xs[l * nw + j], hx);
              xh = cfma(Xs[i * nw + l], Hs[l * nw + j], xh);
            }
            K = make_double2(hx.y - xh.y, -(hx.x - xh.x));
          }
          group_sync(g, G);
        }
        if (s == 0) {
          S = K;
        } else {
          const double wgt = s == 3 ? 1.0 : 2.0;
          S.x += wgt * K.x;
          S.y += wgt * K.y;
        }
      }
      r.x = r.x + prefac * S.x;
      r.y = r.y + prefac * S.y;

      // Current partials: sum_ij W_ij conj(rho_ij), reduced over the CTA in a fixed order.
      double jr[3], jim[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        double2 c = zero;
        if (own && a < t.nj) c = cmul(wk[a], cconj(r));
        jr[a] = warp_sum(c.x);
        jim[a] = warp_sum(c.y);
      }
      double2* slot = Jw + (ti & 1) * nwarps * 3;
      if (lane == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) slot[warp * 3 + a] = make_double2(jr[a], jim[a]);
      }
      __syncthreads();
      if (tid < t.nj) {
        double2 acc = zero;
        for (int w = 0; w < nwarps; ++w) {
          acc.x += slot[w * 3 + tid].x;
          acc.y += slot[w * 3 + tid].y;
        }
        double2* dst = Jpart + ((size_t)blockIdx.x * nt + ti) * 3 + t.j_id[tid];
        double2 old = *dst;
        *dst = make_double2(old.x + acc.x, old.y + acc.y);
      }
    }
    if (own) rho[(size_t)k * nw2 + e] = r;
  }
}

// J[a][ti] = (1/Nk) sum_cta Jpart[cta][ti][a], summed in CTA order.
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

// Cyclic complex Jacobi on a Hermitian nw x nw matrix (row-major in A), eigenvectors as columns of V.
__device__ void jacobi_hermitian(int n, double2* A, double2* V, double* w) {
  for (int p = 0; p < n * n; ++p) V[p] = make_double2(0.0, 0.0);
  for (int p = 0; p < n; ++p) V[p * n + p] = make_double2(1.0, 0.0);
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int p = 0; p < n; ++p)
      for (int q = 0; q < n; ++q) {
        const double a2 = A[p * n + q].x * A[p * n + q].x + A[p * n + q].y * A[p * n + q].y;
        tot += a2;
        if (p != q) off += a2;
      }
    if (off == 0.0 || off <= 1e-32 * tot) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double2 apq = A[p * n + q];
        const double mag = hypot(apq.x, apq.y);
        if (mag == 0.0) continue;
        const double2 ph = make_double2(apq.x / mag, apq.y / mag);
        const double tau = (A[q * n + q].x - A[p * n + p].x) / (2.0 * mag);
        const double tt = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        const double c = 1.0 / sqrt(1.0 + tt * tt), s = tt * c;
        const double2 se = make_double2(s * ph.x, s * ph.y), sec = make_double2(s * ph.x, -s * ph.y);
        for (int k = 0; k < n; ++k) {
          const double2 akp = A[k * n + p], akq = A[k * n + q];
          const double2 t1 = cmul(sec, akq), t2 = cmul(se, akp);
          A[k * n + p] = make_double2(c * akp.x - t1.x, c * akp.y - t1.y);
          A[k * n + q] = make_double2(t2.x + c * akq.x, t2.y + c * akq.y);
        }
        for (int k = 0; k < n; ++k) {
          const double2 apk = A[p * n + k], aqk = A[q * n + k];
          const double2 t1 = cmul(se, aqk), t2 = cmul(sec, apk);
          A[p * n + k] = make_double2(c * apk.x - t1.x, c * apk.y - t1.y);
          A[q * n + k] = make_double2(t2.x + c * aqk.x, t2.y + c * aqk.y);
        }
        A[p * n + q] = make_double2(0.0, 0.0);
        A[q * n + p] = make_double2(0.0, 0.0);
        for (int k = 0; k < n; ++k) {
          const double2 vkp = V[k * n + p], vkq = V[k * n + q];
          const double2 t1 = cmul(sec, vkq), t2 = cmul(se, vkp);
          V[k * n + p] = make_double2(c * vkp.x - t1.x, c * vkp.y - t1.y);
          V[k * n + q] = make_double2(t2.x + c * vkq.x, t2.y + c * vkq.y);
        }
      }
  }
  for (int p = 0; p < n; ++p) w[p] = A[p * n + p].x;
}

// rho0(k) = U f U^+, f_n = [E_n(k) < 0]: the equilibrium of src/rdm.cpp:23-38 taken back to the
// W gauge (src/swe.cpp:80-90), with H(k) from the field-free Wannier sum.
__global__ void rho0_fp64_kernel(SolveTables t, double2* rho) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= t.Nk) return;
  const int nw = t.nw, nw2 = t.nw2;
  const int m1 = k / t.N2, m2 = k % t.N2;
  double2 A[kMaxOrb * kMaxOrb], B[kMaxOrb * kMaxOrb], V[kMaxOrb * kMaxOrb];
  double w[kMaxOrb];
  for (int o = 0; o < nw2; ++o) A[o] = make_double2(0.0, 0.0);
  for (int c = 0; c < t.ncell; ++c) {
    const int2 n = t.cell_n[c];
    int i1 = (int)(((long long)m1 * n.x) % t.N1);
    if (i1 < 0) i1 += t.N1;
    int i2 = (int)(((long long)m2 * n.y) % t.N2);
    if (i2 < 0) i2 += t.N2;
    const double2 p = cmul(t.T1[i1], t.T2[i2]);
    for (int o = 0; o < nw2; ++o) A[o] = cfma(p, t.H0[(size_t)c * nw2 + o], A[o]);
  }
  // zheevd(..., 'L') reads the lower triangle (src/hamiltonian.cpp:83-91).
  for (int p = 0; p < nw; ++p) {
    B[p * nw + p] = make_double2(A[p * nw + p].x, 0.0);
    for (int q = 0; q < p; ++q) {
      B[p * nw + q] = A[p * nw + q];
      B[q * nw + p] = cconj(A[p * nw + q]);
    }
  }
  jacobi_hermitian(nw, B, V, w);
  // Occupation from Re (U^+ H U)_nn with the full H, as the reference rotates H (src/operator.cpp:165-221)
  // before src/rdm.cpp:23-38 reads its diagonal; equal to the eigenvalue when H is Hermitian.
  for (int n = 0; n < nw; ++n) {
    double d = 0.0;
    for (int p = 0; p < nw; ++p) {
      double2 hv = make_double2(0.0, 0.0);
      for (int q = 0; q < nw; ++q) hv = cfma(A[p * nw + q], V[q * nw + n], hv);
      const double2 u = V[p * nw + n];
      d += u.x * hv.x + u.y * hv.y;
    }
    w[n] = d;
  }
  for (int p = 0; p < nw; ++p)
    for (int q = 0; q < nw; ++q) {
      double2 acc = make_double2(0.0, 0.0);
      for (int n = 0; n < nw; ++n)
        if (w[n] < 0.0) acc = cfma(V[p * nw + n], cconj(V[q * nw + n]), acc);
      rho[(size_t)k * nw2 + p * nw + q] = acc;
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

}  // namespace

bool plan_propagate(const SolveTables& t, int sm_count, LaunchShape* out, char* why, int why_len) {
  if (t.nw < 1 || t.nw > kMaxOrb) {
    snprintf(why, why_len, "num_orb=%d outside the supported range 1..%d", t.nw, kMaxOrb);
    return false;
  }
  int G;
  if (t.nw2 <= 32) {
    G = 1;
    while (G < t.nw2) G <<= 1;
  } else {
    G = (t.nw2 + 31) / 32 * 32;
  }
  const int per = 3 * t.nw2 + t.ncell + kWindow;
  int kpc_max = kMaxThreads / G;
  if (G > 32 && kpc_max > 15) kpc_max = 15;  // one named barrier per group, ids 1..15
  if (kpc_max < 1) {
    snprintf(why, why_len, "num_orb=%d needs %d threads per k-point (> %d)", t.nw, G, kMaxThreads);
    return false;
  }
  auto smem_of = [&](int kpc) {
    const int threads = kpc * G;
    const int nwarps = (threads + 31) / 32;
    return (size_t)(kpc * per + 2 * nwarps * 3) * sizeof(double2);
  };
  while (kpc_max > 1 && smem_of(kpc_max) > 200 * 1024) --kpc_max;
  if (smem_of(kpc_max) > 200 * 1024) {
    snprintf(why, why_len, "model with %d support cells does not fit in shared memory", t.ncell);
    return false;
  }
  // Whole warps per CTA when several k-points share a warp.
  const int gran = G < 32 ? 32 / G : 1;
  kpc_max = kpc_max / gran * gran;
  if (kpc_max < gran) kpc_max = gran;
  int occ = 0;
  cudaFuncSetAttribute(propagate_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_of(kpc_max));
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, propagate_fp64_kernel, kpc_max * G, smem_of(kpc_max));
  if (occ < 1) occ = 1;
  const long slots = (long)occ * sm_count;
  const long ntiles_max = (t.Nk + kpc_max - 1) / kpc_max;
  const long rounds = (ntiles_max + slots - 1) / slots;
  // Spread the k-points evenly over rounds x slots.
  long kpc = (t.Nk + rounds * slots - 1) / (rounds * slots);
  kpc = (kpc + gran - 1) / gran * gran;
  if (kpc > kpc_max) kpc = kpc_max;
  if (kpc < gran) kpc = gran;
  const long ntiles = (t.Nk + kpc - 1) / kpc;
  out->k_per_cta = (int)kpc;
  out->group = G;
  out->ctas = (int)(ntiles < slots ? ntiles : slots);
  out->smem = smem_of((int)kpc);
  return true;
}

int launch_propagate_fp64(const SolveTables& t, const LaunchShape& s, double2* rho, double2* Jpart, double2* J,
                          cudaStream_t stream, cudaEvent_t after_propagate) {
  cudaFuncSetAttribute(propagate_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem);
  propagate_fp64_kernel<<<s.ctas, s.k_per_cta * s.group, s.smem, stream>>>(t, s.k_per_cta, s.group, rho, Jpart);
  if (after_propagate) cudaEventRecord(after_propagate, stream);
  const int n = 3 * t.nt;
  reduce_current_kernel<<<(n + 255) / 256, 256, 0, stream>>>(Jpart, s.ctas, t.nt, 1.0 / (double)t.Nk, J);
  return 2;
}

int launch_rho0_fp64(const SolveTables& t, double2* rho, cudaStream_t stream) {
  rho0_fp64_kernel<<<(t.Nk + 63) / 64, 64, 0, stream>>>(t, rho);
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
