// Column-tile FP64 propagation for nw <= 2 with a Hermitian placement (the 2-orbital configurations).
//
// Same propagation as propagate_kpt_kernel (the k-space-resident RK4 of src/solver.cpp:86-181 with
// the current of src/observable.cpp:16-30, or the k-space solver of src/solver_kspace.cpp), with the
// Wannier sums in separable form shared by a k-grid column:
//
//   H(k) = sum_n1 e^{-2 pi i m1 n1 / N1} G(n1),   G(n1) = P1(n1) sum_n2 e^{-2 pi i m2 n2 / N2} P2(n2) X(n1, n2)
//
// (P = the per-point factors: Peierls powers e^{i n A.a}, or the k-space solver's interpolation
// factors) and likewise for the current window.  A CTA owns R consecutive rows m1 of one column m2,
// one thread per k-point with its state in registers.  Every kRing steps the CTA computes the
// column's G for all points of the chunk into shared memory (one pair of barriers per chunk); per
// step each thread then sums the box rows (n1 >= 0 only when the placement is Hermitian and the box
// symmetric) and 4 window rows with its own row twiddles, instead of every cell of the support and
// window.
#include <cstdio>
#include <algorithm>
#include <cstdlib>

#include "sbe_device.h"
#include "sbe_herm2.cuh"

namespace hhg {
namespace {

__device__ __forceinline__ double2 kc_mul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 kc_fma(double2 a, double2 b, double2 c) {
  c.x = fma(a.x, b.x, c.x);
  c.x = fma(-a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y);
  c.y = fma(a.y, b.x, c.y);
  return c;
}
__device__ __forceinline__ double kc_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Steps per flush of the window-contracted current partials (see the kernel).
constexpr int kRJ = 16;
// Row stride (doubles) of a warp's staged state in the current contraction: 32 lanes + 4, so the
// eight 16-byte pairs one load instruction touches (4 state values x 2 lane halves, the halves
// interleaved by pairs) fall in distinct banks.
constexpr int kYS = 36;

__device__ __forceinline__ int kc_wrap(long long x, int n) {
  int r = (int)(x % n);
  return r < 0 ? r + n : r;
}

constexpr int kKcolMaxThreads = 256;

// Hermitian halving of the box rows: with H(-n) = H(n)^+ on the grid and a box symmetric about
// zero, G(-n1) = G(n1)^+, so only n1 = 0 .. (b1n - 1)/2 are summed per column.
__host__ __device__ inline bool kcol_half(const SolveTables& t) {
  return t.hermitian && t.b1lo == -(t.b1n - 1) / 2 && t.b1n % 2 == 1 && t.b2lo == -(t.b2n - 1) / 2 && t.b2n % 2 == 1;
}

// Shared-memory layout (complex double units unless noted), shared by host planning and kernel.
struct KcolLayout {
  size_t t1, G, GW, p2, total_cx, E_d, J_d, Y_d;
  int nq1, tstride;
  bool rj;  // window-contracted current (nw = 2)
  __host__ __device__ KcolLayout(const SolveTables& t, int threads, bool half) {
    rj = t.nw == 2;
    nq1 = half ? (t.b1n + 1) / 2 : t.b1n;
    tstride = threads + 2;  // twiddle rows: +2 keeps the current contraction's loads conflict-free
    const size_t nmat = 1 + t.nax, nw2 = t.nw2, pts = t.kmode ? 2 * kRing + 1 : kRing;
    size_t p = 0;
    t1 = p;
    p += (size_t)(nq1 + 4) * tstride;            // per-thread row twiddles: box rows, window rows
    G = p;
    p += pts * nq1 * nmat * nw2;                 // column sums of the chunk's points
    GW = p;
    p += (t.kmode ? 1 : kRing) * 4 * (size_t)t.nj * nw2;  // window column sums (constant: k-space solver)
    p2 = p;
    p += pts * (size_t)(t.b2n + 4);              // column factors of each point
    total_cx = p;
    E_d = 0;
    J_d = kRing * 9;
    Y_d = J_d + (rj ? (size_t)kRJ * (threads / 32) * 32 : (size_t)kRing * (threads / 32) * 2 * 3);
  }
  __host__ __device__ size_t bytes(int threads) const {
    const size_t yd = rj ? (size_t)(threads / 32) * 4 * kYS : 0;
    return total_cx * sizeof(double2) + (Y_d + yd) * sizeof(double);
  }
};

// HALF: the box sums run over n1 >= 0 with G(-n1) = G(n1)^+.  Per point, box row q = n1 and matrix
// the column sums are stored as: q = 0, G(0) in slots (G00, G11, G01, G10); q > 0, (2 G00, 2 G11,
// G01 + conj(G10), G01 - conj(G10)), so that with t = e^{-2 pi i m1 n1 / N1} = a + ib the pair
// t G(n1) + conj(t) G(n1)^+ adds 2 Re(t G_ii) on the diagonal and a S + i b D to the upper element.
template <int NW, int NAXc, int NJc, bool KM, bool HALF>
__global__ void __maxnreg__(168) propagate_kcol_kernel(SolveTables t, GroupTables gt, int R,
                                                                         int vctas, double2* rho, double2* Jpart) {
  constexpr int NW2 = NW * NW;
  // Window-contracted current (nw = 2): J_a = sum_{w1,e} GW_a,e(w1) R(w1, e) with
  // R(w1, e) = sum_k tw1(k, w1) conj(rho_e(k)), the same sum as sum_k Tr(W_a(k) rho(k)^*) in another
  // order.  Each step a warp stages its 32 k-points' state (rho00, rho11, rho01) in shared memory and
  // lane (h, w1, c) sums tw1(k, w1) (held in registers for the tile) times state value c over the
  // k-points of lane half h (both parts of tw1); every kRJ steps the CTA adds the warps' sums and
  // contracts them with the column's window sums.
  constexpr bool RJ = NW == 2;  // (the k-space solver's window sums GW are the same for every step)
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nax = NAXc ? NAXc : t.nax, nj = NJc ? NJc : t.nj, nmat = 1 + nax;
  const int b1n = t.b1n, b2n = t.b2n, npw = 2 * t.np + 1;
  const int nthr = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = nthr >> 5;
  const KcolLayout L(t, nthr, HALF);
  const int nq1 = L.nq1, q1s = b1n - nq1, ts = L.tstride;
  double2* sm = reinterpret_cast<double2*>(smraw);
  double2* sT1 = sm + L.t1;
  double2* sG = sm + L.G;
  double2* sGW = sm + L.GW;
  double2* sp2 = sm + L.p2;
  double* sE = reinterpret_cast<double*>(sm + L.total_cx) + L.E_d;
  double* sJ = reinterpret_cast<double*>(sm + L.total_cx) + L.J_d;
  double* sY = reinterpret_cast<double*>(sm + L.total_cx) + L.Y_d + (size_t)warp * 4 * kYS;
  const double2* X = gt.Xbox64;  // [nmat][b1n][b2n][NW2]
  const double2* V = gt.Xwin64;  // [nj][4][4][NW2]
  const double2* P = gt.P64;     // [points][2][npw]
  const int ppr = KM ? 2 : 1, cstride = b2n + 4;
  const double dt = t.dt;
  const double prefac = 0.1666666666666 * dt;
  const int rows = t.row1 - t.row0, tpc = (rows + R - 1) / R, ntiles = t.N2 * tpc;

  double hd[NW], rd[3][NW];
  double2 hu[NW2], ru[3][NW2], w[3][NW2];
  // Box sums of chunk point pt (Hermitian parts: diagonal real, upper triangle complex).
  auto box_sums = [&](int pt) {
    if constexpr (HALF) {
      const double2* g0 = sG + (size_t)pt * nq1 * nmat * NW2;  // n1 = 0
#pragma unroll
      for (int i = 0; i < NW; ++i) {
        hd[i] = g0[i].x;
#pragma unroll
        for (int a = 0; a < 3; ++a) rd[a][i] = a < nax ? g0[(1 + a) * NW2 + i].x : 0.0;
      }
      if constexpr (NW == 2) {
        hu[1] = g0[2];
#pragma unroll
        for (int a = 0; a < 3; ++a) ru[a][1] = a < nax ? g0[(1 + a) * NW2 + 2] : make_double2(0.0, 0.0);
      }
#pragma unroll 2
      for (int q = 1; q < nq1; ++q) {
        const double2 tw = sT1[q * ts + tid];
        const double2* g = g0 + (size_t)q * nmat * NW2;
#pragma unroll
        for (int i = 0; i < NW; ++i) hd[i] = fma(tw.x, g[i].x, fma(-tw.y, g[i].y, hd[i]));
        if constexpr (NW == 2) {
          const double2 S = g[2], D = g[3];
          hu[1].x = fma(tw.x, S.x, fma(-tw.y, D.y, hu[1].x));
          hu[1].y = fma(tw.x, S.y, fma(tw.y, D.x, hu[1].y));
        }
#pragma unroll
        for (int a = 0; a < 3; ++a)
          if (a < nax) {
            const double2* ga = g + (1 + a) * NW2;
#pragma unroll
            for (int i = 0; i < NW; ++i) rd[a][i] = fma(tw.x, ga[i].x, fma(-tw.y, ga[i].y, rd[a][i]));
            if constexpr (NW == 2) {
              const double2 S = ga[2], D = ga[3];
              ru[a][1].x = fma(tw.x, S.x, fma(-tw.y, D.y, ru[a][1].x));
              ru[a][1].y = fma(tw.x, S.y, fma(tw.y, D.x, ru[a][1].y));
            }
          }
      }
    } else {
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
      for (int q1 = 0; q1 < b1n; ++q1) {
        const double2 tw = sT1[q1 * ts + tid];
        const double2* g = sG + ((size_t)pt * b1n + q1) * nmat * NW2;
#pragma unroll
        for (int i = 0; i < NW; ++i) {
          hd[i] = fma(tw.x, g[i * NW + i].x, fma(-tw.y, g[i * NW + i].y, hd[i]));
#pragma unroll
          for (int j = i + 1; j < NW; ++j) hu[i * NW + j] = kc_fma(tw, g[i * NW + j], hu[i * NW + j]);
        }
#pragma unroll
        for (int a = 0; a < 3; ++a)
          if (a < nax) {
            const double2* ga = g + (1 + a) * NW2;
#pragma unroll
            for (int i = 0; i < NW; ++i) {
              rd[a][i] = fma(tw.x, ga[i * NW + i].x, fma(-tw.y, ga[i * NW + i].y, rd[a][i]));
#pragma unroll
              for (int j = i + 1; j < NW; ++j) ru[a][i * NW + j] = kc_fma(tw, ga[i * NW + j], ru[a][i * NW + j]);
            }
          }
      }
    }
  };
  // Window velocity W_a(k) from the column sums of slot s.
  auto window_sums = [&](int s) {
#pragma unroll
    for (int e = 0; e < NW2; ++e)
#pragma unroll
      for (int a = 0; a < 3; ++a) w[a][e] = make_double2(0.0, 0.0);
#pragma unroll
    for (int w1 = 0; w1 < 4; ++w1) {
      const double2 tw = sT1[(nq1 + w1) * ts + tid];
      const double2* g = sGW + ((size_t)s * 4 + w1) * nj * NW2;
#pragma unroll
      for (int a = 0; a < 3; ++a)
        if (a < nj)
#pragma unroll
          for (int e = 0; e < NW2; ++e) w[a][e] = kc_fma(tw, g[a * NW2 + e], w[a][e]);
    }
  };
  // Column sum of point s, box row q1 (table index), matrix mat, element e, times the row factor.
  auto column_sum = [&](int s, int q1, int mat, int e, int j0) {
    const double2* x = X + ((size_t)(mat * b1n + q1) * b2n) * NW2 + e;
    const double2* p2 = sp2 + s * cstride;
    double2 acc = make_double2(0.0, 0.0);
    for (int q2 = 0; q2 < b2n; ++q2) acc = kc_fma(p2[q2], x[(size_t)q2 * NW2], acc);
    return kc_mul(P[(size_t)(j0 + s) * 2 * npw + t.np + t.b1lo + q1], acc);
  };

  // Virtual CTA v owns tiles v, v + vctas, ... and its own row of current partials.
  for (int v = blockIdx.x; v < vctas; v += gridDim.x)
  for (int tile = v; tile < ntiles; tile += vctas) {
    const int m2 = tile / tpc, m1r = t.row0 + (tile % tpc) * R + tid;
    const bool kval = tid < R && m1r < t.row1;
    const int m1 = kval ? m1r : t.row0;
    const size_t k = (size_t)m1 * t.N2 + m2;
    double2 r[NW2];
#pragma unroll
    for (int e = 0; e < NW2; ++e) r[e] = kval ? rho[k * NW2 + e] : make_double2(0.0, 0.0);
    for (int q = 0; q < nq1; ++q) sT1[q * ts + tid] = t.T1[kc_wrap((long long)m1 * (t.b1lo + q1s + q), t.N1)];
    for (int q = 0; q < 4; ++q) sT1[(nq1 + q) * ts + tid] = t.T1[kc_wrap((long long)m1 * (q - 2), t.N1)];
    // This lane's twiddles in the current contraction (RJ): tw1(k, w1) of the warp's k-points
    // k = 4j + 2h + b (j < 8, b < 2) of lane half h, for the lane's window row w1.
    double2 twc[RJ ? 16 : 1];
    if constexpr (RJ) {
      const int h = lane >> 4, w1 = (lane >> 2) & 3, m1w = t.row0 + (tile % tpc) * R + warp * 32;
#pragma unroll
      for (int j = 0; j < 16; ++j)
        twc[j] = t.T1[kc_wrap((long long)(m1w + 4 * (j >> 1) + 2 * h + (j & 1)) * (w1 - 2), t.N1)];
    }

    for (int ti0 = t.step0; ti0 < t.step1; ti0 += kRing) {
      const int nsteps = min(kRing, t.step1 - ti0);
      const int npts = KM ? 2 * nsteps + 1 : nsteps, j0 = ppr * ti0;
      __syncthreads();  // the previous chunk's readers are done
      // (a) column factors of each point: box n2 = b2lo + q, then window n2 = -2..1
      for (int idx = tid; idx < npts * cstride; idx += nthr) {
        const int s = idx / cstride, q = idx % cstride;
        const int n2 = q < b2n ? t.b2lo + q : q - b2n - 2;
        const double2 tw = t.T2[kc_wrap((long long)m2 * n2, t.N2)];
        sp2[idx] = (KM && q >= b2n) ? tw : kc_mul(tw, P[((size_t)(j0 + s) * 2 + 1) * npw + t.np + n2]);
      }
      for (int idx = tid; idx < nsteps * 9; idx += nthr) sE[idx] = t.es[(size_t)ti0 * 9 + idx];
      __syncthreads();
      // (b) the column's sums G(n1) of each point, times the row factor P1(n1)
      const int nG = npts * nq1 * nmat * NW2;
      for (int idx = tid; idx < nG; idx += nthr) {
        const int e = idx % NW2;
        int rest = idx / NW2;
        const int mat = rest % nmat;
        rest /= nmat;
        const int q = rest % nq1, s = rest / nq1;
        double2 val;
        if constexpr (HALF) {
          // slot e of the stored form (see above); element index i * NW + j
          if (q == 0 || e < NW) {
            const int src = NW == 2 ? (e == 0 ? 0 : e == 1 ? 3 : e == 2 ? 1 : 2) : 0;
            val = column_sum(s, q1s + q, mat, src, j0);
            if (q > 0) val = make_double2(2.0 * val.x, 2.0 * val.y);
          } else {
            const double2 g01 = column_sum(s, q1s + q, mat, 1, j0), g10 = column_sum(s, q1s + q, mat, 2, j0);
            val = e == 2 ? make_double2(g01.x + g10.x, g01.y - g10.y) : make_double2(g01.x - g10.x, g01.y + g10.y);
          }
        } else {
          val = column_sum(s, q, mat, e, j0);
        }
        sG[idx] = val;
      }
      const bool win_now = !KM || ti0 == t.step0;  // the k-space solver's window sums are constant
      if (win_now) {
        const int nW = (KM ? 1 : nsteps) * 4 * nj * NW2;
        for (int idx = tid; idx < nW; idx += nthr) {
          const int e = idx % NW2;
          int rest = idx / NW2;
          const int a = rest % nj;
          rest /= nj;
          const int w1 = rest % 4, s = rest / 4;
          const double2* vv = V + ((size_t)(a * 4 + w1) * 4) * NW2 + e;
          const double2* p2 = sp2 + s * cstride + b2n;
          double2 acc = make_double2(0.0, 0.0);
#pragma unroll
          for (int w2 = 0; w2 < 4; ++w2) acc = kc_fma(p2[w2], vv[(size_t)w2 * NW2], acc);
          sGW[idx] = KM ? acc : kc_mul(P[(size_t)(j0 + s) * 2 * npw + t.np + (w1 - 2)], acc);
        }
      }
      __syncthreads();
      if (KM && !RJ && ti0 == t.step0) window_sums(0);

      for (int s = 0; s < nsteps; ++s) {
        if (!KM) {
          box_sums(s);
          if (!RJ) window_sums(s);
        } else if (s == 0) {
          box_sums(0);  // point t of the chunk's first step; later steps carry it from stage 4
        }
        if constexpr (NW == 2) {
          herm2_rk4_step<NAXc>(r, hd, hu, rd, ru, nax, t.ax_id, sE + s * 9, dt, prefac, [&](int f) {
            if (KM) box_sums(2 * s + f);  // the k-space solver's points t + dt/2, t + dt
          });
        } else {
          // One orbital: k = -i (h x - conj(h x)) = 2 h Im(x) is real, so Im(x) = Im(rho) in every stage
          // (src/solver.cpp:157-163: fields at t, t+dt/2, t+dt/2, t+dt).
          double sk = 0.0;
#pragma unroll
          for (int st = 0; st < 4; ++st) {
            const int f = st == 0 ? 0 : (st == 3 ? 2 : 1);
            const double* es = sE + s * 9 + f * 3;
            if (KM && (st == 1 || st == 3)) box_sums(2 * s + f);  // points t + dt/2, t + dt
            double h = hd[0];
#pragma unroll
            for (int a = 0; a < 3; ++a)
              if (a < nax) h = fma(es[t.ax_id[a]], rd[a][0], h);
            const double kx = 2.0 * (h * r[0].y);
            sk = st == 0 ? kx : fma(st == 3 ? 1.0 : 2.0, kx, sk);
          }
          r[0].x = fma(prefac, sk, r[0].x);
        }

        // Current partials.
        if constexpr (RJ) {
          __syncwarp();  // the previous step's readers of this warp's staging rows are done
          sY[lane] = kval ? r[0].x : 0.0;
          sY[kYS + lane] = kval ? r[3].x : 0.0;
          sY[2 * kYS + lane] = kval ? r[1].x : 0.0;
          sY[3 * kYS + lane] = kval ? r[1].y : 0.0;
          __syncwarp();
          const int h = lane >> 4, w1 = (lane >> 2) & 3, c = lane & 3;
          const double* yp = sY + c * kYS + 2 * h;
          double bx0 = 0.0, by0 = 0.0, bx1 = 0.0, by1 = 0.0;
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const double2 y = *reinterpret_cast<const double2*>(yp + 4 * j);  // k = 4j + 2h, 4j + 2h + 1
            bx0 = fma(twc[2 * j].x, y.x, bx0);
            by0 = fma(twc[2 * j].y, y.x, by0);
            bx1 = fma(twc[2 * j + 1].x, y.y, bx1);
            by1 = fma(twc[2 * j + 1].y, y.y, by1);
          }
          double bx = bx0 + bx1, by = by0 + by1;
          bx += __shfl_xor_sync(0xffffffffu, bx, 16);
          by += __shfl_xor_sync(0xffffffffu, by, 16);
          if (h == 0)
            reinterpret_cast<double2*>(sJ)[((s % kRJ) * nwarps + warp) * 16 + w1 * 4 + c] = make_double2(bx, by);
          if (s % kRJ == kRJ - 1 || s == nsteps - 1) {
            const int s0f = s - s % kRJ, ns = s - s0f + 1;
            __syncthreads();
            // Warps' partials, in warp order, into warp 0's slot.
            for (int idx = tid; idx < ns * 32; idx += nthr) {
              const int ss = idx >> 5, l = idx & 31;
              double acc = 0.0;
              for (int q = 0; q < nwarps; ++q) acc += sJ[(ss * nwarps + q) * 32 + l];
              sJ[(ss * nwarps) * 32 + l] = acc;
            }
            __syncthreads();
            for (int idx = tid; idx < ns * nj; idx += nthr) {
              const int ss = idx / nj, a = idx % nj;
              const double* B = sJ + (ss * nwarps) * 32;  // B[(w1 * 4 + c) * 2 + part]
              double re = 0.0, im = 0.0;
#pragma unroll
              for (int w1 = 0; w1 < 4; ++w1) {
                const double2* g = sGW + ((size_t)((KM ? 0 : s0f + ss) * 4 + w1) * nj + a) * NW2;
                const double* b = B + w1 * 8;
                // R(w1, e) = sum_k tw1 conj(rho_e): e = 00, 01, 10, 11 from the state values' sums
                const double2 Rv[4] = {make_double2(b[0], b[1]), make_double2(b[4] + b[7], b[5] - b[6]),
                                       make_double2(b[4] - b[7], b[5] + b[6]), make_double2(b[2], b[3])};
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                  re = fma(g[e].x, Rv[e].x, fma(-g[e].y, Rv[e].y, re));
                  im = fma(g[e].x, Rv[e].y, fma(g[e].y, Rv[e].x, im));
                }
              }
              double2* dst = Jpart + ((size_t)v * t.nt + ti0 + s0f + ss) * 3 + t.j_id[a];
              // the virtual CTA's first tile writes its row (cleared before the launch) without reading it
              const double2 old = tile == v ? make_double2(0.0, 0.0) : *dst;
              *dst = make_double2(old.x + re, old.y + im);
            }
            __syncthreads();  // the slots are rewritten by the next steps
          }
        } else {
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
            re = kc_warp_sum(re);
            im = kc_warp_sum(im);
            if (lane == 0) {
              sJ[(s * nwarps + warp) * 2 * nj + 2 * a] = re;
              sJ[(s * nwarps + warp) * 2 * nj + 2 * a + 1] = im;
            }
          }
        }
      }
      if constexpr (RJ) continue;  // flushed inside the step loop
      __syncthreads();
      // Add the chunk's per-warp partials into this virtual CTA's row.
      for (int idx = tid; idx < nsteps * nj; idx += nthr) {
        const int s = idx / nj, a = idx % nj;
        double re = 0.0, im = 0.0;
        for (int q = 0; q < nwarps; ++q) {
          re += sJ[(s * nwarps + q) * 2 * nj + 2 * a];
          im += sJ[(s * nwarps + q) * 2 * nj + 2 * a + 1];
        }
        double2* dst = Jpart + ((size_t)v * t.nt + ti0 + s) * 3 + t.j_id[a];
        const double2 old = tile == v ? make_double2(0.0, 0.0) : *dst;
        *dst = make_double2(old.x + re, old.y + im);
      }
    }
    if (kval) {
#pragma unroll
      for (int e = 0; e < NW2; ++e) rho[k * NW2 + e] = r[e];
    }
  }
}

using KcolKernel = void (*)(SolveTables, GroupTables, int, int, double2*, double2*);

// Halving applies unless HHG_KCOL_FULLBOX=1 (both forms are tested against the goldens).
bool kcol_use_half(const SolveTables& t) {
  const char* e = std::getenv("HHG_KCOL_FULLBOX");
  return kcol_half(t) && !(e && e[0] == '1');
}

template <bool KM, bool HALF>
KcolKernel kcol_kernel_t(const SolveTables& t) {
  if (t.nw == 2 && t.nj == 2) {
    if (t.nax == 1) return propagate_kcol_kernel<2, 1, 2, KM, HALF>;
    if (t.nax == 2) return propagate_kcol_kernel<2, 2, 2, KM, HALF>;
  }
  return t.nw == 1 ? propagate_kcol_kernel<1, 0, 0, KM, HALF> : propagate_kcol_kernel<2, 0, 0, KM, HALF>;
}
KcolKernel kcol_kernel_for(const SolveTables& t, bool half) {
  if (t.kmode) return half ? kcol_kernel_t<true, true>(t) : kcol_kernel_t<true, false>(t);
  return half ? kcol_kernel_t<false, true>(t) : kcol_kernel_t<false, false>(t);
}

}  // namespace

bool plan_kcol(const SolveTables& t, int sm_count, LaunchShape* out, size_t smem_max, int parts_hint) {
  if (t.nw > 2 || !t.hermitian) return false;
  const int rows = t.row1 - t.row0;
  // Rows per tile: equal parts of at most 128 rows (measured on the 200x200 grid: 100-row tiles,
  // four resident CTAs per SM, beat whole 200-row columns by 16 % and 50-row tiles by 30 %).
  int parts = (rows + 127) / 128;
  if (parts_hint > 0) parts = std::max((rows + kKcolMaxThreads - 1) / kKcolMaxThreads, parts_hint);
  if (const char* e = std::getenv("HHG_KCOL_PARTS")) parts = std::max(parts, std::atoi(e));  // tuning override
  const int R = (rows + parts - 1) / parts;
  const int threads = (R + 31) / 32 * 32;
  const long ntiles = (long)t.N2 * ((rows + R - 1) / R);
  const bool half = kcol_use_half(t);
  const KcolLayout L(t, threads, half);
  const size_t smem = L.bytes(threads);
  if (smem > smem_max || threads > kKcolMaxThreads) return false;
  KcolKernel kern = kcol_kernel_for(t, half);
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem);
  if (occ < 1) return false;
  const long slots = (long)occ * sm_count;
  out->kernel = 3;
  out->kmode = t.kmode;
  out->k_per_cta = R;
  out->group = 1;
  out->threads = threads;
  out->ntiles = (int)ntiles;
  out->ctas = (int)(ntiles < slots ? ntiles : slots);
  out->vctas = out->ctas;
  out->box_sm = out->win_sm = 0;
  out->ept = 1;
  out->variant = half ? 1 : 0;
  out->smem = smem;
  return true;
}

void launch_kcol(const SolveTables& t, const GroupTables& gt, const LaunchShape& s, double2* rho, double2* Jpart,
                 cudaStream_t stream) {
  KcolKernel kern = kcol_kernel_for(t, s.variant == 1);
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem);
  kern<<<s.ctas, s.threads, s.smem, stream>>>(t, gt, s.k_per_cta, s.vctas, rho, Jpart);
}

}  // namespace hhg
