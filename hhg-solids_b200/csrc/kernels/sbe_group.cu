// Element-group SBE propagation kernel for any nw <= 16, in two precisions.
//
// Same propagation as the kernels of sbe_fp64.cu (k-space-resident RK4 of the reference's
// src/solver.cpp:86-181 and the windowed current of src/observable.cpp:16-30); this file holds the
// layout used for larger orbital counts:
//
//  * a k-point is a group of G threads, thread e owning matrix element e = i*nw + j; a CTA holds
//    B k-points of one k-grid column m2 (rows m1 = m10 .. m10+B-1);
//  * the Wannier sum is separable: H_s(k) = sum_n1 p1(k, n1) G(n1), G(n1) = sum_n2 p2(n2) X(n1, n2)
//    with p_a = e^{-i n (2 pi m_a / N_a - A(t).a_a)}; the inner sums G depend only on the column and
//    the step, so the CTA computes them once for its B k-points.  For Hermitian placements with a
//    symmetric cell box only the rows n1 >= 0 are summed: G(-n1) = G(n1)^+.
//  * G for step t+1 is computed during step t into the other half of a double buffer, so each step
//    needs one CTA barrier; the phase factors of step t+2 are prepared two steps ahead in a
//    three-slot ring.
//  * the constant cell tables are copied to shared memory once per launch when they fit.
//  * shapes with a Hermitian 7x7 cell box (TMD-like models of 6, 11 and 12 orbitals) are compiled with the
//    box fixed (WBc), and may take the inner sums precomputed (PG): group_sums_kernel forms the sums
//    of every column for a chunk of 64 steps, once per column instead of once per CTA of the column,
//    and the propagation copies each step's block into shared memory with cp.async one step ahead.
//  * in the mixed form such shapes hold two k-points per thread group (KP), each thread owning one
//    element of both, and form the commutator's product in 2x2 register tiles.
//
// Precision.  Real = double: everything FP64 (the plain form).  Real = float (the mixed form): the
// Wannier sums of H0 and r, the field coupling and the RK4 commutators in complex FP32; the state rho,
// the RK4 accumulation rho + dt/6 (k1 + 2 k2 + 2 k3 + k4), the windowed velocity sum and the
// current's k-sum stay in FP64.
#include <cstdio>
#include <algorithm>
#include <cstdlib>
#include <stdexcept>

#include "sbe_device.h"
#include "warp_reduce.cuh"

namespace hhg {
namespace {

template <typename Real>
struct Cx;
template <>
struct Cx<double> {
  using T = double2;
  static __device__ __forceinline__ T make(double a, double b) { return make_double2(a, b); }
};
template <>
struct Cx<float> {
  using T = float2;
  static __device__ __forceinline__ T make(float a, float b) { return make_float2(a, b); }
};

__device__ __forceinline__ double2 mul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 mul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 fmac(double2 a, double2 b, double2 c) {
  c.x = fma(a.x, b.x, c.x);
  c.x = fma(-a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y);
  c.y = fma(a.y, b.x, c.y);
  return c;
}
__device__ __forceinline__ float2 fmac(float2 a, float2 b, float2 c) {
  c.x = fmaf(a.x, b.x, c.x);
  c.x = fmaf(-a.y, b.y, c.x);
  c.y = fmaf(a.x, b.y, c.y);
  c.y = fmaf(a.y, b.x, c.y);
  return c;
}
template <typename V>
__device__ __forceinline__ V conjugate(V a) {
  a.y = -a.y;
  return a;
}
template <typename V>
__device__ __forceinline__ V add(V a, V b) {
  a.x += b.x;
  a.y += b.y;
  return a;
}


__device__ __forceinline__ int wrap_mod(long long x, int n) {
  int r = (int)(x % n);
  return r < 0 ? r + n : r;
}

__device__ __forceinline__ void group_sync(int g, int G) {
  if (G <= 32) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(G) : "memory");
  }
}

// Upper bound on threads per CTA: 640 (96 registers per thread) with one element per thread, 768
// (80 registers) when the inner sums come precomputed, 512 (128 registers) with two.
template <int EPT, bool PG = false>
constexpr int group_threads() {
  return EPT == 1 ? (PG ? 768 : 640) : 512;
}
constexpr int kJRing = 16;          // steps per current-partial flush

// Row stride (complex values) of the k-point-pair tile layout of side np (even): an odd number of
// 16-byte units, so that the owners' transposed accesses spread over the banks.
__host__ __device__ constexpr int tile_stride(int np) { return (np / 2) % 2 == 1 ? np : np + 2; }

// Threads per k-point for nw2 elements at ept per thread: the next power of two up to a warp,
// whole warps beyond it.
__host__ __device__ constexpr int group_size(int nw2, int ept) {
  const int per = (nw2 + ept - 1) / ept;
  int g = 1;
  while (g < per && g < 32) g <<= 1;
  return per <= 32 ? g : (per + 31) / 32 * 32;
}

// Geometry shared by host planning and the kernel.
struct GroupGeom {
  int W1n, W2n;   // cell box
  int q1s;        // first box row summed (n1 = 0 row when halving, else 0)
  int nq1;        // box rows summed
  int nmat;       // 1 + nax (H0 and field-coupled r)
  int nbrows;     // nmat * nq1
  int nwrows;     // nj * 4 window rows
  int half;       // Hermitian halving of the box rows
};

__host__ __device__ inline GroupGeom group_geom(const SolveTables& t) {
  GroupGeom g;
  g.W1n = t.b1n;
  g.W2n = t.b2n;
  g.nmat = 1 + t.nax;
  g.half = t.hermitian && (t.b1lo == -(t.b1n - 1) / 2) && (t.b1n % 2 == 1) && (t.b2lo == -(t.b2n - 1) / 2) &&
           (t.b2n % 2 == 1);
  g.q1s = g.half ? (t.b1n - 1) / 2 : 0;
  g.nq1 = t.b1n - g.q1s;
  g.nbrows = g.nmat * g.nq1;
  g.nwrows = t.nj * 4;
  return g;
}

// Shared-memory layout (element counts in units of complex Real unless noted).
template <typename Real>
struct GroupLayout {
  // Offsets: first block in complex Real (box part), then a block in complex double (window part:
  // the velocity sum feeds the current and stays FP64 in both precisions), then the current ring.
  using V = typename Cx<Real>::T;
  size_t groups, tw1, tw2, pw1, pw2, G, Xbox, total_cx;
  size_t wtw1, wtw2, wpw1, wpw2, GW, Xwin, total_dcx, sJ_doubles;
  // kstride: complex values per k-point in the per-k-point area (3 nw2, or three padded tiles).
  __host__ __device__ GroupLayout(const SolveTables& t, const GroupGeom& gg, int B, int nwarps, bool box_sm,
                                  bool win_sm, int kstride) {
    const size_t nw2 = t.nw2, W1 = gg.W1n, W2 = gg.W2n;
    size_t p = 0;
    groups = p;
    p += (size_t)B * kstride;
    tw1 = p;
    p += (size_t)B * W1;
    tw2 = p;
    p += W2;
    const size_t ring = t.kmode ? 6 : 3, gbufs = t.kmode ? 4 : 2;
    pw1 = p;
    p += ring * (size_t)B * W1;
    pw2 = p;
    p += ring * W2;
    p = (p * sizeof(V) + 15) / 16 * 16 / sizeof(V);  // 16-byte copies land in G
    G = p;
    p += gbufs * (size_t)gg.nbrows * nw2;
    Xbox = p;
    if (box_sm) p += (size_t)gg.nmat * gg.nq1 * gg.W2n * nw2;
    total_cx = (p * sizeof(V) + 15) / 16 * 16 / sizeof(V);
    size_t q = 0;
    wtw1 = q;
    q += (size_t)B * 4;
    wtw2 = q;
    q += 4;
    wpw1 = q;
    q += ring * (size_t)B * 4;
    wpw2 = q;
    q += ring * 4;
    GW = q;
    q += 2 * (size_t)gg.nwrows * nw2;
    Xwin = q;
    if (win_sm) q += (size_t)t.nj * 16 * nw2;
    total_dcx = q;
    sJ_doubles = 2 * (size_t)kJRing * nwarps * 2 * t.nj;
  }
  __host__ __device__ size_t bytes() const {
    return total_cx * sizeof(V) + total_dcx * sizeof(double2) + sJ_doubles * sizeof(double);
  }
};

// Per-precision device tables: box [nmat][W1n][W2n][nw2], window [nj][4][4][nw2], P [nt][2][2np+1],
// twiddles [N1], [N2].
template <typename Real>
struct GroupData {
  using V = typename Cx<Real>::T;
  const V* Xbox;
  const V* P;
  const V* T1;
  const V* T2;
  const double2* Xwin;  // window velocity and its phases: FP64 in both precisions
  const double2* Pd;
  const double2* T1d;
  const double2* T2d;
  const V* Gpre;          // precomputed inner sums [point in chunk][N2][nbrows][nw2] (or null)
  const double2* GWpre;   // window rows [point in chunk][N2][nwrows][nw2] (k-space solver: [N2][nwrows][nw2])
};

// 16-byte asynchronous copy global -> shared (completes at cp_async_wait_all).
__device__ __forceinline__ void cp_async16(void* dst_smem, const void* src_gmem) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src_gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Runs virtual CTAs v_first, v_first + v_step, ... (< vctas) of one solve on this CTA.
// NWc, NAXc, NJc: orbital count, field axes and current axes fixed at compile time (0: read from t).
// WBc > 0: a square WBc x WBc cell box with Hermitian halving, fixed at compile time, so that the
// Wannier-sum loops unroll with constant offsets.
// KP (k-point pairs; mixed form, Hermitian, compile-time orbital count): a group of threads holds two
// k-points, thread e0 owning element e0 of both, so each load of an inner Wannier sum G(n1) or of a
// window row serves two k-points; the commutator's product H X is formed in 2x2 register tiles from
// a column-major H and a row-major X padded to an even side NP (one 16-byte load of two H values
// and one of two X values per four complex multiply-adds), then read back by the element owners.
// Rows are an odd number of 16-byte units apart (tile_stride), which spreads the transposed
// accesses of the owners over the banks.
// PG: the inner sums of every evaluation point come precomputed (group_sums_kernel) and are copied
// into shared memory with cp.async one step ahead, instead of being formed by every CTA of the column.
template <typename Real, int EPT, int NWc, int NAXc, int NJc, bool KM, int WBc = 0, bool KP = false,
          bool PG = false>
__device__ __forceinline__ void group_vctas(const SolveTables& t, const GroupData<Real>& d, int B, int G_in, int box_sm,
                                            int win_sm, int v_first, int v_step, int vctas, double2* rho,
                                            double2* Jpart) {
  using V = typename Cx<Real>::T;
  extern __shared__ __align__(16) unsigned char smraw[];
  const GroupGeom gg = group_geom(t);
  const int nw = NWc ? NWc : t.nw, nw2 = nw * nw, nax = NAXc ? NAXc : t.nax, nj = NJc ? NJc : t.nj;
  static_assert(!KP || (EPT == 2 && NWc > 0 && sizeof(Real) == 4 && !KM), "k-point pairs: mixed form, fixed shape");
  constexpr int KPG = KP ? 2 : 1;                      // k-points per thread group
  constexpr int EU = KP ? 1 : EPT;                     // distinct elements per thread
  constexpr int NP = KP ? (NWc + 1) / 2 * 2 : 1;       // padded side of the tile layout
  constexpr int NS = tile_stride(NP);                  // its row stride: an odd number of 16-byte units
  constexpr int Gc = NWc ? group_size(NWc * NWc, EU) : 0;
  const int G = Gc ? Gc : G_in;
  const int nthr = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = (nthr + 31) >> 5;
  const int g = tid / G, e0 = tid % G, ngroups = B / KPG;
  // Slot u of this thread: element e0 + u*G of k-point g, or (KP) element e0 of k-point 2g + u.
  int eu[EPT], iu[EPT], ju[EPT], eTu[EPT];
  bool actu[EPT];
#pragma unroll
  for (int u = 0; u < EPT; ++u) {
    eu[u] = KP ? e0 : e0 + u * G;
    actu[u] = eu[u] < nw2;
    iu[u] = actu[u] ? eu[u] / nw : 0;
    ju[u] = actu[u] ? eu[u] % nw : 0;
    eTu[u] = ju[u] * nw + iu[u];
  }
  constexpr bool kBox = WBc > 0;
  const int W1n = kBox ? WBc : gg.W1n, W2n = kBox ? WBc : gg.W2n, W1 = W1n, W2 = W2n;
  const int q1s = kBox ? (WBc - 1) / 2 : gg.q1s, nq1 = kBox ? WBc - (WBc - 1) / 2 : gg.nq1;
  const int nmat = NAXc ? 1 + NAXc : gg.nmat, nbrows = nmat * nq1, nwrows = NJc ? 4 * NJc : gg.nwrows;
  const int kstride = KP ? 3 * NP * NS : 3 * nw2;
  const GroupLayout<Real> L(t, gg, B, nwarps, box_sm, win_sm, kstride);
  V* sm = reinterpret_cast<V*>(smraw);
  double2* dsm = reinterpret_cast<double2*>(sm + L.total_cx);
  V* Hs = sm + L.groups + (size_t)g * KPG * kstride;
  V* Xs = Hs + nw2;
  V* HXs = Xs + nw2;
  V* tw1 = sm + L.tw1;
  V* tw2 = sm + L.tw2;
  V* pw1 = sm + L.pw1;
  V* pw2 = sm + L.pw2;
  V* Gb = sm + L.G;
  double2* wtw1 = dsm + L.wtw1;
  double2* wtw2 = dsm + L.wtw2;
  double2* wpw1 = dsm + L.wpw1;
  double2* wpw2 = dsm + L.wpw2;
  double2* GWb = dsm + L.GW;
  const V* Xbox = box_sm ? sm + L.Xbox : d.Xbox;
  const double2* Xwin = win_sm ? dsm + L.Xwin : d.Xwin;
  double* sJ = reinterpret_cast<double*>(dsm + L.total_dcx);
  const int npw = 2 * t.np + 1;
  const double dt = t.dt;
  const double prefac = 0.1666666666666 * dt;
  const int rows = t.row1 - t.row0;
  const int bpc = (rows + B - 1) / B;
  const int ntiles = t.N2 * bpc;
  const V vzero = Cx<Real>::make(0, 0);
  const size_t gbuf = (size_t)nbrows * nw2, wbuf = (size_t)nwrows * nw2;
  constexpr bool km = KM;             // k-space solver: three evaluation points per step
  const int ring = km ? 6 : 3, gbufs = km ? 4 : 2;

  // Constant tables into shared memory (once per launch).
  if (box_sm) {
    const size_t n = (size_t)nq1 * W2n * nw2;
    for (int mat = 0; mat < nmat; ++mat)
      for (size_t idx = tid; idx < n; idx += nthr)
        sm[L.Xbox + mat * n + idx] = d.Xbox[((size_t)mat * W1n + q1s) * W2n * nw2 + idx];
  }
  if (win_sm)
    for (size_t idx = tid; idx < (size_t)nj * 16 * nw2; idx += nthr) dsm[L.Xwin + idx] = d.Xwin[idx];
  // Tile layout: the padding rows and columns are never written and must read as zero.
  if (KP)
    for (size_t idx = tid; idx < (size_t)B * kstride; idx += nthr) sm[L.groups + idx] = vzero;

  // Virtual CTA v owns tiles v, v + vctas, ... and its own row of current partials, so the result
  // does not depend on how many physical CTAs share the work.
  for (int v = v_first; v < vctas; v += v_step)
  for (int tile = v; tile < ntiles; tile += vctas) {
    const int m2 = tile / bpc, m10 = t.row0 + (tile % bpc) * B;
    bool own[EPT];
    size_t kk[EPT];
    double2 r[EPT];
#pragma unroll
    for (int u = 0; u < EPT; ++u) {
      const int m1 = m10 + (KP ? KPG * g + u : g);
      kk[u] = (size_t)m1 * t.N2 + m2;
      own[u] = actu[u] && m1 < t.row1;
      r[u] = own[u] ? rho[kk[u] * nw2 + eu[u]] : make_double2(0.0, 0.0);
    }

    // Twiddles e^{-2 pi i m n / N} of the box offsets, and (FP64) of the window offsets -2..1.
    for (int idx = tid; idx < W2; idx += nthr) tw2[idx] = d.T2[wrap_mod((long long)m2 * (t.b2lo + idx), t.N2)];
    for (int idx = tid; idx < B * W1; idx += nthr) {
      const int gq = idx / W1, q = idx % W1;
      tw1[idx] = d.T1[wrap_mod((long long)min(m10 + gq, t.row1 - 1) * (t.b1lo + q), t.N1)];
    }
    for (int idx = tid; idx < 4; idx += nthr) wtw2[idx] = d.T2d[wrap_mod((long long)m2 * (idx - 2), t.N2)];
    for (int idx = tid; idx < B * 4; idx += nthr) {
      const int gq = idx / 4, q = idx % 4;
      wtw1[idx] = d.T1d[wrap_mod((long long)min(m10 + gq, t.row1 - 1) * (q - 2), t.N1)];
    }
    __syncthreads();

    // Phase factors of evaluation point s into ring slot s % ring: p = twiddle x P(s), with P the
    // Peierls factor e^{i n A(t_s).a} (real-space solver: one point per step) or the interpolation
    // multiplier (k-space solver: points t, t + dt/2, t + dt of every step).  The window's factors
    // are the Peierls ones, or 1 in the k-space solver (made once, `win` false afterwards).
    auto make_phases = [&](int s, bool win) {
      const V* P1 = d.P + (size_t)s * 2 * npw + t.np;
      const V* P2 = P1 + npw;
      const double2* P1d = d.Pd + (size_t)s * 2 * npw + t.np;
      const double2* P2d = P1d + npw;
      V* q2 = pw2 + (s % ring) * W2;
      V* q1 = pw1 + (s % ring) * B * W1;
      double2* w2 = wpw2 + (s % ring) * 4;
      double2* w1 = wpw1 + (s % ring) * B * 4;
      const int nA = W2, nB = nA + B * W1, nC = nB + (win ? 4 : 0), nD = nC + (win ? B * 4 : 0);
      for (int idx = tid; idx < nD; idx += nthr) {
        if (idx < nA) {
          q2[idx] = mul(tw2[idx], P2[t.b2lo + idx]);
        } else if (idx < nB) {
          const int id1 = idx - nA;
          q1[id1] = mul(tw1[id1], P1[t.b1lo + id1 % W1]);
        } else if (idx < nC) {
          const int q = idx - nB;
          w2[q] = km ? wtw2[q] : mul(wtw2[q], P2d[q - 2]);
        } else {
          const int id1 = idx - nC;
          w1[id1] = km ? wtw1[id1] : mul(wtw1[id1], P1d[id1 % 4 - 2]);
        }
      }
    };
    // Inner sums of point s into buffer s % gbufs (rows assigned to groups, elements to threads);
    // window rows into buffer s & 1 when `win`.
    auto inner_sums = [&](int s, bool win) {
      const V* q2 = pw2 + (s % ring) * W2;
      const double2* w2 = wpw2 + (s % ring) * 4;
      V* Gd = Gb + (s % gbufs) * gbuf;
      double2* GWd = GWb + (s & 1) * wbuf;
      for (int row = g; row < nbrows + (win ? nwrows : 0); row += ngroups) {
        if (row < nbrows) {
          const int mat = row / nq1, qq = row % nq1;
          const V* X = box_sm ? Xbox + (((size_t)mat * nq1 + qq) * W2n) * nw2
                              : Xbox + (((size_t)mat * W1n + q1s + qq) * W2n) * nw2;
          V acc[EPT];
#pragma unroll
          for (int u = 0; u < EU; ++u) acc[u] = vzero;
#pragma unroll(kBox ? (WBc + 3) / 4 : 1)
          for (int q0 = 0; q0 < W2n; q0 += 4) {
            V xv[4][EPT];
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
              for (int u = 0; u < EU; ++u)
                if (q0 + q < W2n && actu[u]) xv[q][u] = X[(size_t)(q0 + q) * nw2 + eu[u]];
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
              for (int u = 0; u < EU; ++u)
                if (q0 + q < W2n && actu[u]) acc[u] = fmac(q2[q0 + q], xv[q][u], acc[u]);
          }
#pragma unroll
          for (int u = 0; u < EU; ++u)
            if (actu[u]) Gd[(size_t)row * nw2 + eu[u]] = acc[u];
        } else {
          const int wr = row - nbrows;  // a * 4 + q1
          const double2* X = Xwin + (size_t)wr * 4 * nw2;
#pragma unroll
          for (int u = 0; u < EU; ++u)
            if (actu[u]) {
              double2 xv[4], wacc = make_double2(0.0, 0.0);
#pragma unroll
              for (int q = 0; q < 4; ++q) xv[q] = X[(size_t)q * nw2 + eu[u]];
#pragma unroll
              for (int q = 0; q < 4; ++q) wacc = fmac(w2[q], xv[q], wacc);
              GWd[(size_t)wr * nw2 + eu[u]] = wacc;
            }
        }
      }
    };

    const int step0 = t.step0, step1 = t.step1;
    // Precomputed inner sums of point s (box rows into buffer s % gbufs, window rows into s & 1).
    // The k-space solver's points are 2 step0 ... 2 step1 and its window rows are the same for all
    // of them (one block per column).
    auto fetch_sums = [&](int s, bool win) {
      const size_t blk = (size_t)(s - (km ? 2 * step0 : step0)) * t.N2 + m2;
      const char* src = reinterpret_cast<const char*>(d.Gpre + blk * gbuf);
      char* dst = reinterpret_cast<char*>(Gb + (s % gbufs) * gbuf);
      const double2* wsrc = d.GWpre + (km ? (size_t)m2 : blk) * wbuf;
      double2* wdst = GWb + (s & 1) * wbuf;
      const int nA = (int)(gbuf * sizeof(V) / 16), nB = win ? (int)wbuf : 0;
      for (int idx = tid; idx < nA + nB; idx += nthr) {
        if (idx < nA)
          cp_async16(dst + (size_t)idx * 16, src + (size_t)idx * 16);
        else
          cp_async16(wdst + (idx - nA), wsrc + (idx - nA));
      }
      cp_async_commit();
    };
    // Outer sums over n1 of point s for this k-point: H0(k) and r_a(k) at the point's shift.
    auto outer_box = [&](int s, V* h0o, V (*rko)[EPT]) {
#pragma unroll
      for (int u = 0; u < EPT; ++u) {
        h0o[u] = vzero;
#pragma unroll
        for (int a = 0; a < 3; ++a) rko[a][u] = vzero;
      }
      const V* p1 = pw1 + (s % ring) * B * W1 + g * KPG * W1;
      const V* Gd = Gb + (s % gbufs) * gbuf;
#pragma unroll(kBox ? WBc : 1)
      for (int q1 = 0; q1 < W1n; ++q1) {
        const V ph = p1[q1];
        const bool neg = q1 < q1s;  // G(-n1) = G(n1)^+
        const int row = neg ? (W1n - 1 - q1) - q1s : q1 - q1s;
        if constexpr (KP) {
          const V ph1 = p1[W1 + q1];
          if (actu[0]) {
            const int el = neg ? eTu[0] : eu[0];
            V gv = Gd[(size_t)row * nw2 + el];
            if (neg) gv = conjugate(gv);
            h0o[0] = fmac(ph, gv, h0o[0]);
            h0o[1] = fmac(ph1, gv, h0o[1]);
#pragma unroll
            for (int a = 0; a < 3; ++a)
              if (a < nax) {
                V rv = Gd[(size_t)((1 + a) * nq1 + row) * nw2 + el];
                if (neg) rv = conjugate(rv);
                rko[a][0] = fmac(ph, rv, rko[a][0]);
                rko[a][1] = fmac(ph1, rv, rko[a][1]);
              }
          }
        } else {
#pragma unroll
          for (int u = 0; u < EPT; ++u)
            if (actu[u]) {
              const int el = neg ? eTu[u] : eu[u];
              V gv = Gd[(size_t)row * nw2 + el];
              if (neg) gv = conjugate(gv);
              h0o[u] = fmac(ph, gv, h0o[u]);
#pragma unroll
              for (int a = 0; a < 3; ++a)
                if (a < nax) {
                  V rv = Gd[(size_t)((1 + a) * nq1 + row) * nw2 + el];
                  if (neg) rv = conjugate(rv);
                  rko[a][u] = fmac(ph, rv, rko[a][u]);
                }
            }
        }
      }
    };
    // Outer sum of the window velocity of point s: W_a(k).
    double2 wk[3][EPT];
    auto outer_window = [&](int s) {
#pragma unroll
      for (int u = 0; u < EPT; ++u)
#pragma unroll
        for (int a = 0; a < 3; ++a) wk[a][u] = make_double2(0.0, 0.0);
      const double2* GWd = GWb + (s & 1) * wbuf;
      const double2* w1 = wpw1 + (s % ring) * B * 4 + g * KPG * 4;
#pragma unroll
      for (int q1 = 0; q1 < 4; ++q1) {
        const double2 ph = w1[q1];
        if constexpr (KP) {
          const double2 ph1 = w1[4 + q1];
          if (actu[0])
#pragma unroll
            for (int a = 0; a < 3; ++a)
              if (a < nj) {
                const double2 gw = GWd[(size_t)(a * 4 + q1) * nw2 + eu[0]];
                wk[a][0] = fmac(ph, gw, wk[a][0]);
                wk[a][1] = fmac(ph1, gw, wk[a][1]);
              }
        } else {
#pragma unroll
          for (int u = 0; u < EPT; ++u)
            if (actu[u])
#pragma unroll
              for (int a = 0; a < 3; ++a)
                if (a < nj) wk[a][u] = fmac(ph, GWd[(size_t)(a * 4 + q1) * nw2 + eu[u]], wk[a][u]);
        }
      }
    };
    // H0(k), r_a(k) of the point of stage 0 (k-space solver: carried from the previous step's stage 3).
    V hc[EPT], rc[3][EPT];
    if (!km) {
      make_phases(step0, true);
      if (step0 + 1 < step1) make_phases(step0 + 1, true);
      __syncthreads();
      if constexpr (PG) {
        fetch_sums(step0, true);
        cp_async_wait_all();
      } else {
        inner_sums(step0, true);
      }
      __syncthreads();
    } else {
      // Points 2 step0 .. 2 step0 + 4: phases of all, inner sums of the first three, then the
      // stage-0 sums of the first step and the (constant) window sum.
      const int j0 = 2 * step0, jmax = 2 * step1;
      for (int j = j0; j <= j0 + 4 && j <= jmax; ++j) make_phases(j, j == j0);
      __syncthreads();
      for (int j = j0; j <= j0 + 2 && j <= jmax; ++j) {
        if constexpr (PG)
          fetch_sums(j, j == j0);
        else
          inner_sums(j, j == j0);
      }
      if constexpr (PG) cp_async_wait_all();
      __syncthreads();
      outer_box(j0, hc, rc);
      outer_window(j0);
      __syncthreads();
    }

    for (int ti = step0; ti < step1; ++ti) {
      // (1) outer sums: real-space solver, the step's one point (and the window); k-space solver,
      //     the mid point (stages 2 and 3)
      V h0[EPT], rk[3][EPT];
      if (!km) {
        outer_box(ti, h0, rk);
        outer_window(ti);
      } else {
        outer_box(2 * ti + 1, h0, rk);
      }
      // (2) later points' phase factors and inner sums, off this step's critical path
      if (!km) {
        if (ti + 2 < step1) make_phases(ti + 2, true);
        if constexpr (PG) {
          if (ti + 1 < step1) fetch_sums(ti + 1, true);
        } else {
          if (ti + 1 < step1) inner_sums(ti + 1, true);
        }
      } else {
        if (2 * ti + 5 <= 2 * step1) make_phases(2 * ti + 5, false);
        if (2 * ti + 6 <= 2 * step1) make_phases(2 * ti + 6, false);
        if constexpr (PG) {
          if (2 * ti + 3 <= 2 * step1) fetch_sums(2 * ti + 3, false);
          if (2 * ti + 4 <= 2 * step1) fetch_sums(2 * ti + 4, false);
        } else {
          if (2 * ti + 3 <= 2 * step1) inner_sums(2 * ti + 3, false);
          if (2 * ti + 4 <= 2 * step1) inner_sums(2 * ti + 4, false);
        }
      }

      // (3) RK4 stages (src/solver.cpp:157-163): fields at t, t+dt/2, t+dt/2, t+dt
      const double* esb = t.es + (size_t)ti * 9;
      V K[EPT];
      double2 S[EPT];
#pragma unroll
      for (int u = 0; u < EPT; ++u) {
        K[u] = vzero;
        S[u] = make_double2(0.0, 0.0);
      }
#pragma unroll 1
      for (int st = 0; st < 4; ++st) {
        const int f = st == 0 ? 0 : (st == 3 ? 2 : 1);
        Real ea[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) ea[a] = a < nax ? (Real)esb[f * 3 + t.ax_id[a]] : (Real)0;
        const double cs = (st == 3 ? 1.0 : 0.5) * dt;
        // k-space solver: stage 1 uses the carried point t, stage 4 the point t + dt (carried on).
        if (km && st == 3) outer_box(2 * ti + 2, hc, rc);
        const bool use_c = km && (st == 0 || st == 3);
#pragma unroll
        for (int u = 0; u < EPT; ++u)
          if (actu[u]) {
            V hs = use_c ? hc[u] : h0[u];
#pragma unroll
            for (int a = 0; a < 3; ++a)
              if (a < nax) {
                const V rv = use_c ? rc[a][u] : rk[a][u];
                hs.x += ea[a] * rv.x;
                hs.y += ea[a] * rv.y;
              }
            double2 x = r[u];
            if (st > 0) {
              x.x = r[u].x + cs * (double)K[u].x;
              x.y = r[u].y + cs * (double)K[u].y;
            }
            if constexpr (KP) {
              V* base = Hs + u * kstride;
              base[ju[u] * NS + iu[u]] = hs;                                        // H column-major
              base[NP * NS + iu[u] * NS + ju[u]] = Cx<Real>::make((Real)x.x, (Real)x.y);  // X row-major
            } else {
              Hs[eu[u]] = hs;
              Xs[eu[u]] = Cx<Real>::make((Real)x.x, (Real)x.y);
            }
          }
        group_sync(g, G);
        V hx[EPT];
        if constexpr (KP) {
          // 2x2 tiles of H X: tile p of the pair's 2 (NP/2)^2 covers rows 2ti, 2ti+1, columns 2tj, 2tj+1.
          constexpr int NT = NP / 2;
          if (e0 < KPG * NT * NT) {
            const int pk = e0 / (NT * NT), pt = e0 % (NT * NT), ti = pt / NT, tj = pt % NT;
            V* base = Hs + pk * kstride;
            const float4* HT4 = reinterpret_cast<const float4*>(base) + ti;
            const float4* XP4 = reinterpret_cast<const float4*>(base + NP * NS) + tj;
            V c00 = vzero, c01 = vzero, c10 = vzero, c11 = vzero;
#pragma unroll
            for (int l = 0; l < NWc; ++l) {
              const float4 hv = HT4[l * (NS / 2)], xv = XP4[l * (NS / 2)];
              const V h0v = Cx<Real>::make(hv.x, hv.y), h1v = Cx<Real>::make(hv.z, hv.w);
              const V x0v = Cx<Real>::make(xv.x, xv.y), x1v = Cx<Real>::make(xv.z, xv.w);
              c00 = fmac(h0v, x0v, c00);
              c01 = fmac(h0v, x1v, c01);
              c10 = fmac(h1v, x0v, c10);
              c11 = fmac(h1v, x1v, c11);
            }
            float4* HX4 = reinterpret_cast<float4*>(base + 2 * NP * NS);
            HX4[(2 * ti) * (NS / 2) + tj] = make_float4(c00.x, c00.y, c01.x, c01.y);
            HX4[(2 * ti + 1) * (NS / 2) + tj] = make_float4(c10.x, c10.y, c11.x, c11.y);
          }
          group_sync(g, G);
#pragma unroll
          for (int u = 0; u < EPT; ++u)
            if (actu[u]) {
              const V* HXP = Hs + u * kstride + 2 * NP * NS;
              const V hv = HXP[iu[u] * NS + ju[u]], ht = HXP[ju[u] * NS + iu[u]];
              K[u] = Cx<Real>::make(hv.y + ht.y, -(hv.x - ht.x));  // -i (HX - (HX)^+)
            }
        } else if (t.hermitian) {
#pragma unroll
          for (int u = 0; u < EPT; ++u) {
            hx[u] = vzero;
            if (actu[u]) {
              const V* hrow = Hs + iu[u] * nw;
              const V* xcol = Xs + ju[u];
              V h2 = vzero;
              int l = 0;
#pragma unroll
              for (; l + 1 < nw; l += 2) {
                hx[u] = fmac(hrow[l], xcol[l * nw], hx[u]);
                h2 = fmac(hrow[l + 1], xcol[(l + 1) * nw], h2);
              }
              if (l < nw) hx[u] = fmac(hrow[l], xcol[l * nw], hx[u]);
              hx[u] = add(hx[u], h2);
              HXs[eu[u]] = hx[u];
            }
          }
          group_sync(g, G);
#pragma unroll
          for (int u = 0; u < EPT; ++u)
            if (actu[u]) {
              const V ht = HXs[eTu[u]];
              K[u] = Cx<Real>::make(hx[u].y + ht.y, -(hx[u].x - ht.x));  // -i (HX - (HX)^+)
            }
        } else {
#pragma unroll
          for (int u = 0; u < EPT; ++u)
            if (actu[u]) {
              V a1 = vzero, xh = vzero;
#pragma unroll
              for (int l = 0; l < nw; ++l) {
                a1 = fmac(Hs[iu[u] * nw + l], Xs[l * nw + ju[u]], a1);
                xh = fmac(Xs[iu[u] * nw + l], Hs[l * nw + ju[u]], xh);
              }
              K[u] = Cx<Real>::make(a1.y - xh.y, -(a1.x - xh.x));  // -i (HX - XH)
            }
          group_sync(g, G);
        }
        const double wgt = st == 0 ? 1.0 : (st == 3 ? 1.0 : 2.0);
#pragma unroll
        for (int u = 0; u < EPT; ++u) {
          if (st == 0) {
            S[u] = make_double2((double)K[u].x, (double)K[u].y);
          } else {
            S[u].x += wgt * (double)K[u].x;
            S[u].y += wgt * (double)K[u].y;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < EPT; ++u) {
        r[u].x = r[u].x + prefac * S[u].x;
        r[u].y = r[u].y + prefac * S[u].y;
      }

      // (4) current partials, summed over k in FP64
      const int slot = (ti / kJRing) & 1, s = ti % kJRing;
      {
        double re[3] = {0.0, 0.0, 0.0}, im[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int a = 0; a < 3; ++a)
          if (a < nj) {
#pragma unroll
            for (int u = 0; u < EPT; ++u)
              if (own[u]) {
                const double wx = wk[a][u].x, wy = wk[a][u].y;
                re[a] = fma(wx, r[u].x, fma(wy, r[u].y, re[a]));
                im[a] = fma(wy, r[u].x, fma(-wx, r[u].y, im[a]));
              }
          }
        warp_store_current(re, im, nj, lane, sJ + (((size_t)slot * kJRing + s) * nwarps + warp) * 2 * nj);
      }
      if constexpr (PG) cp_async_wait_all();  // the next step's sums, before the barrier publishes them
      __syncthreads();
      // Flush a completed ring half: the other half is being written meanwhile.
      if (s == kJRing - 1 || ti == step1 - 1) {
        const int ti0 = max(ti - s, step0), nsteps = ti - ti0 + 1;  // a chunk may start inside a ring half
        const double* half = sJ + ((size_t)slot * kJRing + (ti0 % kJRing)) * nwarps * 2 * nj;
        for (int idx = tid; idx < nsteps * nj; idx += nthr) {
          const int ss = idx / nj, a = idx % nj;
          double re = 0.0, im = 0.0;
          for (int w = 0; w < nwarps; ++w) {
            re += half[(ss * nwarps + w) * 2 * nj + 2 * a];
            im += half[(ss * nwarps + w) * 2 * nj + 2 * a + 1];
          }
          // (selects, not an indexed read: an indexed read of the descriptor would move it to local memory)
          const int ja = a == 0 ? t.j_id[0] : (a == 1 ? t.j_id[1] : t.j_id[2]);
          double2* dst = Jpart + ((size_t)v * t.nt + ti0 + ss) * 3 + ja;
          const double2 old = *dst;
          *dst = make_double2(old.x + re, old.y + im);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < EPT; ++u)
      if (own[u]) rho[kk[u] * nw2 + eu[u]] = r[u];
    __syncthreads();
  }
}

constexpr int kMaxPreBox = 64;  // widest cell box of the precomputed-sum shapes
constexpr int kPreChunk = 64;   // steps per precompute + propagate launch pair

// Inner Wannier sums of every column for the steps [t.step0, t.step1): block (point group, m2) forms,
// for kSumPts consecutive points s of the chunk, the box rows G_e = sum_q p2(q) X(mat, q1s + qq, q)_e
// and the window rows, with the operations (and their order) of group_vctas's inner_sums, into
// [s - t.step0][m2][row][nw2]; each thread loads a row's X values once for all of the block's points.
// For the k-space solver the points are 2 step0 ... 2 step1 and the window rows, the same for every
// point, are written once per column ([m2][row][nw2], by the block of the first point).
constexpr int kSumPts = 8;
template <typename Real>
__global__ void __launch_bounds__(256) group_sums_kernel(SolveTables t, GroupData<Real> d, int q1s, int nq1,
                                                         int nbrows, int nwrows, typename Cx<Real>::T* Gpre,
                                                         double2* GWpre, int npts) {
  using V = typename Cx<Real>::T;
  __shared__ V q2[kSumPts][kMaxPreBox];
  __shared__ double2 w2[kSumPts][4];
  const int sg = blockIdx.x / t.N2, m2 = blockIdx.x % t.N2, sl0 = sg * kSumPts;
  const int ns = min(kSumPts, npts - sl0);
  const int npw = 2 * t.np + 1, W1n = t.b1n, W2n = t.b2n, nw2 = t.nw2;
  for (int idx = threadIdx.x; idx < ns * (W2n + 4); idx += blockDim.x) {
    const int j = idx / (W2n + 4), q = idx % (W2n + 4);
    const int s = (t.kmode ? 2 * t.step0 : t.step0) + sl0 + j;
    if (q < W2n) {
      const V* P2 = d.P + (size_t)s * 2 * npw + t.np + npw;
      q2[j][q] = mul(d.T2[wrap_mod((long long)m2 * (t.b2lo + q), t.N2)], P2[t.b2lo + q]);
    } else {
      const int qw = q - W2n;
      const double2* P2d = d.Pd + (size_t)s * 2 * npw + t.np + npw;
      const double2 tw = d.T2d[wrap_mod((long long)m2 * (qw - 2), t.N2)];
      w2[j][qw] = t.kmode ? tw : mul(tw, P2d[qw - 2]);
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < nbrows * nw2; idx += blockDim.x) {
    const int row = idx / nw2, e = idx % nw2, mat = row / nq1, qq = row % nq1;
    const V* X = d.Xbox + ((size_t)(mat * W1n + q1s + qq) * W2n) * nw2;
    V acc[kSumPts];
#pragma unroll
    for (int j = 0; j < kSumPts; ++j) acc[j] = Cx<Real>::make(0, 0);
    for (int q = 0; q < W2n; ++q) {
      const V x = X[(size_t)q * nw2 + e];
#pragma unroll
      for (int j = 0; j < kSumPts; ++j)
        if (j < ns) acc[j] = fmac(q2[j][q], x, acc[j]);
    }
#pragma unroll
    for (int j = 0; j < kSumPts; ++j)
      if (j < ns) Gpre[((size_t)(sl0 + j) * t.N2 + m2) * nbrows * nw2 + idx] = acc[j];
  }
  const int nwp = t.kmode ? (sl0 == 0 ? 1 : 0) : ns;  // points whose window rows this block writes
  for (int idx = threadIdx.x; idx < nwrows * nw2; idx += blockDim.x) {
    const int wr = idx / nw2, e = idx % nw2;
    const double2* X = d.Xwin + (size_t)wr * 4 * nw2;
    double2 xv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) xv[q] = X[(size_t)q * nw2 + e];
    for (int j = 0; j < nwp; ++j) {
      double2 acc = make_double2(0.0, 0.0);
#pragma unroll
      for (int q = 0; q < 4; ++q) acc = fmac(w2[j][q], xv[q], acc);
      GWpre[((size_t)(t.kmode ? m2 : (sl0 + j) * t.N2 + m2)) * nwrows * nw2 + idx] = acc;
    }
  }
}

// Launches group_sums_kernel over the npts points of the chunk that starts at t.step0.
template <typename Real>
void launch_group_sums(const SolveTables& t, const GroupData<Real>& d, int q1s, int nq1, int nbrows, int nwrows,
                       typename Cx<Real>::T* Gpre, double2* GWpre, int npts, cudaStream_t stream) {
  const int groups = (npts + kSumPts - 1) / kSumPts;
  group_sums_kernel<Real><<<groups * t.N2, 256, 0, stream>>>(t, d, q1s, nq1, nbrows, nwrows, Gpre, GWpre, npts);
}

template <typename Real>
__device__ __forceinline__ GroupData<Real> group_data(const GroupTables& gt) {
  GroupData<Real> d;
  if constexpr (sizeof(Real) == 8) {
    d = {gt.Xbox64, gt.P64, gt.T1_64, gt.T2_64, gt.Xwin64, gt.P64, gt.T1_64, gt.T2_64, nullptr, nullptr};
  } else {
    d = {gt.Xbox32, gt.P32, gt.T1_32, gt.T2_32, gt.Xwin64, gt.P64, gt.T1_64, gt.T2_64, nullptr, nullptr};
  }
  return d;
}

#include "sbe_frag.cuh"
#include "sbe_dfrag.cuh"
#include "sbe_mtile.cuh"

// One solve: physical CTA b runs virtual CTAs b, b + gridDim.x, ...
template <typename Real, int EPT, int NWc, int NAXc, int NJc, bool KM = false, int WBc = 0, bool KP = false,
          bool PG = false>
__global__ void __launch_bounds__(group_threads<EPT, PG>(), 1)
    propagate_group_kernel(SolveTables t, GroupData<Real> d, int B, int G, int box_sm, int win_sm, int vctas,
                           double2* rho, double2* Jpart) {
  group_vctas<Real, EPT, NWc, NAXc, NJc, KM, WBc, KP, PG>(t, d, B, G, box_sm, win_sm, blockIdx.x, gridDim.x, vctas, rho, Jpart);
}

// Many solves of one kernel shape: persistent CTAs take (solve, virtual CTA) items from a packed
// work list through an atomic counter.  Which CTA runs an item does not change its result.
template <typename Real, int EPT, int NWc, int NAXc, int NJc, bool KM = false, int WBc = 0, bool KP = false>
__global__ void __launch_bounds__(group_threads<EPT>(), 1)
    propagate_group_batch_kernel(const BatchDesc* descs, const int2* items, int nitems, int* counter) {
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();  // s_item is rewritten by the next iteration
    if (it >= nitems) break;
    const int2 w = items[it];  // (solve, virtual CTA)
    // The descriptor in registers (read-only, uniform across the CTA): the hot loop reads its fields
    // every step, which would be shared-memory loads if it stayed in shared memory.
    const BatchDesc dsc = descs[w.x];
    group_vctas<Real, EPT, NWc, NAXc, NJc, KM, WBc, KP>(dsc.t, group_data<Real>(dsc.gt), dsc.B, dsc.G, dsc.box_sm, dsc.win_sm,
                                               w.y, dsc.vctas, dsc.vctas, dsc.rho, dsc.Jpart);
    __syncthreads();
  }
}

constexpr size_t kSmemMax = 220 * 1024;

template <typename Real, int EPT, int NWc, int NAXc, int NJc, bool KM = false, int WBc = 0, bool KP = false,
          bool PG = false>
bool plan_group_t(const SolveTables& t, int sm_count, LaunchShape* out, char* why, int why_len, int tile_hint) {
  const GroupGeom gg = group_geom(t);
  constexpr int KPG = KP ? 2 : 1;  // k-points per thread group
  const int G = group_size(t.nw2, KP ? 1 : EPT);
  const int step = (G < 32 ? 32 / G : 1) * KPG;  // whole warps (and whole groups) per CTA
  int Bmax = group_threads<EPT, PG>() / G * KPG;
  if (G > 32 && Bmax > 15 * KPG) Bmax = 15 * KPG;  // one named barrier per group, ids 1..15
  Bmax = Bmax / step * step;
  const int kstride = KP ? 3 * ((t.nw + 1) / 2 * 2) * tile_stride((t.nw + 1) / 2 * 2) : 3 * t.nw2;
  if (Bmax < 1) {
    snprintf(why, why_len, "num_orb=%d needs %d threads per k-point", t.nw, G);
    return false;
  }
  // Shared-memory placement of the tables: both, box only, none.
  auto bytes = [&](int B, bool bs, bool ws) {
    return GroupLayout<Real>(t, gg, B, (B / KPG * G + 31) / 32, bs, ws, kstride).bytes();
  };
  int box_sm = 1, win_sm = 1;
  while (Bmax > step && bytes(Bmax, false, false) > kSmemMax) Bmax -= step;
  if (bytes(Bmax, false, false) > kSmemMax) {
    snprintf(why, why_len, "model (%d orbitals, %dx%d cell box) does not fit in shared memory", t.nw, t.b1n, t.b2n);
    return false;
  }
  // B = the largest count that fits, unless a tile hint (the autotuner's choice) asks for fewer: the
  // tile shape is a property of the kernel shape, the model and the hint, the same alone and in a batch.
  const int best = tile_hint > 0 ? std::max(step, std::min(Bmax, tile_hint / step * step)) : Bmax;
  if (bytes(best, true, true) > kSmemMax) win_sm = 0;
  if (bytes(best, true, win_sm) > kSmemMax) box_sm = 0;
  if (!box_sm && bytes(best, false, true) <= kSmemMax) win_sm = 1;
  out->pre_chunk = 0;
  out->pre_bytes = 0;
  if constexpr (PG) {
    // The tables are read by the precompute kernel only; the propagation copies finished sums.
    box_sm = win_sm = 0;
    const size_t gbytes = (size_t)gg.nbrows * t.nw2 * sizeof(typename Cx<Real>::T);
    const size_t wbytes = (size_t)gg.nwrows * t.nw2 * sizeof(double2);
    if (gbytes % 16 != 0 || gg.W2n > kMaxPreBox) {
      snprintf(why, why_len, "precomputed sums need 16-byte rows and a box of at most %d cells", kMaxPreBox);
      return false;
    }
    out->pre_chunk = std::min(kPreChunk, t.nt);
    out->pre_bytes = KM ? (size_t)(2 * out->pre_chunk + 1) * t.N2 * gbytes + (size_t)t.N2 * wbytes
                        : (size_t)out->pre_chunk * t.N2 * (gbytes + wbytes);
  }
  auto kern = propagate_group_kernel<Real, EPT, NWc, NAXc, NJc, KM, WBc, KP, PG>;
  const size_t smem_max = bytes(best, box_sm, win_sm);
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max);
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, best / KPG * G, smem_max);
  if (occ < 1) occ = 1;
  const long slots = (long)occ * sm_count;
  const int rows = t.row1 - t.row0;
  const long ntiles = (long)t.N2 * ((rows + best - 1) / best);
  out->kernel = sizeof(Real) == 8 ? 1 : 2;
  out->kmode = KM ? 1 : 0;
  out->ept = EPT;
  out->k_per_cta = best;
  out->group = G;
  out->threads = best / KPG * G;
  out->ntiles = (int)ntiles;
  out->ctas = (int)(ntiles < slots ? ntiles : slots);
  out->vctas = out->ctas;
  out->box_sm = box_sm;
  out->win_sm = win_sm;
  out->smem = bytes(best, box_sm, win_sm);
  return true;
}

template <typename Real, int EPT, int NWc, int NAXc, int NJc, bool KM = false, int WBc = 0, bool KP = false,
          bool PG = false>
int launch_group_t(const SolveTables& t, const GroupTables& gt, const LaunchShape& s, double2* rho, double2* Jpart,
                   cudaStream_t stream) {
  using V = typename Cx<Real>::T;
  GroupData<Real> d;
  if constexpr (sizeof(Real) == 8) {
    d = {gt.Xbox64, gt.P64, gt.T1_64, gt.T2_64, gt.Xwin64, gt.P64, gt.T1_64, gt.T2_64, nullptr, nullptr};
  } else {
    d = {gt.Xbox32, gt.P32, gt.T1_32, gt.T2_32, gt.Xwin64, gt.P64, gt.T1_64, gt.T2_64, nullptr, nullptr};
  }
  if constexpr (PG) {
    if (!gt.pre || s.pre_chunk <= 0)
      throw std::runtime_error("element-group launch: a precomputed-sum shape needs its scratch (GroupTables::pre)");
    const GroupGeom gg = group_geom(t);
    const size_t gbuf = (size_t)gg.nbrows * t.nw2, wbuf = (size_t)gg.nwrows * t.nw2;
    V* Gpre = static_cast<V*>(gt.pre);
    const size_t npts_max = KM ? 2 * (size_t)s.pre_chunk + 1 : (size_t)s.pre_chunk;
    double2* GWpre = reinterpret_cast<double2*>(static_cast<char*>(gt.pre) + npts_max * t.N2 * gbuf * sizeof(V));
    d.Gpre = Gpre;
    d.GWpre = GWpre;
    auto kern = propagate_group_kernel<Real, EPT, NWc, NAXc, NJc, KM, WBc, KP, true>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem);
    int launches = 0;
    for (int c0 = t.step0; c0 < t.step1; c0 += s.pre_chunk) {
      SolveTables tc = t;
      tc.step0 = c0;
      tc.step1 = std::min(c0 + s.pre_chunk, t.step1);
      const int npts = KM ? 2 * (tc.step1 - c0) + 1 : tc.step1 - c0;
      launch_group_sums<Real>(tc, d, gg.q1s, gg.nq1, gg.nbrows, gg.nwrows, Gpre, GWpre, npts, stream);
      kern<<<s.ctas, s.threads, s.smem, stream>>>(tc, d, s.k_per_cta, s.group, s.box_sm, s.win_sm, s.vctas, rho, Jpart);
      launches += 2;
    }
    (void)wbuf;
    return launches;
  } else {
    auto kern = propagate_group_kernel<Real, EPT, NWc, NAXc, NJc, KM, WBc, KP, false>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem);
    kern<<<s.ctas, s.threads, s.smem, stream>>>(t, d, s.k_per_cta, s.group, s.box_sm, s.win_sm, s.vctas, rho, Jpart);
    return 1;
  }
}

template <typename Real, int EPT, int NWc, int NAXc, int NJc, bool KM = false, int WBc = 0, bool KP = false>
int launch_group_batch_t(const BatchDesc* descs, const int2* items, int nitems, int* counter, int threads, size_t smem,
                         int sm_count, cudaStream_t stream) {
  auto kern = propagate_group_batch_kernel<Real, EPT, NWc, NAXc, NJc, KM, WBc, KP>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem);
  if (occ < 1) occ = 1;
  const int grid = std::min(nitems, occ * sm_count);
  kern<<<grid, threads, smem, stream>>>(descs, items, nitems, counter);
  return grid;
}

// Tensor-core fragment kernel (mixed form): precomputed inner sums, compiled 7x7 box, KPC k-points per CTA.
template <int NW, int NAX, int NJ, int KPC>
bool plan_frag_t(const SolveTables& t, int sm_count, LaunchShape* out, char* why, int why_len) {
  using FG = frag::Geom<NW, NAX, NJ, KPC>;
  auto kern = frag::propagate_frag_kernel<NW, NAX, NJ, KPC>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FG::BYTES) != cudaSuccess) {
    cudaGetLastError();
    snprintf(why, why_len, "fragment kernel: %zu bytes of shared memory not available", FG::BYTES);
    return false;
  }
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, KPC * 32, FG::BYTES);
  if (occ < 1) occ = 1;
  const long slots = (long)occ * sm_count;
  const int rows = t.row1 - t.row0;
  const long ntiles = (long)t.N2 * ((rows + KPC - 1) / KPC);
  out->kernel = 4;
  out->kmode = 0;
  out->ept = 8;
  out->k_per_cta = KPC;
  out->group = 32;
  out->threads = KPC * 32;
  out->ntiles = (int)ntiles;
  out->ctas = (int)(ntiles < slots ? ntiles : slots);
  out->vctas = out->ctas;
  out->box_sm = out->win_sm = 0;
  out->smem = FG::BYTES;
  out->pre_chunk = std::min(kPreChunk, t.nt);
  out->pre_bytes = (size_t)out->pre_chunk * t.N2 *
                   ((size_t)FG::NBROWS * FG::NW2 * sizeof(float2) + (size_t)FG::NWROWS * FG::NW2 * sizeof(double2));
  return true;
}

template <int NW, int NAX, int NJ, int KPC>
int launch_frag_t(const SolveTables& t, const GroupTables& gt, const LaunchShape& s, double2* rho, double2* Jpart,
                  cudaStream_t stream) {
  using FG = frag::Geom<NW, NAX, NJ, KPC>;
  if (!gt.pre || s.pre_chunk <= 0)
    throw std::runtime_error("fragment kernel launch: needs its precomputed-sum scratch (GroupTables::pre)");
  GroupData<float> d = {gt.Xbox32, gt.P32, gt.T1_32, gt.T2_32, gt.Xwin64, gt.P64, gt.T1_64, gt.T2_64, nullptr, nullptr};
  const size_t gbuf = (size_t)FG::NBROWS * FG::NW2;
  float2* Gpre = static_cast<float2*>(gt.pre);
  double2* GWpre = reinterpret_cast<double2*>(Gpre + (size_t)s.pre_chunk * t.N2 * gbuf);
  d.Gpre = Gpre;
  d.GWpre = GWpre;
  auto kern = frag::propagate_frag_kernel<NW, NAX, NJ, KPC>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem);
  int launches = 0;
  for (int c0 = t.step0; c0 < t.step1; c0 += s.pre_chunk) {
    SolveTables tc = t;
    tc.step0 = c0;
    tc.step1 = std::min(c0 + s.pre_chunk, t.step1);
    launch_group_sums<float>(tc, d, 3, 4, FG::NBROWS, FG::NWROWS, Gpre, GWpre, tc.step1 - c0, stream);
    kern<<<s.ctas, s.threads, s.smem, stream>>>(tc, d, s.vctas, rho, Jpart);
    launches += 2;
  }
  return launches;
}

// Mixed-form tile kernel: precomputed inner sums, compiled 7x7 box, KPC k-points per CTA (half a warp each).
template <int NW, int NAX, int NJ, int KPC, bool KM>
bool plan_mtile_t(const SolveTables& t, int sm_count, LaunchShape* out, char* why, int why_len) {
  using FG = mtile::Geom<NW, NAX, NJ, KPC, KM>;
  auto kern = mtile::propagate_mtile_kernel<NW, NAX, NJ, KPC, KM>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FG::BYTES) != cudaSuccess) {
    cudaGetLastError();
    snprintf(why, why_len, "tile kernel: %zu bytes of shared memory not available", FG::BYTES);
    return false;
  }
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, FG::NTHR, FG::BYTES);
  if (occ < 1) occ = 1;
  const long slots = (long)occ * sm_count;
  const int rows = t.row1 - t.row0;
  const long ntiles = (long)t.N2 * ((rows + KPC - 1) / KPC);
  out->kernel = 6;
  out->kmode = KM ? 1 : 0;
  out->ept = 9;
  out->k_per_cta = KPC;
  out->group = FG::LPK;
  out->threads = FG::NTHR;
  out->ntiles = (int)ntiles;
  out->ctas = (int)(ntiles < slots ? ntiles : slots);
  out->vctas = out->ctas;
  out->box_sm = out->win_sm = 0;
  out->smem = FG::BYTES;
  out->pre_chunk = std::min(kPreChunk, t.nt);
  const size_t gbytes = (size_t)FG::NBROWS * FG::NW2 * sizeof(float2), wbytes = (size_t)FG::NWROWS * FG::NW2 * sizeof(double2);
  out->pre_bytes = KM ? (size_t)(2 * out->pre_chunk + 1) * t.N2 * gbytes + (size_t)t.N2 * wbytes
                      : (size_t)out->pre_chunk * t.N2 * (gbytes + wbytes);
  return true;
}

template <int NW, int NAX, int NJ, int KPC, bool KM>
int launch_mtile_t(const SolveTables& t, const GroupTables& gt, const LaunchShape& s, double2* rho, double2* Jpart,
                   cudaStream_t stream) {
  using FG = mtile::Geom<NW, NAX, NJ, KPC, KM>;
  if (!gt.pre || s.pre_chunk <= 0)
    throw std::runtime_error("tile kernel launch: needs its precomputed-sum scratch (GroupTables::pre)");
  GroupData<float> d = {gt.Xbox32, gt.P32, gt.T1_32, gt.T2_32, gt.Xwin64, gt.P64, gt.T1_64, gt.T2_64, nullptr, nullptr};
  const size_t gbuf = (size_t)FG::NBROWS * FG::NW2;
  float2* Gpre = static_cast<float2*>(gt.pre);
  const size_t npts_max = KM ? 2 * (size_t)s.pre_chunk + 1 : (size_t)s.pre_chunk;
  double2* GWpre = reinterpret_cast<double2*>(Gpre + npts_max * t.N2 * gbuf);
  d.Gpre = Gpre;
  d.GWpre = GWpre;
  auto kern = mtile::propagate_mtile_kernel<NW, NAX, NJ, KPC, KM>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem);
  int launches = 0;
  for (int c0 = t.step0; c0 < t.step1; c0 += s.pre_chunk) {
    SolveTables tc = t;
    tc.step0 = c0;
    tc.step1 = std::min(c0 + s.pre_chunk, t.step1);
    const int npts = KM ? 2 * (tc.step1 - c0) + 1 : tc.step1 - c0;
    launch_group_sums<float>(tc, d, 3, 4, FG::NBROWS, FG::NWROWS, Gpre, GWpre, npts, stream);
    kern<<<s.ctas, s.threads, s.smem, stream>>>(tc, d, s.vctas, rho, Jpart);
    launches += 2;
  }
  return launches;
}

struct MtileVariant {
  int nw, nax, nj, kpc;
  bool km;
  bool (*plan)(const SolveTables&, int, LaunchShape*, char*, int);
  int (*launch)(const SolveTables&, const GroupTables&, const LaunchShape&, double2*, double2*, cudaStream_t);
};
#define HHG_MTILE_VARIANT(NW, NAX, NJ, KPC, KM) \
  {NW, NAX, NJ, KPC, KM, plan_mtile_t<NW, NAX, NJ, KPC, KM>, launch_mtile_t<NW, NAX, NJ, KPC, KM>}
// (12 x 12 frame: 8 k-points per CTA; 6 x 6 frame: 32.  The k-space solver's ring of four inner-sum
// slots leaves three CTAs per SM for 11 orbitals with one field axis, two for its other 12 x 12 shapes,
// which still run 1.2-2x faster than the element-group kernel.)
const MtileVariant kMtileVariants[] = {
    HHG_MTILE_VARIANT(11, 1, 2, 8, false), HHG_MTILE_VARIANT(11, 2, 2, 8, false),
    HHG_MTILE_VARIANT(12, 1, 2, 8, false), HHG_MTILE_VARIANT(12, 2, 2, 8, false),
    HHG_MTILE_VARIANT(11, 1, 2, 8, true),  HHG_MTILE_VARIANT(11, 2, 2, 8, true),
    HHG_MTILE_VARIANT(12, 1, 2, 8, true),  HHG_MTILE_VARIANT(12, 2, 2, 8, true),
    HHG_MTILE_VARIANT(6, 1, 2, 32, false),  HHG_MTILE_VARIANT(6, 2, 2, 32, false),
    HHG_MTILE_VARIANT(6, 1, 2, 32, true),   HHG_MTILE_VARIANT(6, 2, 2, 32, true),
};
#undef HHG_MTILE_VARIANT

// The tile kernel for a mixed-form solve (Hermitian halved 7x7 box; either solver), or null.
// HHG_MTILE=0 turns it off (measurements): the element-group kernel then runs the solve.
const MtileVariant* find_mtile(const SolveTables& t) {
  if (const char* off = std::getenv("HHG_MTILE"))
    if (off[0] == '0') return nullptr;
  const GroupGeom gg = group_geom(t);
  if (!t.hermitian || !gg.half || t.b1n != 7 || t.b2n != 7) return nullptr;
  for (const MtileVariant& v : kMtileVariants)
    if (v.nw == t.nw && v.nax == t.nax && v.nj == t.nj && v.km == (t.kmode != 0)) return &v;
  return nullptr;
}

// FP64 tensor-core fragment kernel (plain form): precomputed inner sums, compiled 7x7 box, 8 k-points per CTA.
template <int NW, int NAX, int NJ, bool KM>
bool plan_dfrag_t(const SolveTables& t, int sm_count, LaunchShape* out, char* why, int why_len) {
  using FG = dfrag::Geom<NW, NAX, NJ, KM>;
  auto kern = dfrag::propagate_dfrag_kernel<NW, NAX, NJ, KM>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FG::BYTES) != cudaSuccess) {
    cudaGetLastError();
    snprintf(why, why_len, "FP64 fragment kernel: %zu bytes of shared memory not available", FG::BYTES);
    return false;
  }
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, FG::KPC * 32, FG::BYTES);
  if (occ < 1) occ = 1;
  const long slots = (long)occ * sm_count;
  const int rows = t.row1 - t.row0;
  const long ntiles = (long)t.N2 * ((rows + FG::KPC - 1) / FG::KPC);
  out->kernel = 5;
  out->kmode = KM ? 1 : 0;
  out->ept = 8;
  out->k_per_cta = FG::KPC;
  out->group = 32;
  out->threads = FG::KPC * 32;
  out->ntiles = (int)ntiles;
  out->ctas = (int)(ntiles < slots ? ntiles : slots);
  out->vctas = out->ctas;
  out->box_sm = out->win_sm = 0;
  out->smem = FG::BYTES;
  out->pre_chunk = std::min(kPreChunk, t.nt);
  const size_t gbytes = (size_t)FG::NBROWS * FG::NW2 * sizeof(double2), wbytes = (size_t)FG::NWROWS * FG::NW2 * sizeof(double2);
  out->pre_bytes = KM ? (size_t)(2 * out->pre_chunk + 1) * t.N2 * gbytes + (size_t)t.N2 * wbytes
                      : (size_t)out->pre_chunk * t.N2 * (gbytes + wbytes);
  return true;
}

template <int NW, int NAX, int NJ, bool KM>
int launch_dfrag_t(const SolveTables& t, const GroupTables& gt, const LaunchShape& s, double2* rho, double2* Jpart,
                   cudaStream_t stream) {
  using FG = dfrag::Geom<NW, NAX, NJ, KM>;
  if (!gt.pre || s.pre_chunk <= 0)
    throw std::runtime_error("FP64 fragment kernel launch: needs its precomputed-sum scratch (GroupTables::pre)");
  GroupData<double> d = {gt.Xbox64, gt.P64, gt.T1_64, gt.T2_64, gt.Xwin64, gt.P64, gt.T1_64, gt.T2_64, nullptr, nullptr};
  const size_t gbuf = (size_t)FG::NBROWS * FG::NW2;
  double2* Gpre = static_cast<double2*>(gt.pre);
  const size_t npts_max = KM ? 2 * (size_t)s.pre_chunk + 1 : (size_t)s.pre_chunk;
  double2* GWpre = Gpre + npts_max * t.N2 * gbuf;
  d.Gpre = Gpre;
  d.GWpre = GWpre;
  auto kern = dfrag::propagate_dfrag_kernel<NW, NAX, NJ, KM>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem);
  int launches = 0;
  for (int c0 = t.step0; c0 < t.step1; c0 += s.pre_chunk) {
    SolveTables tc = t;
    tc.step0 = c0;
    tc.step1 = std::min(c0 + s.pre_chunk, t.step1);
    const int npts = KM ? 2 * (tc.step1 - c0) + 1 : tc.step1 - c0;
    launch_group_sums<double>(tc, d, 3, 4, FG::NBROWS, FG::NWROWS, Gpre, GWpre, npts, stream);
    kern<<<s.ctas, s.threads, s.smem, stream>>>(tc, d, s.vctas, rho, Jpart);
    launches += 2;
  }
  return launches;
}

struct DfragVariant {
  int nw, nax, nj;
  bool km;
  bool (*plan)(const SolveTables&, int, LaunchShape*, char*, int);
  int (*launch)(const SolveTables&, const GroupTables&, const LaunchShape&, double2*, double2*, cudaStream_t);
};
#define HHG_DFRAG_VARIANT(NW, NAX, NJ, KM) \
  {NW, NAX, NJ, KM, plan_dfrag_t<NW, NAX, NJ, KM>, launch_dfrag_t<NW, NAX, NJ, KM>}
// (The k-space solver's 12-orbital two-axis shape needs more shared memory than a CTA has: the
// element-group kernel runs it.)
const DfragVariant kDfragVariants[] = {
    HHG_DFRAG_VARIANT(11, 1, 2, false), HHG_DFRAG_VARIANT(11, 2, 2, false), HHG_DFRAG_VARIANT(12, 1, 2, false),
    HHG_DFRAG_VARIANT(12, 2, 2, false), HHG_DFRAG_VARIANT(11, 1, 2, true),  HHG_DFRAG_VARIANT(11, 2, 2, true),
    HHG_DFRAG_VARIANT(12, 1, 2, true),
};
#undef HHG_DFRAG_VARIANT

// The FP64 fragment variant for a plain-form solve (Hermitian halved 7x7 box; either solver), or
// null.  HHG_DFRAG=0 turns it off (measurements).
const DfragVariant* find_dfrag(const SolveTables& t) {
  if (const char* env = std::getenv("HHG_DFRAG"))
    if (env[0] == '0') return nullptr;
  const GroupGeom gg = group_geom(t);
  if (!t.hermitian || !gg.half || t.b1n != 7 || t.b2n != 7) return nullptr;
  for (const DfragVariant& v : kDfragVariants)
    if (v.nw == t.nw && v.nax == t.nax && v.nj == t.nj && v.km == (t.kmode != 0)) return &v;
  return nullptr;
}

struct FragVariant {
  int nw, nax, nj, kpc;
  bool (*plan)(const SolveTables&, int, LaunchShape*, char*, int);
  int (*launch)(const SolveTables&, const GroupTables&, const LaunchShape&, double2*, double2*, cudaStream_t);
};
#define HHG_FRAG_VARIANT(NW, NAX, NJ, KPC) {NW, NAX, NJ, KPC, plan_frag_t<NW, NAX, NJ, KPC>, launch_frag_t<NW, NAX, NJ, KPC>}
const FragVariant kFragVariants[] = {
    HHG_FRAG_VARIANT(11, 1, 2, 16), HHG_FRAG_VARIANT(11, 2, 2, 16), HHG_FRAG_VARIANT(12, 1, 2, 16),
    HHG_FRAG_VARIANT(12, 2, 2, 16), HHG_FRAG_VARIANT(11, 1, 2, 8),  HHG_FRAG_VARIANT(11, 2, 2, 8),
    HHG_FRAG_VARIANT(12, 1, 2, 8),  HHG_FRAG_VARIANT(12, 2, 2, 8),
};
#undef HHG_FRAG_VARIANT

// The fragment variant for a mixed-form solve (Hermitian halved 7x7 box, real-space solver), or null.
// tile_hint in 1..8 picks the 8-k-point CTAs.  The kernel is opt-in (HHG_FRAG=1): its tensor-core
// products accumulate with round-toward-zero and it is slower than the element-group kernel (see
// sbe_frag.cuh).  HHG_FRAG_KPC=8|16 fixes the k-points per CTA.
const FragVariant* find_frag(const SolveTables& t, int tile_hint) {
  const char* on = std::getenv("HHG_FRAG");
  if (!on || on[0] != '1') return nullptr;
  const GroupGeom gg = group_geom(t);
  if (t.kmode || !t.hermitian || !gg.half || t.b1n != 7 || t.b2n != 7) return nullptr;
  int kpc = (tile_hint > 0 && tile_hint <= 8) ? 8 : 16;
  if (const char* env = std::getenv("HHG_FRAG_KPC")) kpc = std::atoi(env) == 8 ? 8 : 16;
  for (const FragVariant& v : kFragVariants)
    if (v.nw == t.nw && v.nax == t.nax && v.nj == t.nj && v.kpc == kpc) return &v;
  return nullptr;
}

// Compiled shapes: (orbitals, field axes, current axes) of the configurations this library is built
// for, each in plain FP64 (one element per thread) and mixed precision (two elements per thread);
// any other shape runs the runtime-shaped instance.
using PlanFn = bool (*)(const SolveTables&, int, LaunchShape*, char*, int, int);
using LaunchFn = int (*)(const SolveTables&, const GroupTables&, const LaunchShape&, double2*, double2*, cudaStream_t);
using BatchFn = int (*)(const BatchDesc*, const int2*, int, int*, int, size_t, int, cudaStream_t);
struct GroupVariant {
  int precision, nw, nax, nj, wb;  // wb > 0: square wb x wb cell box with Hermitian halving
  bool kp;                          // k-point pairs
  bool pg;                          // precomputed inner sums
  bool km;                          // k-space solver instance
  PlanFn plan;
  LaunchFn launch;
  BatchFn batch;
};
#define HHG_GROUP_VARIANT_X(P, R, E, NW, NAX, NJ, WB, KP, PG)                                      \
  {P, NW, NAX, NJ, WB, KP, PG, false, plan_group_t<R, E, NW, NAX, NJ, false, WB, KP, PG>,           \
   launch_group_t<R, E, NW, NAX, NJ, false, WB, KP, PG>, launch_group_batch_t<R, E, NW, NAX, NJ, false, WB, KP>}
#define HHG_GROUP_VARIANT(P, R, E, NW, NAX, NJ, WB) HHG_GROUP_VARIANT_X(P, R, E, NW, NAX, NJ, WB, false, false)
#define HHG_GROUP_VARIANT_KM(P, R, E, NW, NAX, NJ, WB, PG)                                         \
  {P, NW, NAX, NJ, WB, false, PG, true, plan_group_t<R, E, NW, NAX, NJ, true, WB, false, PG>,      \
   launch_group_t<R, E, NW, NAX, NJ, true, WB, false, PG>, launch_group_batch_t<R, E, NW, NAX, NJ, true, WB>}
// Listed in order of preference: a solve runs the first one that matches it.  (The persistent batch
// launch of a precomputed-sum shape runs its in-kernel-sum instance.)
const GroupVariant kGroupVariants[] = {
    HHG_GROUP_VARIANT_X(1, float, 2, 11, 1, 2, 7, true, true),  HHG_GROUP_VARIANT_X(1, float, 2, 11, 2, 2, 7, true, true),
    HHG_GROUP_VARIANT_X(1, float, 2, 12, 1, 2, 7, true, true),  HHG_GROUP_VARIANT_X(1, float, 2, 12, 2, 2, 7, true, true),
    HHG_GROUP_VARIANT_X(1, float, 2, 6, 1, 2, 7, true, true),   HHG_GROUP_VARIANT_X(1, float, 2, 6, 2, 2, 7, true, true),
    HHG_GROUP_VARIANT_X(0, double, 1, 6, 1, 2, 7, false, true), HHG_GROUP_VARIANT_X(0, double, 1, 6, 2, 2, 7, false, true),
    HHG_GROUP_VARIANT_X(1, float, 2, 11, 1, 2, 7, true, false), HHG_GROUP_VARIANT_X(1, float, 2, 11, 2, 2, 7, true, false),
    HHG_GROUP_VARIANT_X(1, float, 2, 12, 1, 2, 7, true, false), HHG_GROUP_VARIANT_X(1, float, 2, 12, 2, 2, 7, true, false),
    HHG_GROUP_VARIANT_X(1, float, 2, 6, 1, 2, 7, true, false),  HHG_GROUP_VARIANT_X(1, float, 2, 6, 2, 2, 7, true, false),
    HHG_GROUP_VARIANT_X(0, double, 1, 11, 1, 2, 7, false, true), HHG_GROUP_VARIANT_X(0, double, 1, 11, 2, 2, 7, false, true),
    HHG_GROUP_VARIANT_X(0, double, 1, 12, 1, 2, 7, false, true), HHG_GROUP_VARIANT_X(0, double, 1, 12, 2, 2, 7, false, true),
    HHG_GROUP_VARIANT_X(1, float, 2, 12, 1, 2, 7, false, true),  HHG_GROUP_VARIANT_X(1, float, 2, 12, 2, 2, 7, false, true),
    HHG_GROUP_VARIANT(0, double, 1, 11, 1, 2, 7), HHG_GROUP_VARIANT(0, double, 1, 11, 2, 2, 7),
    HHG_GROUP_VARIANT(0, double, 1, 12, 1, 2, 7), HHG_GROUP_VARIANT(0, double, 1, 12, 2, 2, 7),
    HHG_GROUP_VARIANT(1, float, 2, 11, 1, 2, 7),  HHG_GROUP_VARIANT(1, float, 2, 11, 2, 2, 7),
    HHG_GROUP_VARIANT(1, float, 2, 12, 1, 2, 7),  HHG_GROUP_VARIANT(1, float, 2, 12, 2, 2, 7),
    HHG_GROUP_VARIANT(0, double, 1, 11, 1, 2, 0), HHG_GROUP_VARIANT(0, double, 1, 11, 2, 2, 0),
    HHG_GROUP_VARIANT(0, double, 1, 12, 1, 2, 0), HHG_GROUP_VARIANT(0, double, 1, 12, 2, 2, 0),
    HHG_GROUP_VARIANT(0, double, 1, 6, 1, 2, 0),  HHG_GROUP_VARIANT(0, double, 1, 6, 2, 2, 0),
    HHG_GROUP_VARIANT(1, float, 2, 11, 1, 2, 0),  HHG_GROUP_VARIANT(1, float, 2, 11, 2, 2, 0),
    HHG_GROUP_VARIANT(1, float, 2, 12, 1, 2, 0),  HHG_GROUP_VARIANT(1, float, 2, 12, 2, 2, 0),
    HHG_GROUP_VARIANT(1, float, 1, 6, 1, 2, 0),   HHG_GROUP_VARIANT(1, float, 1, 6, 2, 2, 0),
    HHG_GROUP_VARIANT(1, float, 1, 2, 1, 2, 0),   HHG_GROUP_VARIANT(1, float, 1, 2, 2, 2, 0),
    // k-space solver (three evaluation points per step): the compiled 7x7 box only.
    HHG_GROUP_VARIANT_KM(0, double, 1, 11, 1, 2, 7, true), HHG_GROUP_VARIANT_KM(0, double, 1, 11, 2, 2, 7, true),
    HHG_GROUP_VARIANT_KM(0, double, 1, 12, 1, 2, 7, true), HHG_GROUP_VARIANT_KM(0, double, 1, 12, 2, 2, 7, true),
    HHG_GROUP_VARIANT_KM(1, float, 2, 11, 1, 2, 7, true),  HHG_GROUP_VARIANT_KM(1, float, 2, 11, 2, 2, 7, true),
    HHG_GROUP_VARIANT_KM(1, float, 2, 12, 1, 2, 7, true),  HHG_GROUP_VARIANT_KM(1, float, 2, 12, 2, 2, 7, true),
    HHG_GROUP_VARIANT_KM(0, double, 1, 11, 1, 2, 7, false), HHG_GROUP_VARIANT_KM(0, double, 1, 11, 2, 2, 7, false),
    HHG_GROUP_VARIANT_KM(0, double, 1, 12, 1, 2, 7, false), HHG_GROUP_VARIANT_KM(0, double, 1, 12, 2, 2, 7, false),
    HHG_GROUP_VARIANT_KM(1, float, 2, 11, 1, 2, 7, false),  HHG_GROUP_VARIANT_KM(1, float, 2, 11, 2, 2, 7, false),
    HHG_GROUP_VARIANT_KM(1, float, 2, 12, 1, 2, 7, false),  HHG_GROUP_VARIANT_KM(1, float, 2, 12, 2, 2, 7, false),
};
#undef HHG_GROUP_VARIANT
#undef HHG_GROUP_VARIANT_X
#undef HHG_GROUP_VARIANT_KM

const GroupVariant* find_variant(const SolveTables& t, int precision) {
  if (const char* env = std::getenv("HHG_GROUP_GENERIC"))
    if (env[0] == '1') return nullptr;  // tuning override: runtime-shaped instance
  const bool any_box = [] {
    const char* env = std::getenv("HHG_GROUP_ANYBOX");  // tuning override: skip the fixed-box variants
    return env && env[0] == '1';
  }();
  const bool no_pair = [] {
    const char* env = std::getenv("HHG_GROUP_NOPAIR");  // tuning override: skip the k-point-pair variants
    return env && env[0] == '1';
  }();
  const bool no_pre = [] {
    const char* env = std::getenv("HHG_GROUP_NOPRE");  // tuning override: skip the precomputed-sum variants
    return env && env[0] == '1';
  }();
  const GroupGeom gg = group_geom(t);
  for (const GroupVariant& v : kGroupVariants) {
    if (v.precision != precision || v.nw != t.nw || v.nax != t.nax || v.nj != t.nj) continue;
    if (v.km != (t.kmode != 0)) continue;
    if (v.wb > 0 && (any_box || !gg.half || t.b1n != v.wb || t.b2n != v.wb)) continue;
    if (v.kp && no_pair) continue;
    if (v.pg && no_pre) continue;
    return &v;
  }
  return nullptr;
}

}  // namespace

bool plan_group(const SolveTables& t, int precision, int sm_count, LaunchShape* out, char* why, int why_len,
                int tile_hint) {
  if (precision == 0)
    if (const DfragVariant* f = find_dfrag(t)) {
      out->variant = (int)(f - kDfragVariants);
      if (f->plan(t, sm_count, out, why, why_len)) return true;
    }
  if (precision == 1)  // (the opt-in fragment kernel first: HHG_FRAG=1 asks for it)
    if (const FragVariant* f = find_frag(t, tile_hint)) {
      out->variant = (int)(f - kFragVariants);
      if (f->plan(t, sm_count, out, why, why_len)) return true;
    }
  if (precision == 1)
    if (const MtileVariant* m = find_mtile(t)) {
      out->variant = (int)(m - kMtileVariants);
      if (m->plan(t, sm_count, out, why, why_len)) return true;
    }
  if (const GroupVariant* v = find_variant(t, precision)) {
    out->variant = (int)(v - kGroupVariants);
    return v->plan(t, sm_count, out, why, why_len, tile_hint);
  }
  out->variant = -1;
  // Runtime-shaped: two elements per thread in the mixed form once a k-point needs more than a warp.
  const bool two = precision == 1 && t.nw2 > 32;
  if (t.kmode) {
    if (precision == 1)
      return two ? plan_group_t<float, 2, 0, 0, 0, true>(t, sm_count, out, why, why_len, tile_hint)
                 : plan_group_t<float, 1, 0, 0, 0, true>(t, sm_count, out, why, why_len, tile_hint);
    return plan_group_t<double, 1, 0, 0, 0, true>(t, sm_count, out, why, why_len, tile_hint);
  }
  if (precision == 1)
    return two ? plan_group_t<float, 2, 0, 0, 0>(t, sm_count, out, why, why_len, tile_hint)
               : plan_group_t<float, 1, 0, 0, 0>(t, sm_count, out, why, why_len, tile_hint);
  return plan_group_t<double, 1, 0, 0, 0>(t, sm_count, out, why, why_len, tile_hint);
}

namespace {
template <bool KM>
int launch_group_batch_generic(const LaunchShape& s, const BatchDesc* descs, const int2* items, int nitems,
                               int* counter, size_t smem, int sm_count, cudaStream_t stream) {
  if (s.kernel == 2)
    return s.ept == 2 ? launch_group_batch_t<float, 2, 0, 0, 0, KM>(descs, items, nitems, counter, s.threads, smem,
                                                                     sm_count, stream)
                      : launch_group_batch_t<float, 1, 0, 0, 0, KM>(descs, items, nitems, counter, s.threads, smem,
                                                                     sm_count, stream);
  return launch_group_batch_t<double, 1, 0, 0, 0, KM>(descs, items, nitems, counter, s.threads, smem, sm_count,
                                                      stream);
}
template <bool KM>
int launch_group_generic(const SolveTables& t, const GroupTables& gt, const LaunchShape& s, double2* rho,
                         double2* Jpart, cudaStream_t stream) {
  if (s.kernel == 2)
    return s.ept == 2 ? launch_group_t<float, 2, 0, 0, 0, KM>(t, gt, s, rho, Jpart, stream)
                      : launch_group_t<float, 1, 0, 0, 0, KM>(t, gt, s, rho, Jpart, stream);
  return launch_group_t<double, 1, 0, 0, 0, KM>(t, gt, s, rho, Jpart, stream);
}
}  // namespace

int launch_group_batch(const LaunchShape& s, const BatchDesc* descs, const int2* items, int nitems, int* counter,
                       size_t smem, int sm_count, cudaStream_t stream) {
  if (s.variant >= 0)
    return kGroupVariants[s.variant].batch(descs, items, nitems, counter, s.threads, smem, sm_count, stream);
  return s.kmode ? launch_group_batch_generic<true>(s, descs, items, nitems, counter, smem, sm_count, stream)
                 : launch_group_batch_generic<false>(s, descs, items, nitems, counter, smem, sm_count, stream);
}

int launch_group(const SolveTables& t, const GroupTables& gt, const LaunchShape& s, double2* rho, double2* Jpart,
                 cudaStream_t stream) {
  if (s.kernel == 4) return kFragVariants[s.variant].launch(t, gt, s, rho, Jpart, stream);
  if (s.kernel == 5) return kDfragVariants[s.variant].launch(t, gt, s, rho, Jpart, stream);
  if (s.kernel == 6) return kMtileVariants[s.variant].launch(t, gt, s, rho, Jpart, stream);
  if (s.variant >= 0) return kGroupVariants[s.variant].launch(t, gt, s, rho, Jpart, stream);
  if (s.kmode) return launch_group_generic<true>(t, gt, s, rho, Jpart, stream);
  return launch_group_generic<false>(t, gt, s, rho, Jpart, stream);
}

}  // namespace hhg
