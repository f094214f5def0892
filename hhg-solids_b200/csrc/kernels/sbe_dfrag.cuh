// FP64 tensor-core form of the plain propagation for 9..16 orbitals (included by sbe_group.cu, inside
// its anonymous namespace: it uses GroupData, the precomputed inner sums of group_sums_kernel and the
// helpers defined there).
//
// Same propagation as group_vctas in FP64 (k-space-resident RK4 of the reference's
// src/solver.cpp:86-181, 1428-1726, and the windowed current of src/observable.cpp:16-30), for solves
// whose cell box is the Hermitian-halved 7x7 one and whose inner Wannier sums come precomputed per
// column and step.  The products run on the FP64 tensor cores (mma.m8n8k4.f64: IEEE double products
// and sums, no splitting, no precision lost against the FP64 pipe).
//
// Layout.  A CTA holds KPC = 8 consecutive k-points (rows m1) of one k-grid column, one warp per
// k-point.  A k-point's nw x nw matrices live in a 16 x 16 frame spread over its warp in the layout
// of the m8n8k4 accumulator: lane (g = lane/4, c = lane%4) holds frame rows g, g+8 and frame columns
// 2c, 2c+1, 8+2c, 9+2c ("slots" s = 4 rb + 2 cb + e: row 8 rb + g, column 8 cb + 2c + e).  Orbital
// o sits at frame position o for o < 8 and 8 + 2 (o - 8) beyond, so positions 9, 11, 13 and 15 stay
// empty and the product needs three k-steps instead of four.
//
//  * Commutator.  k-step (cb, e) contracts frame columns 8 cb + 2c + e (c = 0..3 of the lanes): its A
//    operand (A[g][c] = H[8 rb + g][8 cb + 2c + e]) is the lane's slot (rb, cb, e) of H, and because X
//    is Hermitian its B operand (B[c][g] = X[8 cb + 2c + e][8 nb + g] = conj(X[8 nb + g][8 cb + 2c + e]))
//    is the conjugate of the lane's slot (nb, cb, e) of X.  So P = H X (four 8 x 8 blocks, 36 mma per
//    stage: three real products per complex one) is formed from registers, P^+ comes from the same registers by
//    movmatrix transposes of the 16-bit pieces of each double, and k = -i (P - P^+) and the next
//    stage's X = rho + c k stay in the lane's slots.
//  * Outer Wannier sums.  H0(k) and r_a(k) of the CTA's 8 k-points are one complex GEMM per step,
//    [8 k-points x 8] x [8 x nw^2] (A = the phases of the seven box rows and a zero row, B = the inner
//    sums G(n1), G(-n1) = G(n1)^+ read transposed), on the same tensor cores; its result goes through
//    shared memory to the k-point warps.
//  * Window velocity and current on the FP64 pipe in a dense layout (each thread one k-point and a
//    strided set of elements, so no lane idles on the frame's padding); the state rho is kept in
//    registers through the step and in shared memory for the current.

namespace dfrag {

// (not volatile: the compiler may interleave independent accumulations to hide the mma latency)
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ unsigned movmatrix_trans(unsigned x) {
  unsigned r;
  asm volatile("movmatrix.sync.aligned.m8n8.trans.b16 %0, %1;" : "=r"(r) : "r"(x));
  return r;
}
// Transposes an 8 x 8 block of doubles held as (row g, columns 2c, 2c+1) pairs: each of the four
// 16-bit pieces of the two doubles goes through one b16 transpose.
__device__ __forceinline__ void transpose8(double& a, double& b) {
  const unsigned a0 = __double2loint(a), a1 = __double2hiint(a), b0 = __double2loint(b), b1 = __double2hiint(b);
  const unsigned p0 = movmatrix_trans(__byte_perm(a0, b0, 0x5410)), p1 = movmatrix_trans(__byte_perm(a0, b0, 0x7632));
  const unsigned p2 = movmatrix_trans(__byte_perm(a1, b1, 0x5410)), p3 = movmatrix_trans(__byte_perm(a1, b1, 0x7632));
  a = __hiloint2double((int)__byte_perm(p2, p3, 0x5410), (int)__byte_perm(p0, p1, 0x5410));
  b = __hiloint2double((int)__byte_perm(p2, p3, 0x7632), (int)__byte_perm(p0, p1, 0x7632));
}

// Orbital at frame position p (or -1): o at o < 8, at 8 + 2 (o - 8) beyond.
__device__ __forceinline__ int frame_orbital(int p, int nw) {
  const int o = p < 8 ? p : ((p & 1) ? 99 : 8 + (p - 8) / 2);
  return o < nw ? o : -1;
}

template <int NW, int NAX, int NJ, bool KM>
struct Geom {
  static constexpr int KPC = 8;
  static constexpr int NW2 = NW * NW;
  static constexpr int NMAT = 1 + NAX;
  static constexpr int NBROWS = NMAT * 4;      // halved 7 x 7 box: inner-sum rows n1 = 0..3 per matrix
  static constexpr int NWROWS = NJ * 4;        // window rows
  static constexpr int NTILE = (NW2 + 7) / 8;  // n-tiles of one matrix in the outer sums
  // Outer-sum buffers: one point per step (real-space solver), or the k-space solver's points t (carried
  // from the previous step, two buffers by step parity), t + dt/2 and t + dt.
  static constexpr int NHK = KM ? 3 : 1;
  // Inner-sum buffers: real-space solver, this step's point and the next one's (prefetched); k-space
  // solver, the step's two new points (refilled for the next step once the outer sums have read them).
  // Window rows: per point and double-buffered (real-space solver), constant (k-space solver).
  static constexpr int NWB = KM ? 1 : 2;
  static constexpr size_t RHO = 0;                                       // [KPC][NW2] double2
  static constexpr size_t HK = RHO + (size_t)KPC * NW2 * 16;             // [NHK][KPC][NMAT][NW2] double2
  static constexpr size_t GS = HK + (size_t)NHK * KPC * NMAT * NW2 * 16;  // [2][NBROWS][NW2] double2
  static constexpr size_t GWS = GS + 2 * (size_t)NBROWS * NW2 * 16;      // [NWB][NWROWS][NW2] double2
  static constexpr size_t TW1 = GWS + (size_t)NWB * NWROWS * NW2 * 16;   // [KPC][8] double2
  static constexpr size_t WTW1 = TW1 + (size_t)KPC * 8 * 16;             // [KPC][4] double2
  static constexpr size_t SJ = WTW1 + (size_t)KPC * 4 * 16;              // [2][kJRing][KPC][2 NJ] double
  static constexpr size_t BYTES = SJ + 2 * (size_t)kJRing * KPC * 2 * NJ * 8;
  static_assert(NW > 8 && NW <= 12, "frame: 9..12 orbitals (positions 0..7, 8, 10, 12, 14)");
};

// KM: the reference's k-space solver (src/solver_kspace.cpp:167-270): the stages see H at points
// 2 ti (t), 2 ti + 1 (t + dt/2) and 2 ti + 2 (t + dt) of the interpolation tables, and the window of
// the current has no phase (its sums are one block per column).
template <int NW, int NAX, int NJ, bool KM>
__global__ void __launch_bounds__(256, 1)
    propagate_dfrag_kernel(SolveTables t, GroupData<double> d, int vctas, double2* rho, double2* Jpart) {
  using FG = Geom<NW, NAX, NJ, KM>;
  constexpr int KPC = FG::KPC, NW2 = FG::NW2, NMAT = FG::NMAT, NTILE = FG::NTILE;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* RHO = reinterpret_cast<double2*>(smraw + FG::RHO);
  double2* HK = reinterpret_cast<double2*>(smraw + FG::HK);
  double2* GS = reinterpret_cast<double2*>(smraw + FG::GS);
  double2* GWS = reinterpret_cast<double2*>(smraw + FG::GWS);
  double2* TW1 = reinterpret_cast<double2*>(smraw + FG::TW1);
  double2* WTW1 = reinterpret_cast<double2*>(smraw + FG::WTW1);
  double* SJ = reinterpret_cast<double*>(smraw + FG::SJ);

  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, g = lane >> 2, c4 = lane & 3;
  constexpr int NTHR = KPC * 32;
  const int rows = t.row1 - t.row0, bpc = (rows + KPC - 1) / KPC, ntiles = t.N2 * bpc;
  const int step0 = t.step0, step1 = t.step1, npw = 2 * t.np + 1;
  const double dt = t.dt, prefac = 0.1666666666666 * dt;
  constexpr size_t gbuf = (size_t)FG::NBROWS * NW2, wbuf = (size_t)FG::NWROWS * NW2, hbuf = (size_t)KPC * NMAT * NW2;
  const double2 dzero = make_double2(0.0, 0.0);

  // This lane's slots: element index (or -1 on the frame's padding).
  int el[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const int orow = frame_orbital(8 * (s >> 2) + g, NW), ocol = frame_orbital(8 * ((s >> 1) & 1) + 2 * c4 + (s & 1), NW);
    el[s] = (orow >= 0 && ocol >= 0) ? orow * NW + ocol : -1;
  }
  // Outer-sum buffer of evaluation point p (k-space solver: even points by step parity, odd ones in one).
  auto hk_of = [&](int p) { return KM ? HK + (size_t)((p & 1) ? 2 : (p >> 1) & 1) * hbuf : HK; };

  for (int v = blockIdx.x; v < vctas; v += gridDim.x)
    for (int tile = v; tile < ntiles; tile += vctas) {
      const int m2 = tile / bpc, m10 = t.row0 + (tile % bpc) * KPC;
      const int nown = min(KPC, t.row1 - m10);

      // Inner sums of point p into GS[slot] (and, real-space solver, its window rows into GWS[slot]).
      auto fetch_point = [&](int p, int slot) {
        const size_t blk = (size_t)(p - (KM ? 2 * step0 : step0)) * t.N2 + m2;
        const double2* src = d.Gpre + blk * gbuf;
        double2* dst = GS + (size_t)slot * gbuf;
        const int nw_rows = KM ? 0 : (int)wbuf;
        const double2* wsrc = d.GWpre + blk * wbuf;
        double2* wdst = GWS + (size_t)slot * wbuf;
        for (int idx = tid; idx < (int)gbuf + nw_rows; idx += NTHR) {
          if (idx < (int)gbuf)
            cp_async16(dst + idx, src + idx);
          else
            cp_async16(wdst + (idx - gbuf), wsrc + (idx - gbuf));
        }
      };
      auto flush = [&](int ti_end) {
        const int slot = (ti_end / kJRing) & 1, s = ti_end % kJRing;
        const int ti0 = max(ti_end - s, step0), nsteps = ti_end - ti0 + 1;
        const double* half = SJ + ((size_t)slot * kJRing + (ti0 % kJRing)) * KPC * 2 * NJ;
        for (int idx = tid; idx < nsteps * NJ; idx += NTHR) {
          const int ss = idx / NJ, a = idx % NJ;
          double re = 0.0, im = 0.0;
          for (int ww = 0; ww < KPC; ++ww) {
            re += half[(ss * KPC + ww) * 2 * NJ + 2 * a];
            im += half[(ss * KPC + ww) * 2 * NJ + 2 * a + 1];
          }
          const int ja = a == 0 ? t.j_id[0] : (a == 1 ? t.j_id[1] : t.j_id[2]);
          double2* dst = Jpart + ((size_t)v * t.nt + ti0 + ss) * 3 + ja;
          const double2 old = *dst;
          *dst = make_double2(old.x + re, old.y + im);
        }
      };
      // Outer sums of point p from GS[slot]: HK(p)[m][mat][e] = sum_q p1(m, q) G(mat, n1 = q - 3)_e.
      auto outer_sums = [&](int p, int slot) {
        const double2* P1 = d.P + (size_t)p * 2 * npw + t.np;
        double2 pa[2];  // A[g][c] of k-steps 0 and 1: p1(k-point g, box row c and c + 4)
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
          const int q = c4 + 4 * ks;
          pa[ks] = q < 7 ? mul(TW1[g * 8 + q], P1[t.b1lo + q]) : dzero;
        }
        const double2* G = GS + (size_t)slot * gbuf;
        double2* HKp = hk_of(p);
        // The warp's n-tiles nt = w, w + KPC, ... together, so that their accumulations interleave.
        constexpr int NTW = (NMAT * NTILE + KPC - 1) / KPC;
        double2 b0[NTW], b1[NTW];
#pragma unroll
        for (int u = 0; u < NTW; ++u) {
          const int nt_ = w + u * KPC, mat = nt_ / NTILE, j = nt_ % NTILE, e = 8 * j + g;
          // B[c][g] of k-step 0: G(n1 = c - 3)_e (row 3 - c, transposed and conjugated for n1 < 0);
          // of k-step 1: G(n1 = c + 1)_e (c + 4 = 7 is the zero row).
          b0[u] = dzero;
          b1[u] = dzero;
          if (nt_ < NMAT * NTILE && e < NW2) {
            const double2* Gm = G + (size_t)mat * 4 * NW2;
            if (c4 == 3) {
              b0[u] = Gm[e];
            } else {
              const double2 vv = Gm[(3 - c4) * NW2 + (e % NW) * NW + e / NW];
              b0[u] = make_double2(vv.x, -vv.y);
              b1[u] = Gm[(c4 + 1) * NW2 + e];
            }
          }
        }
        // Complex products with three real ones (Gauss): T1 = pr gr, T2 = pi gi, T3 = (pr + pi)(gr + gi),
        // re = T1 - T2, im = T3 - T1 - T2.
        double t1[NTW][2], t2[NTW][2], t3[NTW][2];
#pragma unroll
        for (int u = 0; u < NTW; ++u) t1[u][0] = t1[u][1] = t2[u][0] = t2[u][1] = t3[u][0] = t3[u][1] = 0.0;
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
          const double ps = pa[ks].x + pa[ks].y;
#pragma unroll
          for (int u = 0; u < NTW; ++u) dmma(t1[u], pa[ks].x, ks ? b1[u].x : b0[u].x);
#pragma unroll
          for (int u = 0; u < NTW; ++u) dmma(t2[u], pa[ks].y, ks ? b1[u].y : b0[u].y);
#pragma unroll
          for (int u = 0; u < NTW; ++u) dmma(t3[u], ps, ks ? b1[u].x + b1[u].y : b0[u].x + b0[u].y);
        }
#pragma unroll
        for (int u = 0; u < NTW; ++u) {
          const int nt_ = w + u * KPC, mat = nt_ / NTILE, j = nt_ % NTILE;
          const int e0 = 8 * j + 2 * c4;  // results (k-point g, e0) and (g, e0 + 1)
          if (nt_ < NMAT * NTILE) {
            double2* dst = HKp + ((size_t)g * NMAT + mat) * NW2;
            if (e0 < NW2) dst[e0] = make_double2(t1[u][0] - t2[u][0], t3[u][0] - t1[u][0] - t2[u][0]);
            if (e0 + 1 < NW2) dst[e0 + 1] = make_double2(t1[u][1] - t2[u][1], t3[u][1] - t1[u][1] - t2[u][1]);
          }
        }
      };

      for (int idx = tid; idx < KPC * NW2; idx += NTHR) {
        const int m = idx / NW2, e = idx % NW2;
        RHO[idx] = m < nown ? rho[((size_t)(m10 + m) * t.N2 + m2) * NW2 + e] : dzero;
      }
      for (int idx = tid; idx < KPC * 8; idx += NTHR) {
        const int m = idx / 8, q = idx % 8, m1 = min(m10 + m, t.row1 - 1);
        TW1[idx] = q < 7 ? d.T1[wrap_mod((long long)m1 * (t.b1lo + q), t.N1)] : dzero;
      }
      for (int idx = tid; idx < KPC * 4; idx += NTHR) {
        const int m = idx / 4, q = idx % 4, m1 = min(m10 + m, t.row1 - 1);
        WTW1[idx] = d.T1d[wrap_mod((long long)m1 * (q - 2), t.N1)];
      }
      if constexpr (KM) {
        // The chunk's first point t (then carried from step to step) and the constant window rows.
        fetch_point(2 * step0, 0);
        for (int idx = tid; idx < (int)wbuf; idx += NTHR) cp_async16(GWS + idx, d.GWpre + (size_t)m2 * wbuf + idx);
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        outer_sums(2 * step0, 0);
        __syncthreads();
        fetch_point(2 * step0 + 1, 0);
        fetch_point(2 * step0 + 2, 1);
      } else {
        fetch_point(step0, step0 & 1);
      }
      cp_async_commit();
      cp_async_wait_all();
      __syncthreads();
      // This warp's state in its slots (registers for the whole tile; RHO mirrors it for the current).
      double2 r64[8];
#pragma unroll
      for (int s = 0; s < 8; ++s) r64[s] = (w < nown && el[s] >= 0) ? RHO[w * NW2 + el[s]] : dzero;

      for (int ti = step0; ti < step1; ++ti) {
        const int buf = ti & 1;
        // (1) Outer sums: the step's point (real-space solver), or its points t + dt/2 and t + dt.
        if constexpr (KM) {
          outer_sums(2 * ti + 1, 0);
          outer_sums(2 * ti + 2, 1);
        } else {
          outer_sums(ti, buf);
        }
        __syncthreads();
        if (ti > step0 && (ti - 1) % kJRing == kJRing - 1) flush(ti - 1);
        // The next step's inner sums (the buffers the outer sums just read, or the other one).
        if (ti + 1 < step1) {
          if constexpr (KM) {
            fetch_point(2 * ti + 3, 0);
            fetch_point(2 * ti + 4, 1);
          } else {
            fetch_point(ti + 1, (ti + 1) & 1);
          }
          cp_async_commit();
        }

        // (2) RK4 stages of this warp's k-point (src/solver.cpp:157-180), fields at t, t+dt/2, t+dt/2, t+dt.
        if (w < nown) {
          double2 S[8], X[8], H[8];
#pragma unroll
          for (int s = 0; s < 8; ++s) {
            S[s] = dzero;
            X[s] = r64[s];
          }
          const double* esb = t.es + (size_t)ti * 9;
#pragma unroll 1
          for (int st = 0; st < 4; ++st) {
            const int f = st == 0 ? 0 : (st == 3 ? 2 : 1);
            // k-space solver: the stage's evaluation point 2 ti + f
            const double2* Hm = (KM ? hk_of(2 * ti + f) : HK) + (size_t)w * NMAT * NW2;
            double ea[NAX];
#pragma unroll
            for (int a = 0; a < NAX; ++a) ea[a] = esb[f * 3 + t.ax_id[a]];
            // (the second and third stages share the field and point at t + dt/2: the third keeps the
            // second's H)
#pragma unroll
            for (int s = 0; s < 8; ++s) {
              if (st == 2) continue;
              H[s] = dzero;
              if (el[s] >= 0) {
                H[s] = Hm[el[s]];
#pragma unroll
                for (int a = 0; a < NAX; ++a) {
                  const double2 rv = Hm[(1 + a) * NW2 + el[s]];
                  H[s].x = fma(ea[a], rv.x, H[s].x);
                  H[s].y = fma(ea[a], rv.y, H[s].y);
                }
              }
            }
            // P = H X over k-steps (cb, e) = (0, 0), (0, 1), (1, 0) (frame columns 9, 11, 13, 15 are
            // empty), with B = conj(X slots) and three real products per complex one (Gauss):
            // T1 = Hr Xr, T2 = Hi (-Xi), T3 = (Hr + Hi)(Xr - Xi); Re P = T1 - T2, Im P = T3 - T1 - T2.
            // Block by block, diagonal blocks first, each block's three accumulations interleaved, so
            // that the transposes of finished blocks can overlap the products of the later ones.
            double t1[2][2][2], t2[2][2][2], t3[2][2][2];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int rb = q < 2 ? q : 0, nb = q < 2 ? q : 1;  // (0,0), (1,1), (0,1), (1,0)
              const int rr = q == 3 ? 1 : rb, nn = q == 3 ? 0 : nb;
              t1[rr][nn][0] = t1[rr][nn][1] = t2[rr][nn][0] = t2[rr][nn][1] = t3[rr][nn][0] = t3[rr][nn][1] = 0.0;
#pragma unroll
              for (int ks = 0; ks < 3; ++ks) {
                const int cb = ks >> 1, e = ks & 1;
                const double2 a = H[4 * rr + 2 * cb + e], b = X[4 * nn + 2 * cb + e];
                dmma(t1[rr][nn], a.x, b.x);
                dmma(t2[rr][nn], a.y, -b.y);
                dmma(t3[rr][nn], a.x + a.y, b.x - b.y);
              }
            }
            double pr[2][2][2], pim[2][2][2];
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
              for (int i = 0; i < 2; ++i) {
                pr[q >> 1][q & 1][i] = t1[q >> 1][q & 1][i] - t2[q >> 1][q & 1][i];
                pim[q >> 1][q & 1][i] = t3[q >> 1][q & 1][i] - t1[q >> 1][q & 1][i] - t2[q >> 1][q & 1][i];
              }
            // k = -i (P - P^+): block (rb, nb) of P^+ is block (nb, rb) of P transposed, conjugated.
            const double wgt = (st == 0 || st == 3) ? 1.0 : 2.0;
            const double cn = (st == 2 ? 1.0 : 0.5) * dt;
#pragma unroll
            for (int rb = 0; rb < 2; ++rb)
#pragma unroll
              for (int nb = 0; nb < 2; ++nb) {
                double tr0 = pr[nb][rb][0], tr1 = pr[nb][rb][1], ti0 = pim[nb][rb][0], ti1 = pim[nb][rb][1];
                transpose8(tr0, tr1);
                transpose8(ti0, ti1);
                const double Dr[2] = {tr0, tr1}, Di[2] = {-ti0, -ti1};
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                  const int s = 4 * rb + 2 * nb + e;
                  const double kx = pim[rb][nb][e] - Di[e], ky = -(pr[rb][nb][e] - Dr[e]);
                  S[s].x = fma(wgt, kx, S[s].x);
                  S[s].y = fma(wgt, ky, S[s].y);
                  X[s].x = fma(cn, kx, r64[s].x);
                  X[s].y = fma(cn, ky, r64[s].y);
                }
              }
          }
          // rho += dt/6 (k1 + 2 k2 + 2 k3 + k4) (src/solver.cpp:170-180)
#pragma unroll
          for (int s = 0; s < 8; ++s) {
            r64[s].x = r64[s].x + prefac * S[s].x;
            r64[s].y = r64[s].y + prefac * S[s].y;
            if (el[s] >= 0) RHO[w * NW2 + el[s]] = r64[s];
          }
        }
        if (ti + 1 < step1) cp_async_wait_all();
        __syncthreads();

        // (3) Current partials of step ti (FP64): thread = k-point m, elements e = w 4 + sub + 32 p.
        {
          const int m = lane % KPC, sub = lane / KPC;
          // (the k-space solver's window carries no phase)
          const double2* P1d = d.Pd + (size_t)ti * 2 * npw + t.np;
          double2 wp[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) wp[q] = KM ? WTW1[m * 4 + q] : mul(WTW1[m * 4 + q], P1d[q - 2]);
          double re[3] = {0.0, 0.0, 0.0}, im[3] = {0.0, 0.0, 0.0};
          const double2* GW = GWS + (KM ? 0 : buf * wbuf);
          if (m < nown) {
#pragma unroll 1
            for (int e = w * 4 + sub; e < NW2; e += 32) {
              const double2 r = RHO[m * NW2 + e];
#pragma unroll
              for (int a = 0; a < NJ; ++a) {
                double2 W = dzero;
#pragma unroll
                for (int q = 0; q < 4; ++q) W = fmac(wp[q], GW[(a * 4 + q) * NW2 + e], W);
                re[a] = fma(W.x, r.x, fma(W.y, r.y, re[a]));
                im[a] = fma(W.y, r.x, fma(-W.x, r.y, im[a]));
              }
            }
          }
          const int slot = (ti / kJRing) & 1, s = ti % kJRing;
          warp_store_current(re, im, NJ, lane, SJ + (((size_t)slot * kJRing + s) * KPC + w) * 2 * NJ);
        }
      }
      __syncthreads();
      flush(step1 - 1);
      for (int idx = tid; idx < nown * NW2; idx += NTHR) {
        const int m = idx / NW2, e = idx % NW2;
        rho[((size_t)(m10 + m) * t.N2 + m2) * NW2 + e] = RHO[idx];
      }
      __syncthreads();
    }
}

}  // namespace dfrag
