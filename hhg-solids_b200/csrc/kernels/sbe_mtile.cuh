// Mixed-form propagation for 9..12 orbitals with half a warp per k-point and 3 x 3 register tiles
// (included by sbe_group.cu, inside its anonymous namespace: it uses GroupData, the precomputed inner
// sums of group_sums_kernel and the helpers defined there).
//
// Same propagation as group_vctas in its mixed form (k-space-resident RK4 of the reference's
// src/solver.cpp:86-181, 1428-1726, and the windowed current of src/observable.cpp:16-30), for solves
// whose cell box is the Hermitian-halved 7x7 one and whose inner Wannier sums come precomputed per
// column and step (real-space solver).
//
// Layout.  A CTA holds KPC consecutive k-points (rows m1) of one k-grid column; the k-point's matrices
// are padded to a 12 x 12 frame (9..12 orbitals: 16 lanes, half a warp, per k-point, 8 per CTA) or a
// 6 x 6 one (4..6 orbitals: 4 lanes per k-point, 32 per CTA), lane s owning its 3 x 3 tile (rows
// 3 (s / T) .. +2, columns 3 (s % T) .. +2, T tiles per frame row).  Each lane keeps its tile of the state rho and of the RK4
// sum in FP64 registers; the outer Wannier sums H0(k), r_a(k) of its tile give H = H0 + E.r at the
// step's field samples, the later ones kept in FP32 registers for their stages.
// Per stage:
//  * H = H0 + E.r of the tile goes to shared memory, transposed (H(i, j) at [j][i]), X = rho + c k
//    (FP32) is already there;
//  * the lane forms its tile of P = H X in FP32 from rows l of both arrays (three H and three X
//    values per l: 36 FMA per 6 loads, every load a broadcast to the lanes of its tile row or
//    column);
//  * P replaces X in shared memory, and k = -i (P - P^+) takes P^+ from the transposed tile;
//  * the RK4 sum and the next stage's X are formed in FP64 (X stored as FP32).
// Only the k-point's lanes (within one warp) exchange data, so the stages need __syncwarp only; the CTA meets twice
// per step for the current (its FP64 window rows copied in during the step, then the FP64 state staged
// for it) and once at its end (the next step's inner sums, copied in with cp.async meanwhile, and the
// current partials).  The current is FP64: summed over the CTA's k-points on the FP64 tensor cores, then
// contracted with the window rows.
//
// Precision: as the element-group kernel's mixed form (complex-FP32 Wannier sums and commutator
// products, FP64 state, RK4 accumulation, window velocity and k-sum).

namespace mtile {

// Waits until at most one committed group of this thread's cp.async copies is still in flight.
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

template <int NW, int NAX, int NJ, int KPC, bool KM = false>
struct Geom {
  static constexpr int NW2 = NW * NW;
  static constexpr int NMAT = 1 + NAX;
  static constexpr int NBROWS = NMAT * 4;   // halved 7 x 7 box: inner-sum rows n1 = 0..3 per matrix
  static constexpr int NWROWS = NJ * 4;     // window rows
  // The frame: 12 x 12 (9..12 orbitals) or 6 x 6 (4..6), in 3 x 3 tiles, one lane per tile; a CTA of
  // 128 threads holds KPC = 128 / (lanes per k-point) k-points (8 or 32).
  static constexpr int NWP = NW > 6 ? 12 : 6;
  static constexpr int TD = NWP / 3;        // tiles per frame row
  static constexpr int LPK = TD * TD;       // lanes per k-point
  static constexpr int NWARP = KPC * LPK / 32;
  // Inner-sum slots: this step's point and the next one's (real-space solver); the k-space solver's
  // points t + dt/2 and t + dt of this step and of the next, in a ring of four (point p in (p + 3) % 4).
  static constexpr int NGS = KM ? 4 : 2;
  static constexpr int NTHR = KPC * LPK;
  static constexpr int MS = NWP;            // row stride (float2) of a padded matrix
  static constexpr int KS = NWP * NWP + 1;  // float2 per k-point matrix: the odd 8-byte unit puts a
                                            // warp's k-points in different banks
  static constexpr size_t HS = 0;                                     // [KPC][KS] float2: H, transposed
  static constexpr size_t XP = HS + (size_t)KPC * KS * 8;             // [KPC][KS] float2: X, then P
  static constexpr size_t GS = (XP + (size_t)KPC * KS * 8 + 15) / 16 * 16;  // [NGS][NBROWS][NW2] float2
  static constexpr size_t GWS = GS + NGS * (size_t)NBROWS * NW2 * 8;  // [NWROWS][NW2] double2: one step's
                                                                      // (k-space solver: the column's)
  static constexpr size_t TW1 = GWS + (size_t)NWROWS * NW2 * 16;      // [KPC][8] float2: box rows q = 0..6
  static constexpr size_t WTW1 = TW1 + (size_t)KPC * 8 * 8;           // [KPC][4] double2: window rows
  static constexpr size_t SJ = WTW1 + (size_t)KPC * 4 * 16;           // [2][kJRing][NWARP][2 NJ] double
  static constexpr size_t BYTES = SJ + 2 * (size_t)kJRing * NWARP * 2 * NJ * 8;
  static_assert((NW > 8 && NW <= 12) || (NW >= 4 && NW <= 6), "3 x 3 tiles of a 12 x 12 or 6 x 6 frame");
  static_assert(KPC * LPK == 128, "128 threads per CTA");
  static_assert((NBROWS * NW2 * 8) % 16 == 0, "16-byte copies of the inner sums");
  static_assert((size_t)KPC * NW2 * 16 <= 2 * (size_t)KPC * KS * 8, "the FP64 state fits over the H and X area");
  static_assert(KPC % 4 == 0, "the current's product takes the CTA's k-points as its K dimension (k-steps of 4)");
};

// 128 threads per CTA run three CTAs per SM (at most 168 registers per thread): 12 warps per SM, against
// 8 for 16 k-points of 11 orbitals per CTA at 218 registers (C2: 324 against 416 ms per solve).
// KM: the reference's k-space solver (src/solver_kspace.cpp:167-270): the stages see H at points
// 2 ti (t), 2 ti + 1 (t + dt/2) and 2 ti + 2 (t + dt) of the interpolation tables; the outer sums of
// 2 ti + 2 stay in registers for the next step's first stage, and the window has no phase.
template <int NW, int NAX, int NJ, int KPC, bool KM = false>
__global__ void __launch_bounds__(128, 3)
    propagate_mtile_kernel(SolveTables t, GroupData<float> d, int vctas, double2* rho, double2* Jpart) {
  using FG = Geom<NW, NAX, NJ, KPC, KM>;
  constexpr int NW2 = FG::NW2, NMAT = FG::NMAT, NWARP = FG::NWARP, NTHR = FG::NTHR, MS = FG::MS, KS = FG::KS;
  extern __shared__ __align__(16) unsigned char smraw[];
  float2* HS = reinterpret_cast<float2*>(smraw + FG::HS);
  float2* XPb = reinterpret_cast<float2*>(smraw + FG::XP);
  float2* GS = reinterpret_cast<float2*>(smraw + FG::GS);
  double2* GWS = reinterpret_cast<double2*>(smraw + FG::GWS);
  float2* TW1 = reinterpret_cast<float2*>(smraw + FG::TW1);
  double2* WTW1 = reinterpret_cast<double2*>(smraw + FG::WTW1);
  double* SJ = reinterpret_cast<double*>(smraw + FG::SJ);

  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int kp = tid / FG::LPK, sub = tid % FG::LPK, i0 = 3 * (sub / FG::TD), j0 = 3 * (sub % FG::TD);
  const int rows = t.row1 - t.row0, bpc = (rows + KPC - 1) / KPC, ntiles = t.N2 * bpc;
  const int step0 = t.step0, step1 = t.step1, npw = 2 * t.np + 1;
  const double dt = t.dt, prefac = 0.1666666666666 * dt;
  constexpr size_t gbuf = (size_t)FG::NBROWS * NW2, wbuf = (size_t)FG::NWROWS * NW2;
  float2* Hk = HS + kp * KS;
  float2* Xk = XPb + kp * KS;
  const float2 fzero = make_float2(0.f, 0.f);
  const double2 dzero = make_double2(0.0, 0.0);
  // Tile slot u = 3 a + b is element (i0 + a, j0 + b); on the padding (row or column >= NW) it stays 0.
  auto valid = [&](int u) { return i0 + u / 3 < NW && j0 + u % 3 < NW; };
  auto own = [&](int u) { return (i0 + u / 3) * MS + j0 + u % 3; };   // (i, j) in X, P
  auto tra = [&](int u) { return (j0 + u % 3) * MS + i0 + u / 3; };   // (j, i): H, P^+

  for (int v = blockIdx.x; v < vctas; v += gridDim.x)
    for (int tile = v; tile < ntiles; tile += vctas) {
      const int m2 = tile / bpc, m10 = t.row0 + (tile % bpc) * KPC;
      const int nown = min(KPC, t.row1 - m10);
      const bool kval = kp < nown;

      // Inner sums of point p into slot `slot`, and window rows of point p (16-byte asynchronous copies).
      auto fetch_sums = [&](int p, int slot) {
        const size_t blk = (size_t)(p - (KM ? 2 * step0 : step0)) * t.N2 + m2;
        const char* src = reinterpret_cast<const char*>(d.Gpre + blk * gbuf);
        char* dst = reinterpret_cast<char*>(GS + (size_t)slot * gbuf);
        constexpr int nA = (int)(gbuf * 8 / 16);
        for (int idx = tid; idx < nA; idx += NTHR) cp_async16(dst + (size_t)idx * 16, src + (size_t)idx * 16);
      };
      auto fetch_window = [&](int p) {
        const double2* wsrc = d.GWpre + ((KM ? 0 : (size_t)(p - step0) * t.N2) + m2) * wbuf;
        for (int idx = tid; idx < (int)wbuf; idx += NTHR) cp_async16(GWS + idx, wsrc + idx);
      };
      // The warps' current partials of the ring half ending at step ti_end, into this virtual CTA's row.
      auto flush = [&](int ti_end) {
        const int slot = (ti_end / kJRing) & 1, s = ti_end % kJRing;
        const int ti0 = max(ti_end - s, step0), nsteps = ti_end - ti0 + 1;
        const double* half = SJ + ((size_t)slot * kJRing + (ti0 % kJRing)) * NWARP * 2 * NJ;
        for (int idx = tid; idx < nsteps * NJ; idx += NTHR) {
          const int ss = idx / NJ, a = idx % NJ;
          double re = 0.0, im = 0.0;
          for (int ww = 0; ww < NWARP; ++ww) {
            re += half[(ss * NWARP + ww) * 2 * NJ + 2 * a];
            im += half[(ss * NWARP + ww) * 2 * NJ + 2 * a + 1];
          }
          const int ja = a == 0 ? t.j_id[0] : (a == 1 ? t.j_id[1] : t.j_id[2]);
          double2* dst = Jpart + ((size_t)v * t.nt + ti0 + ss) * 3 + ja;
          const double2 old = *dst;
          *dst = make_double2(old.x + re, old.y + im);
        }
      };

      for (int idx = tid; idx < KPC * 8; idx += NTHR) {
        const int m = idx / 8, q = idx % 8, m1 = min(m10 + m, t.row1 - 1);
        TW1[idx] = q < 7 ? d.T1[wrap_mod((long long)m1 * (t.b1lo + q), t.N1)] : fzero;
      }
      for (int idx = tid; idx < KPC * 4; idx += NTHR) {
        const int m = idx / 4, q = idx % 4, m1 = min(m10 + m, t.row1 - 1);
        WTW1[idx] = d.T1d[wrap_mod((long long)m1 * (q - 2), t.N1)];
      }
      // Outer sums of the tile's elements at point p from GS slot `slot`: for matrix mat (H0, then r_a),
      // sum_{q=0..6} p1(k, q) G'(q)_e with G'(q) = G(n1 = q - 3) for q >= 3 and G(3 - q)^+ below;
      // take(u, m) receives element u's NMAT sums.
      auto outer = [&](int p, int slot, auto&& take) {
        const float2* P1 = d.P + (size_t)p * 2 * npw + t.np;
        float2 p1[7];
#pragma unroll
        for (int q = 0; q < 7; ++q) p1[q] = mul(TW1[kp * 8 + q], P1[t.b1lo + q]);
        const float2* G = GS + (size_t)slot * gbuf;
#pragma unroll
        for (int u = 0; u < 9; ++u) {
          float2 m[NMAT];
#pragma unroll
          for (int mat = 0; mat < NMAT; ++mat) {
            float2 acc = fzero;
            if (valid(u)) {
              const int i = i0 + u / 3, j = j0 + u % 3, e = i * NW + j, eT = j * NW + i;
              const float2* Gm = G + (size_t)mat * 4 * NW2;
              acc = mul(p1[3], Gm[e]);
#pragma unroll
              for (int n = 1; n < 4; ++n) {
                acc = fmac(p1[3 + n], Gm[n * NW2 + e], acc);
                acc = fmac(p1[3 - n], conjugate(Gm[n * NW2 + eT]), acc);
              }
            }
            m[mat] = acc;
          }
          take(u, m);
        }
      };
      // The field samples of step ts (t, t + dt/2, t + dt) on the active axes, and H = H0 + E.r.
      auto fields = [&](int ts, float (&ea)[3][NAX]) {
        const double* es = t.es + (size_t)ts * 9;
#pragma unroll
        for (int f = 0; f < 3; ++f)
#pragma unroll
          for (int a = 0; a < NAX; ++a) ea[f][a] = (float)es[f * 3 + t.ax_id[a]];
      };
      auto field_h = [&](const float2 (&m)[NMAT], const float (&e)[NAX]) {
        float2 h = m[0];
#pragma unroll
        for (int a = 0; a < NAX; ++a) {
          h.x = fmaf(e[a], m[1 + a].x, h.x);
          h.y = fmaf(e[a], m[1 + a].y, h.y);
        }
        return h;
      };
      // H of the tile at the step's later stages (registers): real-space solver, at t + dt/2 and t + dt
      // (H at t goes to shared memory as the sums are formed); k-space solver, the next step's H at t.
      float2 Hn[KM ? 1 : 2][9];
      auto gslot = [&](int p) { return KM ? (p + 3) & 3 : p & 1; };

      if constexpr (KM) {
        fetch_sums(2 * step0, gslot(2 * step0));
        fetch_window(0);  // the column's window rows, the same for every step
      } else {
        fetch_sums(step0, gslot(step0));
      }
      cp_async_commit();
      // This lane's tile of the state (FP64 registers for the whole tile).
      const size_t kg = ((size_t)(m10 + (kval ? kp : 0)) * t.N2 + m2) * NW2;
      double2 r[9];
#pragma unroll
      for (int u = 0; u < 9; ++u) r[u] = (kval && valid(u)) ? rho[kg + (i0 + u / 3) * NW + j0 + u % 3] : dzero;
      cp_async_wait_all();
      __syncthreads();
      if constexpr (KM) {
        // The chunk's first point t (then carried from step to step), and the first step's other two.
        {
          float ea[3][NAX];
          fields(step0, ea);
          outer(2 * step0, gslot(2 * step0), [&](int u, const float2 (&m)[NMAT]) { Hn[0][u] = field_h(m, ea[0]); });
        }
        fetch_sums(2 * step0 + 1, gslot(2 * step0 + 1));
        fetch_sums(2 * step0 + 2, gslot(2 * step0 + 2));
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
      }

      for (int ti = step0; ti < step1; ++ti) {
        const int buf = ti & 1;
        if (ti > step0 && (ti - 1) % kJRing == kJRing - 1) flush(ti - 1);
        if constexpr (KM) {
          // The next step's points t + dt/2 and t + dt, into the slots of this step's t and of the
          // previous step's t + dt/2, whose last readers finished before the barrier that ended it.
          if (ti + 1 < step1) {
            fetch_sums(2 * ti + 3, gslot(2 * ti + 3));
            fetch_sums(2 * ti + 4, gslot(2 * ti + 4));
          }
          cp_async_commit();
        } else {
          // This step's window rows (read by the current at its end), then the next step's inner sums
          // into the other slot: both buffers' last readers finished before the barrier that ended the
          // previous step.  Two groups, so that the current can wait for the first alone.
          fetch_window(ti);
          cp_async_commit();
          if (ti + 1 < step1) fetch_sums(ti + 1, gslot(ti + 1));
          cp_async_commit();
          // (1) Outer sums at the step's point: H at t into shared memory (the area's last readers, the
          //     previous step's current, finished before the barrier), at t + dt/2 and t + dt kept.
          float ea[3][NAX];
          fields(ti, ea);
          outer(ti, buf, [&](int u, const float2 (&m)[NMAT]) {
            Hk[tra(u)] = field_h(m, ea[0]);
            Hn[0][u] = field_h(m, ea[1]);
            Hn[1][u] = field_h(m, ea[2]);
          });
        }
        // (2) RK4 stages (src/solver.cpp:157-180), fields at t, t+dt/2, t+dt/2, t+dt; X = rho for the first
        //     (the area held the previous step's FP64 state for the current).
#pragma unroll
        for (int u = 0; u < 9; ++u) Xk[own(u)] = make_float2((float)r[u].x, (float)r[u].y);
        double2 S[9];
#pragma unroll 1
        for (int st = 0; st < 4; ++st) {
          // H of the stage (the third keeps the second's: same field and point).
          if constexpr (KM) {
            float ea[3][NAX];
            fields(ti, ea);
            if (st == 0) {
#pragma unroll
              for (int u = 0; u < 9; ++u) Hk[tra(u)] = Hn[0][u];
            } else if (st == 1) {
              outer(2 * ti + 1, gslot(2 * ti + 1), [&](int u, const float2 (&m)[NMAT]) { Hk[tra(u)] = field_h(m, ea[1]); });
            } else if (st == 3) {
              // the point t + dt: this stage's H, and the next step's H at t (its first field sample)
              float en[3][NAX];
              fields(ti + 1 < step1 ? ti + 1 : ti, en);
              outer(2 * ti + 2, gslot(2 * ti + 2), [&](int u, const float2 (&m)[NMAT]) {
                Hk[tra(u)] = field_h(m, ea[2]);
                Hn[0][u] = field_h(m, en[0]);
              });
            }
          } else {
            if (st == 1) {
#pragma unroll
              for (int u = 0; u < 9; ++u) Hk[tra(u)] = Hn[0][u];
            } else if (st == 3) {
#pragma unroll
              for (int u = 0; u < 9; ++u) Hk[tra(u)] = Hn[1][u];
            }
          }
          __syncwarp();
          // P = H X on the tile: P(i, j) = sum_l H(i, l) X(l, j), H(i, l) from row l of the transposed H.
          float2 P[9];
#pragma unroll
          for (int u = 0; u < 9; ++u) P[u] = fzero;
#pragma unroll
          for (int l = 0; l < NW; ++l) {
            const float2* hr = Hk + l * MS + i0;
            const float2* xr = Xk + l * MS + j0;
            const float2 h0 = hr[0], h1 = hr[1], h2 = hr[2], x0 = xr[0], x1 = xr[1], x2 = xr[2];
            P[0] = fmac(h0, x0, P[0]);
            P[1] = fmac(h0, x1, P[1]);
            P[2] = fmac(h0, x2, P[2]);
            P[3] = fmac(h1, x0, P[3]);
            P[4] = fmac(h1, x1, P[4]);
            P[5] = fmac(h1, x2, P[5]);
            P[6] = fmac(h2, x0, P[6]);
            P[7] = fmac(h2, x1, P[7]);
            P[8] = fmac(h2, x2, P[8]);
          }
          __syncwarp();  // every lane of the k-point has read X
#pragma unroll
          for (int u = 0; u < 9; ++u) Xk[own(u)] = P[u];
          __syncwarp();
          const double wgt = (st == 0 || st == 3) ? 1.0 : 2.0;
          const double cn = (st == 2 ? 1.0 : 0.5) * dt;
          float2 xn[9];
#pragma unroll
          for (int u = 0; u < 9; ++u) {
            const float2 pt = Xk[tra(u)];
            const float kx = P[u].y + pt.y, ky = -(P[u].x - pt.x);  // k = -i (P - P^+)
            if (st == 0) {
              S[u] = make_double2((double)kx, (double)ky);
            } else {
              S[u].x += wgt * (double)kx;
              S[u].y += wgt * (double)ky;
            }
            xn[u] = make_float2((float)(r[u].x + cn * (double)kx), (float)(r[u].y + cn * (double)ky));
          }
          __syncwarp();  // every lane of the k-point has read P
          if (st < 3) {
#pragma unroll
            for (int u = 0; u < 9; ++u) Xk[own(u)] = xn[u];
          }
        }
        // rho += dt/6 (k1 + 2 k2 + 2 k3 + k4) (src/solver.cpp:170-180).
#pragma unroll
        for (int u = 0; u < 9; ++u) {
          r[u].x = r[u].x + prefac * S[u].x;
          r[u].y = r[u].y + prefac * S[u].y;
        }

        // (3) Current partials of step ti (FP64), summed over the CTA's k-points before the window:
        //     J_a = sum_{q,e} GW(a, q)_e R(q, e) with R(q, e) = sum_k wp(k, q) conj(rho_e(k)), the same sum
        //     as sum_k sum_e W_a(k)_e conj(rho_e(k)), W_a(k)_e = sum_q wp(k, q) GW(a, q)_e, in another order.
        //     R is a [4 window rows (of 8)] x [8 k-points] x [nw^2 elements] product on the FP64 tensor
        //     cores (three real m8n8k4 products per complex one) from the state staged in FP64 over the H
        //     and X area, which every k-point's stages have finished with at the barrier.
        if constexpr (!KM) cp_async_wait_one();  // this step's window rows
        __syncthreads();
        double2* RS = reinterpret_cast<double2*>(HS);  // [KPC][NW2] double2
        if (kval) {
#pragma unroll
          for (int u = 0; u < 9; ++u)
            if (valid(u)) RS[kp * NW2 + (i0 + u / 3) * NW + j0 + u % 3] = r[u];
        } else {
#pragma unroll
          for (int u = 0; u < 9; ++u)
            if (valid(u)) RS[kp * NW2 + (i0 + u / 3) * NW + j0 + u % 3] = dzero;
        }
        __syncthreads();
        {
          const int g = lane >> 2, c4 = lane & 3;
          const double2* P1d = d.Pd + (size_t)ti * 2 * npw + t.np;
          // A[g][c] of k-step ks: wp(k-point 4 ks + c, window row g), rows 4..7 zero.
          constexpr int NKS = KPC / 4;
          double2 wa[NKS];
#pragma unroll
          for (int ks = 0; ks < NKS; ++ks)
            wa[ks] = g < 4 ? (KM ? WTW1[(4 * ks + c4) * 4 + g] : mul(WTW1[(4 * ks + c4) * 4 + g], P1d[g - 2])) : dzero;
          double re[3] = {0.0, 0.0, 0.0}, im[3] = {0.0, 0.0, 0.0};
          constexpr int NTR = (NW2 + 7) / 8;
#pragma unroll 1
          for (int nt = w; nt < NTR; nt += NWARP) {
            double t1[2] = {0.0, 0.0}, t2[2] = {0.0, 0.0}, t3[2] = {0.0, 0.0};
            const int eb = 8 * nt + g;  // B[c][g]: conj(rho_eb(k-point 4 ks + c))
#pragma unroll
            for (int ks = 0; ks < NKS; ++ks) {
              const double2 b = eb < NW2 ? RS[(4 * ks + c4) * NW2 + eb] : dzero;
              dfrag::dmma(t1, wa[ks].x, b.x);
              dfrag::dmma(t2, wa[ks].y, -b.y);
              dfrag::dmma(t3, wa[ks].x + wa[ks].y, b.x - b.y);
            }
            if (g < 4) {
#pragma unroll
              for (int jj = 0; jj < 2; ++jj) {
                const int e = 8 * nt + 2 * c4 + jj;  // R(g, e)
                if (e < NW2) {
                  const double rr = t1[jj] - t2[jj], ri = t3[jj] - t1[jj] - t2[jj];
#pragma unroll
                  for (int a = 0; a < NJ; ++a) {
                    const double2 gw = GWS[(a * 4 + g) * NW2 + e];
                    re[a] = fma(gw.x, rr, fma(-gw.y, ri, re[a]));
                    im[a] = fma(gw.x, ri, fma(gw.y, rr, im[a]));
                  }
                }
              }
            }
          }
          const int slot = (ti / kJRing) & 1, s = ti % kJRing;
          warp_store_current(re, im, NJ, lane, SJ + (((size_t)slot * kJRing + s) * NWARP + w) * 2 * NJ);
        }
        cp_async_wait_all();
        __syncthreads();
      }
      flush(step1 - 1);
      if (kval) {
#pragma unroll
        for (int u = 0; u < 9; ++u)
          if (valid(u)) rho[kg + (i0 + u / 3) * NW + j0 + u % 3] = r[u];
      }
      __syncthreads();
    }
}

}  // namespace mtile
