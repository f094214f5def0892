// Tensor-core form of the mixed-precision propagation for 9..16 orbitals (included by sbe_group.cu,
// inside its anonymous namespace: it uses GroupData, the precomputed inner sums of group_sums_kernel
// and the helpers defined there).
//
// Same propagation as group_vctas (k-space-resident RK4 of the reference's src/solver.cpp:86-181,
// 1428-1726, and the windowed current of src/observable.cpp:16-30), for solves whose cell box is the
// Hermitian-halved 7x7 one and whose inner Wannier sums come precomputed per column and step.
//
// Layout.  A CTA holds KPC consecutive k-points (rows m1) of one k-grid column, one warp per k-point.
// A k-point's nw x nw matrices are padded to 16 x 16 and spread over its warp in the accumulator
// layout of mma.m16n8k8: lane (g = lane/4, c = lane%4) holds rows g, g+8 and columns 2c, 2c+1,
// 8+2c, 9+2c, eight elements ("slots" s = 4 rb + 2 cb + e: row g + 8 rb, column 8 cb + 2c + e).
//
//  * Commutator on tensor cores.  For k-tile l the mma's A operand needs rows g, g+8 at two columns
//    of the k-tile per lane, and its B operand rows of the k-tile at column g of the n-tile; with the
//    k index of the tile permuted (physical k c <-> column 8l + 2c, c + 4 <-> 8l + 2c + 1), the A
//    fragment of H is exactly the lane's slots of H, and because X is Hermitian, B[k][n] = X[k][n] =
//    conj(X[n][k]) is the conjugate of the lane's slots of X.  So H X is formed from registers with no
//    data movement, as complex products split into TF32 halves (x = hi + lo, three mma per real
//    product: hi hi + hi lo + lo hi, which carries FP32 accuracy).  (H X)^+ comes from the same
//    registers by movmatrix transposes of the 8 x 8 blocks, so k = -i (H X - (H X)^+) stays in the
//    lane's slots, and so does the next stage's X = rho + c k.
//  * Outer Wannier sums on tensor cores.  H0(k) and r_a(k) of the CTA's k-points are one complex GEMM
//    per step, [k-points x 8] x [8 x nw^2]: A = the phases p1(k, n1) of the seven box rows (plus a
//    zero row), B = the inner sums G(n1) (G(-n1) = G(n1)^+ read transposed), split into TF32 halves
//    as above.  Its result goes through shared memory to the k-point warps.
//  * Window velocity and current in FP64, as in group_vctas, but in a dense layout: each thread takes
//    one k-point and a strided set of elements, so no lane idles on the padding; the state rho stays
//    in shared memory (FP64) where both layouts read it.
//
// Precision: the outer sums, the field coupling and the commutators are split-TF32 products; the
// stage sum k1 + 2 k2 + 2 k3 + k4 is formed in FP32 and added to the FP64 state rho; the window
// velocity sum and the current's k-sum are FP64.  The tensor cores round each mma's FP32 accumulation
// toward zero (measured on B200: 1 + 0.75 ulp accumulates to 1), so the products carry a one-sided
// error that the RK4 integration accumulates over the pulse: on the full pulse of the 11-orbital
// model on a 12 x 12 grid J drifts to 9.0e-6 of the reference (the FP32-pipe element-group kernel:
// 3.3e-7; the same kernel with FP32-pipe outer sums 6.4e-6, with an FP32-pipe product 2.8e-6).  With
// 128 registers per thread and the split and transpose instructions it also runs slower than the
// element-group kernel (C2: 499 vs 441 ms per solve).  It is therefore not chosen by default; set
// HHG_FRAG=1 to run it.

namespace frag {

__device__ __forceinline__ unsigned tf32_bits(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
// x = hi + lo, both TF32: hi is x rounded to TF32, lo the remainder rounded to TF32.
struct Split {
  unsigned h, l;
};
__device__ __forceinline__ Split split(float x) {
  const unsigned h = tf32_bits(x);
  return {h, tf32_bits(x - __uint_as_float(h))};
}
__device__ __forceinline__ Split negated(Split s) { return {s.h ^ 0x80000000u, s.l ^ 0x80000000u}; }

__device__ __forceinline__ void mma_tf32(float (&c)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                         unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
// c += a b for split operands (the small products first; lo lo is below FP32 rounding).
__device__ __forceinline__ void mma3(float (&c)[4], const Split (&a)[4], const Split (&b)[2]) {
  mma_tf32(c, a[0].h, a[1].h, a[2].h, a[3].h, b[0].l, b[1].l);
  mma_tf32(c, a[0].l, a[1].l, a[2].l, a[3].l, b[0].h, b[1].h);
  mma_tf32(c, a[0].h, a[1].h, a[2].h, a[3].h, b[0].h, b[1].h);
}

__device__ __forceinline__ unsigned movmatrix_trans(unsigned x) {
  unsigned r;
  asm volatile("movmatrix.sync.aligned.m8n8.trans.b16 %0, %1;" : "=r"(r) : "r"(x));
  return r;
}
// Transposes an 8 x 8 block of FP32 values held as (row g, columns 2c, 2c+1) pairs: the upper and
// lower 16-bit halves go through separate b16 transposes.
__device__ __forceinline__ void transpose8(float& a, float& b) {
  const unsigned ua = __float_as_uint(a), ub = __float_as_uint(b);
  const unsigned hi = movmatrix_trans(__byte_perm(ua, ub, 0x7632));
  const unsigned lo = movmatrix_trans(__byte_perm(ua, ub, 0x5410));
  a = __uint_as_float(__byte_perm(lo, hi, 0x5410));
  b = __uint_as_float(__byte_perm(lo, hi, 0x7632));
}

// Slot s of lane (g, c): row and column in the padded 16 x 16 matrix.
__device__ __forceinline__ int slot_row(int s, int g) { return g + 8 * (s >> 2); }
__device__ __forceinline__ int slot_col(int s, int c) { return 8 * ((s >> 1) & 1) + 2 * c + (s & 1); }

template <int NW, int NAX, int NJ, int KPC>
struct Geom {
  static constexpr int NW2 = NW * NW;
  static constexpr int NMAT = 1 + NAX;
  static constexpr int NBROWS = NMAT * 4;        // halved 7 x 7 box: inner-sum rows n1 = 0..3 per matrix
  static constexpr int NWROWS = NJ * 4;          // window rows
  static constexpr int NTILE = (NW2 + 7) / 8;    // n-tiles of one matrix in the outer sums
  static constexpr int HKS = (NW2 + 1) / 2 * 2;  // row stride of the outer-sum results (even: 16-byte pairs)
  static constexpr size_t RHO = 0;                                    // [KPC][NW2] double2
  static constexpr size_t HK = RHO + (size_t)KPC * NW2 * 16;          // [KPC][NMAT][HKS] float2
  static constexpr size_t GS = HK + (size_t)KPC * NMAT * HKS * 8;     // [2][NBROWS][NW2] float2
  static constexpr size_t GWS = GS + 2 * (size_t)NBROWS * NW2 * 8;    // [2][NWROWS][NW2] double2
  static constexpr size_t TW1 = GWS + 2 * (size_t)NWROWS * NW2 * 16;  // [KPC][8] float2
  static constexpr size_t WTW1 = TW1 + (size_t)KPC * 8 * 8;           // [KPC][4] double2
  static constexpr size_t SJ = WTW1 + (size_t)KPC * 4 * 16;           // [2][kJRing][KPC][2 NJ] double
  static constexpr size_t BYTES = SJ + 2 * (size_t)kJRing * KPC * 2 * NJ * 8;
  static_assert(NW > 8 && NW <= 16, "fragment layout: 9..16 orbitals");
  static_assert((NBROWS * NW2 * 8) % 16 == 0, "16-byte copies of the inner sums");
  static_assert(KPC == 8 || KPC == 16, "k-points per CTA");
};

template <int NW, int NAX, int NJ, int KPC>
__global__ void __launch_bounds__(KPC * 32, 16 / KPC)
    propagate_frag_kernel(SolveTables t, GroupData<float> d, int vctas, double2* rho, double2* Jpart) {
  using FG = Geom<NW, NAX, NJ, KPC>;
  constexpr int NW2 = FG::NW2, NMAT = FG::NMAT, NTILE = FG::NTILE, HKS = FG::HKS;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* RHO = reinterpret_cast<double2*>(smraw + FG::RHO);
  float2* HK = reinterpret_cast<float2*>(smraw + FG::HK);
  float2* GS = reinterpret_cast<float2*>(smraw + FG::GS);
  double2* GWS = reinterpret_cast<double2*>(smraw + FG::GWS);
  float2* TW1 = reinterpret_cast<float2*>(smraw + FG::TW1);
  double2* WTW1 = reinterpret_cast<double2*>(smraw + FG::WTW1);
  double* SJ = reinterpret_cast<double*>(smraw + FG::SJ);

  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, g = lane >> 2, c4 = lane & 3;
  constexpr int NTHR = KPC * 32;
  const int rows = t.row1 - t.row0, bpc = (rows + KPC - 1) / KPC, ntiles = t.N2 * bpc;
  const int step0 = t.step0, step1 = t.step1, npw = 2 * t.np + 1;
  const double dt = t.dt, prefac = 0.1666666666666 * dt;
  constexpr size_t gbuf = (size_t)FG::NBROWS * NW2, wbuf = (size_t)FG::NWROWS * NW2;
  const float2 fzero = make_float2(0.f, 0.f);

  for (int v = blockIdx.x; v < vctas; v += gridDim.x)
    for (int tile = v; tile < ntiles; tile += vctas) {
      const int m2 = tile / bpc, m10 = t.row0 + (tile % bpc) * KPC;
      const int nown = min(KPC, t.row1 - m10);  // k-points of this tile

      // Precomputed inner sums of point s (box rows into GS[s & 1], window rows into GWS[s & 1]).
      auto fetch = [&](int s) {
        const size_t blk = (size_t)(s - step0) * t.N2 + m2;
        const char* src = reinterpret_cast<const char*>(d.Gpre + blk * gbuf);
        char* dst = reinterpret_cast<char*>(GS + (s & 1) * gbuf);
        const double2* wsrc = d.GWpre + blk * wbuf;
        double2* wdst = GWS + (s & 1) * wbuf;
        constexpr int nA = (int)(gbuf * 8 / 16), nB = (int)wbuf;
        for (int idx = tid; idx < nA + nB; idx += NTHR) {
          if (idx < nA)
            cp_async16(dst + (size_t)idx * 16, src + (size_t)idx * 16);
          else
            cp_async16(wdst + (idx - nA), wsrc + (idx - nA));
        }
        cp_async_commit();
      };
      // Sums the ring half that ends at step ti_end over the warps (fixed order) into this virtual
      // CTA's row of current partials.
      auto flush = [&](int ti_end) {
        const int slot = (ti_end / kJRing) & 1, s = ti_end % kJRing;
        const int ti0 = max(ti_end - s, step0), nsteps = ti_end - ti0 + 1;  // a chunk may start inside a half
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

      // State in; twiddles of the box rows (FP32) and of the window rows (FP64).
      for (int idx = tid; idx < KPC * NW2; idx += NTHR) {
        const int m = idx / NW2, e = idx % NW2;
        RHO[idx] = m < nown ? rho[((size_t)(m10 + m) * t.N2 + m2) * NW2 + e] : make_double2(0.0, 0.0);
      }
      for (int idx = tid; idx < KPC * 8; idx += NTHR) {
        const int m = idx / 8, q = idx % 8, m1 = min(m10 + m, t.row1 - 1);
        TW1[idx] = q < 7 ? d.T1[wrap_mod((long long)m1 * (t.b1lo + q), t.N1)] : fzero;
      }
      for (int idx = tid; idx < KPC * 4; idx += NTHR) {
        const int m = idx / 4, q = idx % 4, m1 = min(m10 + m, t.row1 - 1);
        WTW1[idx] = d.T1d[wrap_mod((long long)m1 * (q - 2), t.N1)];
      }
      fetch(step0);
      cp_async_wait_all();
      __syncthreads();

      for (int ti = step0; ti < step1; ++ti) {
        const int buf = ti & 1;
        // (1) Outer sums of point ti: HK[m][mat][e] = sum_q p1(m, q) G(mat, n1 = q - 3)_e.
        {
          const float2* P1 = d.P + (size_t)ti * 2 * npw + t.np;
          Split ar[4], ai[4], nai[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) {  // a0 (g, c), a1 (g + 8, c), a2 (g, c + 4), a3 (g + 8, c + 4)
            const int m = g + 8 * (r & 1), q = c4 + 4 * (r >> 1);
            float2 p = fzero;
            if (m < KPC && q < 7) p = mul(TW1[m * 8 + q], P1[t.b1lo + q]);
            ar[r] = split(p.x);
            ai[r] = split(p.y);
            nai[r] = negated(ai[r]);
          }
          const float2* G = GS + buf * gbuf;
#pragma unroll 1
          for (int nt_ = w; nt_ < NMAT * NTILE; nt_ += KPC) {
            const int mat = nt_ / NTILE, j = nt_ % NTILE, e = 8 * j + g;
            // b0 = G(n1 = c - 3)_e: row 3 - c of the halved sums, transposed and conjugated for n1 < 0;
            // b1 = G(n1 = c + 1)_e (c + 4 = 7 is the zero row).
            float2 b0 = fzero, b1 = fzero;
            if (e < NW2) {
              const float2* Gm = G + (size_t)mat * 4 * NW2;
              if (c4 == 3) {
                b0 = Gm[e];
              } else {
                const float2 vv = Gm[(3 - c4) * NW2 + (e % NW) * NW + e / NW];
                b0 = make_float2(vv.x, -vv.y);
                b1 = Gm[(c4 + 1) * NW2 + e];
              }
            }
            const Split br[2] = {split(b0.x), split(b1.x)}, bi[2] = {split(b0.y), split(b1.y)};
            float cr[4] = {0.f, 0.f, 0.f, 0.f}, ci[4] = {0.f, 0.f, 0.f, 0.f};
            mma3(cr, ar, br);
            mma3(cr, nai, bi);
            mma3(ci, ar, bi);
            mma3(ci, ai, br);
            const int e0 = 8 * j + 2 * c4;  // results (g, e0), (g, e0 + 1), (g + 8, e0), (g + 8, e0 + 1)
            if (e0 < NW2) {
              if (g < KPC)
                *reinterpret_cast<float4*>(HK + ((size_t)g * NMAT + mat) * HKS + e0) =
                    make_float4(cr[0], ci[0], cr[1], ci[1]);
              if (g + 8 < KPC)
                *reinterpret_cast<float4*>(HK + ((size_t)(g + 8) * NMAT + mat) * HKS + e0) =
                    make_float4(cr[2], ci[2], cr[3], ci[3]);
            }
          }
        }
        __syncthreads();
        // A ring half completed by the previous step is flushed; the next point's sums are fetched
        // (their buffers were last read before this barrier).
        if (ti > step0 && (ti - 1) % kJRing == kJRing - 1) flush(ti - 1);
        if (ti + 1 < step1) fetch(ti + 1);

        // (2) RK4 stages of this warp's k-point (src/solver.cpp:157-180), fields at t, t+dt/2, t+dt/2, t+dt.
        if (w < nown) {
          const float2* Hm = HK + (size_t)w * NMAT * HKS;
          double2* Rm = RHO + (size_t)w * NW2;
          float2 r32[8], S[8], X[8];
#pragma unroll
          for (int s = 0; s < 8; ++s) {
            const int r = slot_row(s, g), cc = slot_col(s, c4);
            r32[s] = fzero;
            if (r < NW && cc < NW) {
              const double2 x = Rm[r * NW + cc];
              r32[s] = make_float2((float)x.x, (float)x.y);
            }
            S[s] = fzero;
            X[s] = r32[s];
          }
          const double* esb = t.es + (size_t)ti * 9;
#pragma unroll 1
          for (int st = 0; st < 4; ++st) {
            const int f = st == 0 ? 0 : (st == 3 ? 2 : 1);
            float ea[NAX];
#pragma unroll
            for (int a = 0; a < NAX; ++a) ea[a] = (float)esb[f * 3 + t.ax_id[a]];
            // H(k) at this stage's field, in the lane's slots (zero on the padding).
            float2 H[8];
#pragma unroll
            for (int s = 0; s < 8; ++s) {
              const int r = slot_row(s, g), cc = slot_col(s, c4);
              H[s] = fzero;
              if (r < NW && cc < NW) {
                const int el = r * NW + cc;
                H[s] = Hm[el];
#pragma unroll
                for (int a = 0; a < NAX; ++a) {
                  const float2 rv = Hm[(1 + a) * HKS + el];
                  H[s].x = fmaf(ea[a], rv.x, H[s].x);
                  H[s].y = fmaf(ea[a], rv.y, H[s].y);
                }
              }
            }
            // P = H X: Re P = Hr Xr + Hi Xi, Im P = Hr (-Xi) + Hi Xr over B = conj(X slots).
            float pr[2][4] = {}, pim[2][4] = {};
#pragma unroll
            for (int l = 0; l < 2; ++l) {
              Split hr[4], hi[4];
#pragma unroll
              for (int r = 0; r < 4; ++r) {
                const int sa = 2 * l + 4 * (r & 1) + (r >> 1);  // a0 (s 2l), a1 (4 + 2l), a2 (2l + 1), a3 (5 + 2l)
                hr[r] = split(H[sa].x);
                hi[r] = split(H[sa].y);
              }
#pragma unroll
              for (int j = 0; j < 2; ++j) {
                const int s0 = 4 * j + 2 * l, s1 = s0 + 1;
                const Split xr[2] = {split(X[s0].x), split(X[s1].x)};
                const Split xi[2] = {split(X[s0].y), split(X[s1].y)};
                const Split nxi[2] = {negated(xi[0]), negated(xi[1])};
                mma3(pr[j], hr, xr);
                mma3(pr[j], hi, xi);
                mma3(pim[j], hr, nxi);
                mma3(pim[j], hi, xr);
              }
            }
            // Slots of P, and of D = P^+ by 8 x 8 transposes (block (rb, cb) of P lands in block (cb, rb)).
            float Pr[8], Pi[8], Dr[8], Di[8];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
              Pr[2 * j] = pr[j][0];
              Pr[2 * j + 1] = pr[j][1];
              Pr[4 + 2 * j] = pr[j][2];
              Pr[5 + 2 * j] = pr[j][3];
              Pi[2 * j] = pim[j][0];
              Pi[2 * j + 1] = pim[j][1];
              Pi[4 + 2 * j] = pim[j][2];
              Pi[5 + 2 * j] = pim[j][3];
            }
#pragma unroll
            for (int rb = 0; rb < 2; ++rb)
#pragma unroll
              for (int cb = 0; cb < 2; ++cb) {
                float a0 = Pr[4 * rb + 2 * cb], a1 = Pr[4 * rb + 2 * cb + 1];
                float b0 = Pi[4 * rb + 2 * cb], b1 = Pi[4 * rb + 2 * cb + 1];
                transpose8(a0, a1);
                transpose8(b0, b1);
                Dr[4 * cb + 2 * rb] = a0;
                Dr[4 * cb + 2 * rb + 1] = a1;
                Di[4 * cb + 2 * rb] = -b0;
                Di[4 * cb + 2 * rb + 1] = -b1;
              }
            // k = -i (P - D); stage sum and the next stage's X = rho + c k.
            const float wgt = (st == 0 || st == 3) ? 1.f : 2.f;
            const float cn = (float)((st == 2 ? 1.0 : 0.5) * dt);
#pragma unroll
            for (int s = 0; s < 8; ++s) {
              const float kx = Pi[s] - Di[s], ky = -(Pr[s] - Dr[s]);
              S[s].x = fmaf(wgt, kx, S[s].x);
              S[s].y = fmaf(wgt, ky, S[s].y);
              X[s].x = fmaf(cn, kx, r32[s].x);
              X[s].y = fmaf(cn, ky, r32[s].y);
            }
          }
          // rho += dt/6 (k1 + 2 k2 + 2 k3 + k4) in FP64.
#pragma unroll
          for (int s = 0; s < 8; ++s) {
            const int r = slot_row(s, g), cc = slot_col(s, c4);
            if (r < NW && cc < NW) {
              double2 x = Rm[r * NW + cc];
              x.x = x.x + prefac * (double)S[s].x;
              x.y = x.y + prefac * (double)S[s].y;
              Rm[r * NW + cc] = x;
            }
          }
        }
        if (ti + 1 < step1) cp_async_wait_all();
        __syncthreads();

        // (3) Current partials of step ti (FP64): thread = k-point m, elements e = w EPP + sub + 32 p.
        {
          constexpr int EPP = 32 / KPC;
          const int m = lane % KPC, sub = lane / KPC;
          const double2* P1d = d.Pd + (size_t)ti * 2 * npw + t.np;
          double2 wp[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) wp[q] = mul(WTW1[m * 4 + q], P1d[q - 2]);
          double re[3] = {0.0, 0.0, 0.0}, im[3] = {0.0, 0.0, 0.0};
          const double2* GW = GWS + buf * wbuf;
          if (m < nown) {
#pragma unroll 1
            for (int e = w * EPP + sub; e < NW2; e += 32) {
              const double2 r = RHO[m * NW2 + e];
#pragma unroll
              for (int a = 0; a < NJ; ++a) {
                double2 W = make_double2(0.0, 0.0);
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

}  // namespace frag
