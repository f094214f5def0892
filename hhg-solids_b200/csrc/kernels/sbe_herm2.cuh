// One RK4 step (src/solver.cpp:157-180) of a k-point with two orbitals and Hermitian H, shared by the
// thread-per-k-point kernels.  The commutator of two Hermitian 2x2 matrices has a closed form: for
// k = -i [H, X],
//   k00 = 2 Im(H01 conj(X01)),   k11 = -k00,   k01 = -i ((H00 - H11) X01 - (X00 - X11) H01),
// the same k as -i (HX - (HX)^+) up to rounding; rho and every k stay Hermitian, so the state is
// rho00, rho11 (real) and rho01.
#pragma once
#include <cuda_runtime.h>

namespace hhg {

// r[4]: rho (row-major) in/out.  hd[2], hu[1], rd[a][2], ru[a][1]: diagonal and upper element of
// H0(k) and r_a(k) at the stage's evaluation point (box_at(f) refreshes them before stages 2 and 4
// when the k-space solver evaluates H at t + dt/2 and t + dt; a no-op otherwise).  es: the step's
// field samples [3 stages][3 axes]; ax_id: the nax field axes.
template <int NAXc, typename BoxAt>
__device__ __forceinline__ void herm2_rk4_step(double2 (&r)[4], const double (&hd)[2], const double2 (&hu)[4],
                                               const double (&rd)[3][2], const double2 (&ru)[3][4], int nax_rt,
                                               const int* ax_id, const double* es_step, double dt, double prefac,
                                               BoxAt&& box_at) {
  const int nax = NAXc ? NAXc : nax_rt;
  const double r00 = r[0].x, r11 = r[3].x;
  const double2 r01 = r[1];
  double k00 = 0.0, s00 = 0.0;
  double2 k01 = make_double2(0.0, 0.0), s01 = make_double2(0.0, 0.0);
#pragma unroll
  for (int st = 0; st < 4; ++st) {
    const int f = st == 0 ? 0 : (st == 3 ? 2 : 1);
    const double* es = es_step + f * 3;
    if (st == 1 || st == 3) box_at(f);
    double h00 = hd[0], h11 = hd[1];
    double2 h01 = hu[1];
#pragma unroll
    for (int a = 0; a < 3; ++a)
      if (a < nax) {
        const double ea = es[ax_id[a]];
        h00 = fma(ea, rd[a][0], h00);
        h11 = fma(ea, rd[a][1], h11);
        h01.x = fma(ea, ru[a][1].x, h01.x);
        h01.y = fma(ea, ru[a][1].y, h01.y);
      }
    const double cs = (st == 3 ? 1.0 : 0.5) * dt;
    const double x00 = st == 0 ? r00 : fma(cs, k00, r00);
    const double x11 = st == 0 ? r11 : fma(-cs, k00, r11);
    const double2 x01 = st == 0 ? r01 : make_double2(fma(cs, k01.x, r01.x), fma(cs, k01.y, r01.y));
    k00 = 2.0 * fma(h01.y, x01.x, -h01.x * x01.y);
    const double dh = h00 - h11, dx = x00 - x11;
    const double tx = fma(dh, x01.x, -dx * h01.x), ty = fma(dh, x01.y, -dx * h01.y);
    k01 = make_double2(ty, -tx);
    if (st == 0) {
      s00 = k00;
      s01 = k01;
    } else {
      const double wgt = st == 3 ? 1.0 : 2.0;
      s00 = fma(wgt, k00, s00);
      s01 = make_double2(fma(wgt, k01.x, s01.x), fma(wgt, k01.y, s01.y));
    }
  }
  const double n00 = fma(prefac, s00, r00), n11 = fma(-prefac, s00, r11);
  const double2 n01 = make_double2(fma(prefac, s01.x, r01.x), fma(prefac, s01.y, r01.y));
  r[0] = make_double2(n00, 0.0);
  r[1] = n01;
  r[2] = make_double2(n01.x, -n01.y);
  r[3] = make_double2(n11, 0.0);
}

}  // namespace hhg
