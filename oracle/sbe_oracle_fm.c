/* Host arithmetic whose exact rounding decides the result -- TEST INFRASTRUCTURE ONLY.
 *
 * Compiled with the reference's own flags (-O3 -ffast-math plus the same ISA level, see Makefile),
 * because three reference formulas have outputs that depend on the last bit of their inputs:
 *  - the Cramer solve of src/vec3_util.cpp:13-36, whose (int) truncation (src/hamiltonian.cpp:19-23)
 *    decides on which grid cell a hopping lands (coefficients like 1.9999999999999998 truncate to 1);
 *  - the supercell positions of src/grid.cpp:81-110 that feed it;
 *  - the field of src/efield.cpp:30-50, which rounds its arguments to float for sinf/sqrtf.
 * The expressions below keep the reference's operand order so that the compiler contracts and
 * folds them the same way; the tests check the results bit for bit against the reference build. */
#include <math.h>

/* src/vec3_util.cpp:13-36: coefficients c with c0 a0 + c1 a1 + c2 a2 = v by Cramer's rule, where
 * m[i] is lattice vector a_i.  The x numerator reads m[2][1] where m[2][0] belongs (kept: it only
 * matters when a3 has an in-plane component). */
__attribute__((noinline)) void oracle_cramer3(double** m, double* v, double* c) {
  double m00 = m[1][1] * m[2][2] - m[2][1] * m[1][2];
  double m01 = m[0][1] * m[2][2] - m[2][1] * m[0][2];
  double m02 = m[0][1] * m[1][2] - m[1][1] * m[0][2];
  double det = m[0][0] * m00 - m[1][0] * m01 + m[2][0] * m02;
  double nx = v[0] * m00 - m[1][0] * (v[1] * m[2][2] - m[2][1] * v[2]) + m[2][1] * (v[1] * m[1][2] - m[1][1] * v[2]);
  double ny = m[0][0] * (v[1] * m[2][2] - m[2][1] * v[2]) - v[0] * m01 + m[2][0] * (m[0][1] * v[2] - v[1] * m[0][2]);
  double nz = m[0][0] * (m[1][1] * v[2] - v[1] * m[1][2]) - m[1][0] * (m[0][1] * v[2] - v[1] * m[0][2]) + v[0] * m02;
  double inv = 1.0 / det;
  c[0] = nx * inv;
  c[1] = ny * inv;
  c[2] = nz * inv;
}

/* src/grid.cpp:64-111: centred cells n_i = -N_i/2 + i, positions R = n1 a1 + n2 a2 + n3 a3 (Angstrom),
 * k = m1/N1 b1 + m2/N2 b2 + m3/N3 b3; flattened index i*N2*N3 + j*N3 + k. */
__attribute__((noinline)) void oracle_supercell(int N1, int N2, int N3, double a[3][3], double b[3][3],
                                                double* R, double* K) {
  for (int i = 0; i < N1; ++i)
    for (int j = 0; j < N2; ++j)
      for (int k = 0; k < N3; ++k) {
        int n1 = -N1 / 2 + i, n2 = -N2 / 2 + j, n3 = -N3 / 2 + k;
        long idx = (long)i * N2 * N3 + (long)j * N3 + k;
        R[3 * idx + 0] = n1 * a[0][0] + n2 * a[1][0] + n3 * a[2][0];
        R[3 * idx + 1] = n1 * a[0][1] + n2 * a[1][1] + n3 * a[2][1];
        R[3 * idx + 2] = n1 * a[0][2] + n2 * a[1][2] + n3 * a[2][2];
        K[3 * idx + 0] = (double)i / (double)N1 * b[0][0] + (double)j / (double)N2 * b[1][0] + (double)k / (double)N3 * b[2][0];
        K[3 * idx + 1] = (double)i / (double)N1 * b[0][1] + (double)j / (double)N2 * b[1][1] + (double)k / (double)N3 * b[2][1];
        K[3 * idx + 2] = (double)i / (double)N1 * b[0][2] + (double)j / (double)N2 * b[1][2] + (double)k / (double)N3 * b[2][2];
      }
}

/* src/grid.cpp:27-46: b_i = 2 pi / V (a_j x a_k). */
__attribute__((noinline)) void oracle_reciprocal(double a[3][3], double b[3][3]) {
  double t[3];
  t[0] = a[1][1] * a[2][2] - a[1][2] * a[2][1];
  t[1] = -a[1][0] * a[2][2] + a[1][2] * a[2][0];
  t[2] = a[1][0] * a[2][1] - a[1][1] * a[2][0];
  double V = a[0][0] * t[0] + a[0][1] * t[1] + a[0][2] * t[2];
  for (int r = 0; r < 3; ++r) {
    int p = (r + 1) % 3, q = (r + 2) % 3;
    t[0] = a[p][1] * a[q][2] - a[p][2] * a[q][1];
    t[1] = -a[p][0] * a[q][2] + a[p][2] * a[q][0];
    t[2] = a[p][0] * a[q][1] - a[p][1] * a[q][0];
    b[r][0] = 2.0 * M_PI / V * t[0];
    b[r][1] = 2.0 * M_PI / V * t[1];
    b[r][2] = 2.0 * M_PI / V * t[2];
  }
}

/* src/grid.cpp:65-67,133-135: t_i = i dt (fs), then converted to au by x (1.0/0.02418884). */
__attribute__((noinline)) void oracle_time_grid(int nt, double dt_fs, double* t) {
  for (int i = 0; i < nt; ++i) t[i] = (double)i * dt_fs;
  for (int i = 0; i < nt; ++i) t[i] *= 1.0 / 0.02418884;
}

static double oracle_env(double ti, double tf) {
  if (ti < tf) return pow(sin(M_PI * ti / tf), 2);
  return 0.0;
}

/* src/efield.cpp:10-11,30-50,72-74 (after the au conversion of src/efield.cpp:66-79). */
__attribute__((noinline)) void oracle_efield(int nt, const double* t, double lambda_nm, double tmax_field_fs,
                                             double intensity, const double* s, const double* phi, double* E,
                                             double* A) {
  double lambda = lambda_nm * 10.0;
  double omega = 2.0 * M_PI * 2997.025 / lambda;
  double tf = tmax_field_fs;
  tf *= 1.0 / 0.02418884;
  omega *= 1.0 / (1.0 / 0.02418884);
  double peak = sqrtf(intensity * 1.0 / 3.56e16);
  double dt = t[1] - t[0];
  double *Ex = E, *Ey = E + nt, *Ez = E + 2 * nt, *Ax = A, *Ay = A + nt, *Az = A + 2 * nt;
  for (int i = 0; i < nt; ++i) {
    Ex[i] = s[0] * peak * oracle_env(t[i], tf) * sinf(omega * t[i] + phi[0]);
    Ey[i] = s[1] * peak * oracle_env(t[i], tf) * sinf(omega * t[i] + phi[1]);
    Ez[i] = s[2] * peak * oracle_env(t[i], tf) * sinf(omega * t[i] + phi[2]);
    Ax[i] = 0.0;
    Ay[i] = 0.0;
    Az[i] = 0.0;
  }
  for (int i = 1; i < nt; ++i) {
    Ax[i] = Ax[i - 1] - Ex[i - 1] * dt;
    Ay[i] = Ay[i - 1] - Ey[i - 1] * dt;
    Az[i] = Az[i - 1] - Ez[i - 1] * dt;
  }
}
