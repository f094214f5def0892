/* CPU restatement of the reference's SBE propagation path -- TEST INFRASTRUCTURE ONLY.
 * See sbe_oracle.h for the scope and the reference files each part follows.  Only the checker
 * (tests/, __graft_entry__.smoke(), bench.py's cpu_baseline leg) may load this library. */
#include "sbe_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

/* Defined in sbe_oracle_fm.c (compiled with the reference's floating-point flags). */
void oracle_cramer3(double** m, double* v, double* c);
void oracle_supercell(int N1, int N2, int N3, double a[3][3], double b[3][3], double* R, double* K);
void oracle_reciprocal(double a[3][3], double b[3][3]);
void oracle_time_grid(int nt, double dt_fs, double* t);
void oracle_efield(int nt, const double* t, double lambda_nm, double tmax_field_fs, double intensity,
                   const double* s, const double* phi, double* E, double* A);

typedef struct {
  int nw, nsites;
  double lat[3][3]; /* Angstrom */
  int (*R)[3];
  cplx* hop; /* [site][n][m] = H_mn (transposed as in src/wannier_tb.cpp:74) */
  cplx* bc[3];
  int* deg;
} tb_model;

/* The optional Wannier90 reading (not the reference's): bit 1 undoes the transpose, bit 0 divides
 * each R block by its degeneracy. */
static void tb_apply_flags(tb_model* m, int flags) {
  const int nw = m->nw, nw2 = nw * nw;
  for (int s = 0; s < m->nsites; ++s) {
    cplx* blocks[4] = {m->hop + (size_t)s * nw2, m->bc[0] + (size_t)s * nw2, m->bc[1] + (size_t)s * nw2,
                       m->bc[2] + (size_t)s * nw2};
    for (int b = 0; b < 4; ++b) {
      if (flags & 2)
        for (int i = 0; i < nw; ++i)
          for (int j = i + 1; j < nw; ++j) {
            cplx t = blocks[b][i * nw + j];
            blocks[b][i * nw + j] = blocks[b][j * nw + i];
            blocks[b][j * nw + i] = t;
          }
      if ((flags & 1) && m->deg[s] > 0)
        for (int o = 0; o < nw2; ++o) blocks[b][o] /= (double)m->deg[s];
    }
  }
}

static void tb_free(tb_model* m) {
  free(m->R);
  free(m->hop);
  for (int a = 0; a < 3; ++a) free(m->bc[a]);
  free(m->deg);
  memset(m, 0, sizeof(*m));
}

static int read_line(FILE* f, char* buf, int n) {
  if (!fgets(buf, n, f)) {
    buf[0] = 0;
    return 0;
  }
  return 1;
}

/* src/wannier_tb.cpp:15-113. */
static int tb_parse(const char* path, tb_model* m) {
  memset(m, 0, sizeof(*m));
  FILE* f = fopen(path, "r");
  if (!f) return -1;
  static char line[1 << 16];
  read_line(f, line, sizeof line); /* comment */
  for (int i = 0; i < 3; ++i) {
    read_line(f, line, sizeof line);
    sscanf(line, "%lf %lf %lf", &m->lat[i][0], &m->lat[i][1], &m->lat[i][2]);
  }
  read_line(f, line, sizeof line);
  m->nw = atoi(line);
  read_line(f, line, sizeof line);
  m->nsites = atoi(line);
  if (m->nw <= 0 || m->nsites <= 0) {
    fclose(f);
    return -2;
  }
  int ndeg = (m->nsites - 1) / 15 + 1;
  m->deg = calloc((size_t)m->nsites, sizeof(int));
  int nd = 0;
  for (int i = 0; i < ndeg; ++i) { /* degeneracies: the reference parses and never applies them */
    read_line(f, line, sizeof line);
    char* p = line;
    int used = 0, v = 0;
    while (nd < m->nsites && sscanf(p, "%d%n", &v, &used) == 1) {
      m->deg[nd++] = v;
      p += used;
    }
  }
  read_line(f, line, sizeof line);
  const int nw = m->nw, nw2 = nw * nw;
  m->R = calloc((size_t)m->nsites, sizeof(*m->R));
  m->hop = calloc((size_t)m->nsites * nw2, sizeof(cplx));
  for (int a = 0; a < 3; ++a) m->bc[a] = calloc((size_t)m->nsites * nw2, sizeof(cplx));
  for (int s = 0; s < m->nsites; ++s) {
    read_line(f, line, sizeof line);
    sscanf(line, "%d %d %d", &m->R[s][0], &m->R[s][1], &m->R[s][2]);
    for (int j = 0; j < nw2; ++j) {
      int o1 = 0, o2 = 0;
      double re = 0, im = 0;
      read_line(f, line, sizeof line);
      sscanf(line, "%d %d %lf %lf", &o1, &o2, &re, &im);
      m->hop[(size_t)s * nw2 + (o2 - 1) * nw + (o1 - 1)] = re + I * im;
    }
    read_line(f, line, sizeof line);
  }
  for (int s = 0; s < m->nsites; ++s) {
    read_line(f, line, sizeof line); /* R line of the position block: not used */
    for (int j = 0; j < nw2; ++j) {
      int o1 = 0, o2 = 0;
      double v[6] = {0, 0, 0, 0, 0, 0};
      read_line(f, line, sizeof line);
      sscanf(line, "%d %d %lf %lf %lf %lf %lf %lf", &o1, &o2, &v[0], &v[1], &v[2], &v[3], &v[4], &v[5]);
      for (int a = 0; a < 3; ++a) m->bc[a][(size_t)s * nw2 + (o2 - 1) * nw + (o1 - 1)] = v[2 * a] + I * v[2 * a + 1];
    }
    read_line(f, line, sizeof line);
  }
  fclose(f);
  return 0;
}

typedef struct {
  int N1, N2, Nk, nw, nw2;
  int* site_of_cell; /* [Nk]: TB site placed on the cell (src/hamiltonian.cpp:19-32), -1 if none */
  double* R;         /* [Nk][3] Angstrom */
  double* K;
} placed_grid;

static void grid_free(placed_grid* g) {
  free(g->site_of_cell);
  free(g->R);
  free(g->K);
}

/* src/grid.cpp + src/hamiltonian.cpp:8-39 (the same search serves src/berry_connection.cpp:7-50). */
static int grid_place(const tb_model* m, const oracle_settings* s, placed_grid* g) {
  g->N1 = s->nr1;
  g->N2 = s->nr2;
  int N3 = s->nr3 > 0 ? s->nr3 : 1;
  /* 2D grids only; odd N makes the reference's fftshift/ifftshift pair shift by one cell and
   * N < 4 makes its 4x4 current window read outside the grid, so both are rejected. */
  if (N3 != 1 || g->N1 < 4 || g->N2 < 4 || (g->N1 % 2) || (g->N2 % 2)) return -3;
  g->Nk = g->N1 * g->N2;
  g->nw = m->nw;
  g->nw2 = m->nw * m->nw;
  double a[3][3], b[3][3];
  memcpy(a, m->lat, sizeof a);
  oracle_reciprocal(a, b);
  g->R = malloc(sizeof(double) * 3 * (size_t)g->Nk);
  g->K = malloc(sizeof(double) * 3 * (size_t)g->Nk);
  oracle_supercell(g->N1, g->N2, 1, a, b, g->R, g->K);
  g->site_of_cell = malloc(sizeof(int) * (size_t)g->Nk);
  double rows[3][3];
  memcpy(rows, m->lat, sizeof rows);
  double* mat[3] = {rows[0], rows[1], rows[2]};
  for (int c = 0; c < g->Nk; ++c) {
    double coef[3];
    oracle_cramer3(mat, g->R + 3 * c, coef);
    int ci[3] = {(int)coef[0], (int)coef[1], (int)coef[2]};
    int hit = -1;
    for (int st = 0; st < m->nsites; ++st)
      if (ci[0] == m->R[st][0] && ci[1] == m->R[st][1] && ci[2] == m->R[st][2]) {
        hit = st;
        break;
      }
    g->site_of_cell[c] = hit;
  }
  return 0;
}

static inline int wrap(long x, int n) {
  long r = x % n;
  return (int)(r < 0 ? r + n : r);
}

int oracle_nt(const oracle_settings* s) { return (int)(s->tmax / s->dt); }

int oracle_model_info(const char* tb, int* nw, int* nsites) {
  tb_model m;
  if (tb_parse(tb, &m)) return -1;
  *nw = m.nw;
  *nsites = m.nsites;
  tb_free(&m);
  return 0;
}

int oracle_fields(const char* tb, const oracle_settings* s, double* t, double* E, double* A) {
  (void)tb;
  int nt = oracle_nt(s);
  if (nt < 2) return -1;
  oracle_time_grid(nt, s->dt, t);
  oracle_efield(nt, t, s->lambda_nm, s->tmax_field, s->intensity, s->pol, s->phi, E, A);
  return nt;
}

int oracle_place(const char* tb, const oracle_settings* s, double* Hout, double* r3out) {
  tb_model m;
  if (tb_parse(tb, &m)) return -1;
  tb_apply_flags(&m, s->tb_flags);
  placed_grid g;
  if (grid_place(&m, s, &g)) {
    tb_free(&m);
    return -3;
  }
  cplx* H = (cplx*)Hout;
  cplx* r3 = (cplx*)r3out;
  memset(H, 0, sizeof(cplx) * (size_t)g.Nk * g.nw2);
  memset(r3, 0, sizeof(cplx) * 3 * (size_t)g.Nk * g.nw2);
  for (int c = 0; c < g.Nk; ++c) {
    int st = g.site_of_cell[c];
    if (st < 0) continue;
    for (int o = 0; o < g.nw2; ++o) {
      H[(size_t)c * g.nw2 + o] = m.hop[(size_t)st * g.nw2 + o];
      for (int a = 0; a < 3; ++a) r3[((size_t)a * g.Nk + c) * g.nw2 + o] = -m.bc[a][(size_t)st * g.nw2 + o];
    }
  }
  int nw = g.nw;
  grid_free(&g);
  tb_free(&m);
  return nw;
}

/* Occupied cells of the placed grid as (n1, n2, site) triples. */
typedef struct {
  int n1, n2, site, cell;
} cell_ref;

static int list_support(const placed_grid* g, cell_ref** out) {
  int cnt = 0;
  for (int c = 0; c < g->Nk; ++c) cnt += g->site_of_cell[c] >= 0;
  cell_ref* L = malloc(sizeof(cell_ref) * (size_t)(cnt > 0 ? cnt : 1));
  int k = 0;
  for (int c = 0; c < g->Nk; ++c)
    if (g->site_of_cell[c] >= 0) {
      L[k].n1 = c / g->N2 - g->N1 / 2;
      L[k].n2 = c % g->N2 - g->N2 / 2;
      L[k].site = g->site_of_cell[c];
      L[k].cell = c;
      ++k;
    }
  *out = L;
  return cnt;
}

static int cell_index(const placed_grid* g, int n1, int n2) {
  int i = wrap((long)n1 + g->N1 / 2, g->N1);
  int j = wrap((long)n2 + g->N2 / 2, g->N2);
  return i * g->N2 + j;
}

/* src/velocity.cpp:41-115 evaluated on the 4x4 window of src/observable.cpp:18-19.  The FFT
 * convolution of the reference is the cyclic convolution over the supercell, taken here directly:
 *   C(n) = sum_{n'} r(n') H(n - n') - H(n') r(n - n'),   v_a(n) = i (R_a(n) H(n) - C(n)). */
static void velocity_window(const tb_model* m, const placed_grid* g, cplx* v3w) {
  const int nw = g->nw, nw2 = g->nw2;
  cell_ref* sup;
  int ns = list_support(g, &sup);
  cplx* acc = malloc(sizeof(cplx) * (size_t)nw2);
  for (int a = 0; a < 3; ++a)
    for (int w = 0; w < 16; ++w) {
      int n1 = w / 4 - 2, n2 = w % 4 - 2;
      int c = cell_index(g, n1, n2);
      for (int o = 0; o < nw2; ++o) acc[o] = 0;
      for (int q = 0; q < ns; ++q) {
        int cd = cell_index(g, n1 - sup[q].n1, n2 - sup[q].n2);
        int sd = g->site_of_cell[cd];
        if (sd < 0) continue;
        const cplx* rq = m->bc[a] + (size_t)sup[q].site * nw2; /* r = -bc */
        const cplx* Hq = m->hop + (size_t)sup[q].site * nw2;
        const cplx* rd = m->bc[a] + (size_t)sd * nw2;
        const cplx* Hd = m->hop + (size_t)sd * nw2;
        for (int i = 0; i < nw; ++i)
          for (int j = 0; j < nw; ++j) {
            cplx sum = 0;
            for (int k = 0; k < nw; ++k) sum += (-rq[i * nw + k]) * Hd[k * nw + j] - Hq[i * nw + k] * (-rd[k * nw + j]);
            acc[i * nw + j] += sum;
          }
      }
      int sc = g->site_of_cell[c];
      double Ra = g->R[3 * c + a];
      for (int o = 0; o < nw2; ++o) {
        cplx h = sc >= 0 ? m->hop[(size_t)sc * nw2 + o] : 0;
        v3w[((size_t)a * 16 + w) * nw2 + o] = I * (Ra * h - acc[o]);
      }
    }
  free(acc);
  free(sup);
}

int oracle_velocity_window(const char* tb, const oracle_settings* s, double* v3w) {
  tb_model m;
  if (tb_parse(tb, &m)) return -1;
  tb_apply_flags(&m, s->tb_flags);
  placed_grid g;
  if (grid_place(&m, s, &g)) {
    tb_free(&m);
    return -3;
  }
  velocity_window(&m, &g, (cplx*)v3w);
  int nw = g.nw;
  grid_free(&g);
  tb_free(&m);
  return nw;
}

/* Cyclic complex Jacobi for a Hermitian n x n matrix A (row-major, destroyed): eigenvalues in w,
 * eigenvectors as the columns of V. */
static void jacobi_herm(int n, cplx* A, double* w, cplx* V) {
  for (int i = 0; i < n * n; ++i) V[i] = 0;
  for (int i = 0; i < n; ++i) V[i * n + i] = 1;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0, tot = 0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double a2 = creal(A[i * n + j]) * creal(A[i * n + j]) + cimag(A[i * n + j]) * cimag(A[i * n + j]);
        tot += a2;
        if (i != j) off += a2;
      }
    if (off <= 1e-32 * tot || off == 0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        cplx apq = A[p * n + q];
        double mag = cabs(apq);
        if (mag == 0) continue;
        cplx e = apq / mag;
        double tau = (creal(A[q * n + q]) - creal(A[p * n + p])) / (2 * mag);
        double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1 + tau * tau));
        double c = 1 / sqrt(1 + t * t), s = t * c;
        /* J = [[c, s e], [-s conj(e), c]] on (p, q); A <- J^+ A J, V <- V J */
        for (int k = 0; k < n; ++k) { /* columns */
          cplx akp = A[k * n + p], akq = A[k * n + q];
          A[k * n + p] = c * akp - s * conj(e) * akq;
          A[k * n + q] = s * e * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) { /* rows */
          cplx apk = A[p * n + k], aqk = A[q * n + k];
          A[p * n + k] = c * apk - s * e * aqk;
          A[q * n + k] = s * conj(e) * apk + c * aqk;
        }
        A[p * n + q] = 0;
        A[q * n + p] = 0;
        for (int k = 0; k < n; ++k) {
          cplx vkp = V[k * n + p], vkq = V[k * n + q];
          V[k * n + p] = c * vkp - s * conj(e) * vkq;
          V[k * n + q] = s * e * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < n; ++i) w[i] = creal(A[i * n + i]);
}

/* e^{-2 pi i j / N} for j in [0, N). */
static cplx* twiddles(int N) {
  cplx* T = malloc(sizeof(cplx) * (size_t)N);
  for (int j = 0; j < N; ++j) {
    double ang = 2.0 * M_PI * (double)j / (double)N;
    T[j] = cos(ang) - I * sin(ang);
  }
  return T;
}

/* rho0(k) = U f U^+ for H(k) = sum_R e^{-ik.R} H_R in au (src/swe.cpp:82-87,
 * src/hamiltonian.cpp:70-101, src/rdm.cpp:23-38).  U holds the eigenvectors of the Hermitian matrix
 * built from the lower triangle (zheevd 'L'); the occupation is f_n = [Re (U^+ H U)_nn < 0] with the
 * full H, as the reference takes it from the rotated H.  The two differ only when the placed H(R)
 * is not Hermitian-symmetric on the grid (a grid smaller than the model's R range). */
static void rho0_at(const tb_model* m, const cell_ref* sup, int ns, const cplx* T1, const cplx* T2, int N1,
                    int N2, int m1, int m2, cplx* Hk, cplx* U, double* w, cplx* rho) {
  const int nw = m->nw, nw2 = nw * nw;
  cplx* Hf = malloc(sizeof(cplx) * nw2);
  for (int o = 0; o < nw2; ++o) Hk[o] = 0;
  for (int q = 0; q < ns; ++q) {
    cplx ph = T1[wrap((long)m1 * sup[q].n1, N1)] * T2[wrap((long)m2 * sup[q].n2, N2)];
    const cplx* h = m->hop + (size_t)sup[q].site * nw2;
    for (int o = 0; o < nw2; ++o) Hk[o] += ph * (h[o] * (1.0 / 27.2114));
  }
  memcpy(Hf, Hk, sizeof(cplx) * nw2);
  for (int i = 0; i < nw; ++i) {
    Hk[i * nw + i] = creal(Hk[i * nw + i]);
    for (int j = i + 1; j < nw; ++j) Hk[i * nw + j] = conj(Hk[j * nw + i]);
  }
  jacobi_herm(nw, Hk, w, U);
  for (int n = 0; n < nw; ++n) {
    cplx d = 0;
    for (int i = 0; i < nw; ++i)
      for (int j = 0; j < nw; ++j) d += conj(U[i * nw + n]) * Hf[i * nw + j] * U[j * nw + n];
    w[n] = creal(d);
  }
  for (int i = 0; i < nw; ++i)
    for (int j = 0; j < nw; ++j) {
      cplx sum = 0;
      for (int n = 0; n < nw; ++n)
        if (w[n] < 0.0) sum += U[i * nw + n] * conj(U[j * nw + n]);
      rho[i * nw + j] = sum;
    }
  free(Hf);
}

int oracle_rho0(const char* tb, const oracle_settings* s, double* rho_out) {
  tb_model m;
  if (tb_parse(tb, &m)) return -1;
  tb_apply_flags(&m, s->tb_flags);
  placed_grid g;
  if (grid_place(&m, s, &g)) {
    tb_free(&m);
    return -3;
  }
  cell_ref* sup;
  int ns = list_support(&g, &sup);
  cplx *T1 = twiddles(g.N1), *T2 = twiddles(g.N2);
  const int nw = g.nw, nw2 = g.nw2;
  cplx* Hk = malloc(sizeof(cplx) * nw2);
  cplx* U = malloc(sizeof(cplx) * nw2);
  double* w = malloc(sizeof(double) * nw);
  cplx* rho = (cplx*)rho_out;
  for (int k = 0; k < g.Nk; ++k)
    rho0_at(&m, sup, ns, T1, T2, g.N1, g.N2, k / g.N2, k % g.N2, Hk, U, w, rho + (size_t)k * nw2);
  free(Hk);
  free(U);
  free(w);
  free(T1);
  free(T2);
  free(sup);
  grid_free(&g);
  tb_free(&m);
  return nw;
}

/* out = -i [H, X] = -i (H X - X H) */
static void rk_stage(int nw, const cplx* H, const cplx* X, cplx* out) {
  for (int i = 0; i < nw; ++i)
    for (int j = 0; j < nw; ++j) {
      cplx c = 0;
      for (int k = 0; k < nw; ++k) c += H[i * nw + k] * X[k * nw + j] - X[i * nw + k] * H[k * nw + j];
      out[i * nw + j] = -I * c;
    }
}

int oracle_run(const char* tb, const oracle_settings* s, int k_begin, int k_end, double* t, double* Jout) {
  return oracle_run_steps(tb, s, k_begin, k_end, -1, t, Jout);
}

int oracle_run_steps(const char* tb, const oracle_settings* s, int k_begin, int k_end, int nsteps, double* t,
                     double* Jout) {
  tb_model m;
  if (tb_parse(tb, &m)) return -1;
  tb_apply_flags(&m, s->tb_flags);
  placed_grid g;
  if (grid_place(&m, s, &g)) {
    tb_free(&m);
    return -3;
  }
  const int nt = oracle_nt(s);
  if (nt < 2) {
    grid_free(&g);
    tb_free(&m);
    return -4;
  }
  const int nw = g.nw, nw2 = g.nw2, N1 = g.N1, N2 = g.N2, Nk = g.Nk;
  if (k_begin < 0) k_begin = 0;
  if (k_end > Nk) k_end = Nk;

  double* E = malloc(sizeof(double) * 3 * nt);
  double* A = malloc(sizeof(double) * 3 * nt);
  oracle_fields(tb, s, t, E, A);
  const double dt = t[1] - t[0];

  cell_ref* sup;
  int ns = list_support(&g, &sup);
  /* Window cells n in {-2..1}^2 and their velocity (SI, with the to-au factor 1.0). */
  cplx* vw = malloc(sizeof(cplx) * 3 * 16 * nw2);
  velocity_window(&m, &g, vw);
  double Rw[16][3];
  int nw_cell[16][2];
  for (int w = 0; w < 16; ++w) {
    nw_cell[w][0] = w / 4 - 2;
    nw_cell[w][1] = w % 4 - 2;
    int c = cell_index(&g, nw_cell[w][0], nw_cell[w][1]);
    for (int a = 0; a < 3; ++a) Rw[w][a] = g.R[3 * c + a] * (1.0 / 0.5291772);
  }
  /* Support operators in au: H0 (eV -> Ha), r_a = -bc (Angstrom -> bohr). */
  cplx* H0 = malloc(sizeof(cplx) * (size_t)ns * nw2);
  cplx* r3 = malloc(sizeof(cplx) * 3 * (size_t)ns * nw2);
  double* Rs = malloc(sizeof(double) * 3 * (size_t)ns);
  for (int q = 0; q < ns; ++q) {
    for (int o = 0; o < nw2; ++o) {
      H0[(size_t)q * nw2 + o] = m.hop[(size_t)sup[q].site * nw2 + o] * (1.0 / 27.2114);
      for (int a = 0; a < 3; ++a)
        r3[((size_t)a * ns + q) * nw2 + o] = -m.bc[a][(size_t)sup[q].site * nw2 + o] * (1.0 / 0.5291772);
    }
    for (int a = 0; a < 3; ++a) Rs[3 * q + a] = g.R[3 * sup[q].cell + a] * (1.0 / 0.5291772);
  }

  cplx *T1 = twiddles(N1), *T2 = twiddles(N2);
  const int nk = k_end > k_begin ? k_end - k_begin : 0;
  cplx* rho = malloc(sizeof(cplx) * (size_t)(nk > 0 ? nk : 1) * nw2);
  {
    cplx* Hk = malloc(sizeof(cplx) * nw2);
    cplx* U = malloc(sizeof(cplx) * nw2);
    double* w = malloc(sizeof(double) * nw);
    for (int k = 0; k < nk; ++k) {
      int kk = k_begin + k;
      rho0_at(&m, sup, ns, T1, T2, N1, N2, kk / N2, kk % N2, Hk, U, w, rho + (size_t)k * nw2);
    }
    free(Hk);
    free(U);
    free(w);
  }

  cplx* J = (cplx*)Jout;
  for (int i = 0; i < 3 * nt; ++i) J[i] = 0;
  cplx* ph = malloc(sizeof(cplx) * (size_t)(ns > 0 ? ns : 1));
  cplx* Hk0 = malloc(sizeof(cplx) * nw2);
  cplx* Rk = malloc(sizeof(cplx) * 3 * nw2);
  cplx* Hs = malloc(sizeof(cplx) * nw2);
  cplx* X = malloc(sizeof(cplx) * nw2);
  cplx* kn[4];
  for (int n = 0; n < 4; ++n) kn[n] = malloc(sizeof(cplx) * nw2);
  cplx* Wk = malloc(sizeof(cplx) * 3 * nw2);
  cplx pw[16];

  const int nrun = (nsteps < 0 || nsteps > nt) ? nt : nsteps;
  for (int ti = 0; ti < nrun; ++ti) {
    /* src/solver.cpp:109-148: field samples at t, t + dt/2 (mean of the end points), t + dt. */
    double Es[3][3];
    for (int a = 0; a < 3; ++a) {
      const double* Ea = E + (size_t)a * nt;
      if (ti < nt - 1) {
        Es[0][a] = Ea[ti];
        Es[1][a] = 0.5 * Ea[ti] + 0.5 * Ea[ti + 1];
        Es[2][a] = Ea[ti + 1];
      } else {
        Es[0][a] = Es[1][a] = Es[2][a] = Ea[nt - 1];
      }
    }
    /* src/swe.cpp:225-233: Peierls phase exp(i A(t_i) . R) at the support and window cells. */
    const double ax = A[ti], ay = A[nt + ti], az = A[2 * nt + ti];
    for (int q = 0; q < ns; ++q) ph[q] = cexp(I * (ax * Rs[3 * q] + ay * Rs[3 * q + 1] + az * Rs[3 * q + 2]));
    for (int w = 0; w < 16; ++w) pw[w] = cexp(I * (ax * Rw[w][0] + ay * Rw[w][1] + az * Rw[w][2]));
    cplx jsum[3] = {0, 0, 0};
    for (int k = 0; k < nk; ++k) {
      const int kk = k_begin + k, m1 = kk / N2, m2 = kk % N2;
      for (int o = 0; o < nw2; ++o) {
        Hk0[o] = 0;
        Rk[o] = Rk[nw2 + o] = Rk[2 * nw2 + o] = 0;
      }
      for (int q = 0; q < ns; ++q) {
        cplx f = T1[wrap((long)m1 * sup[q].n1, N1)] * T2[wrap((long)m2 * sup[q].n2, N2)] * ph[q];
        for (int o = 0; o < nw2; ++o) {
          Hk0[o] += f * H0[(size_t)q * nw2 + o];
          for (int a = 0; a < 3; ++a) Rk[a * nw2 + o] += f * r3[((size_t)a * ns + q) * nw2 + o];
        }
      }
      cplx* r = rho + (size_t)k * nw2;
      static const double cstage[4] = {0.0, 0.5, 0.5, 1.0};
      static const int field_of_stage[4] = {0, 1, 1, 2};
      for (int n = 0; n < 4; ++n) {
        const double* e = Es[field_of_stage[n]];
        for (int o = 0; o < nw2; ++o) {
          Hs[o] = Hk0[o] + e[0] * Rk[o] + e[1] * Rk[nw2 + o] + e[2] * Rk[2 * nw2 + o];
          X[o] = n == 0 ? r[o] : r[o] + cstage[n] * dt * kn[n - 1][o];
        }
        rk_stage(nw, Hs, X, kn[n]);
      }
      for (int o = 0; o < nw2; ++o)
        r[o] = r[o] + (0.1666666666666 * dt) * (kn[0][o] + 2.0 * kn[1][o] + 2.0 * kn[2][o] + kn[3][o]);
      /* src/observable.cpp:16-30 in Parseval form. */
      for (int o = 0; o < 3 * nw2; ++o) Wk[o] = 0;
      for (int w = 0; w < 16; ++w) {
        cplx f = T1[wrap((long)m1 * nw_cell[w][0], N1)] * T2[wrap((long)m2 * nw_cell[w][1], N2)] * pw[w];
        for (int a = 0; a < 3; ++a)
          for (int o = 0; o < nw2; ++o) Wk[a * nw2 + o] += f * vw[((size_t)a * 16 + w) * nw2 + o];
      }
      for (int a = 0; a < 3; ++a)
        for (int o = 0; o < nw2; ++o) jsum[a] += Wk[a * nw2 + o] * conj(r[o]);
    }
    for (int a = 0; a < 3; ++a) J[(size_t)a * nt + ti] = jsum[a] / (double)Nk;
  }

  free(ph);
  free(Hk0);
  free(Rk);
  free(Hs);
  free(X);
  for (int n = 0; n < 4; ++n) free(kn[n]);
  free(Wk);
  free(rho);
  free(T1);
  free(T2);
  free(H0);
  free(r3);
  free(Rs);
  free(vw);
  free(E);
  free(A);
  free(sup);
  grid_free(&g);
  tb_free(&m);
  return nt;
}

/* ---------------------------------------------------------------------------------------------
 * The reference's k-space RK4 solver (src/solver_kspace.cpp:167-451, src/interpolation.cpp:17-43),
 * driven per step like the real-space one but without a Peierls phase (it has none): for every
 * stage, H_eff = H0(k) + E_s . r(k) on the k-grid (the ifftshift + forward FFT of
 * src/solver_kspace.cpp:122-142, i.e. the DFT over the placed cells), interpolated at k - A_s by
 * the Catmull-Rom bicubic of src/interpolation.cpp, with A_s = A(t), the mean of A(t) and A(t+dt)
 * for stages 2 and 3, A(t+dt) (clamped on the last step as the fields are).  The fractional
 * coordinates come from the reference's Cramer solve against the reciprocal vectors (au); the
 * interpolation reads data[yi*N1 + xi] with xi along the first coordinate and yi along the second,
 * as the reference does (on a square grid that is the grid transposed).  The commutator is the
 * full [H, X].  The reference's R<->k round trip of rho each step is the identity for even N and
 * is not repeated.  J: the Observables of src/observable.cpp:16-30 on that rho, in Parseval form
 * with no phase factor. */
static cplx cubic_at(cplx p0, cplx p1, cplx p2, cplx p3, double t) {
  /* Catmull-Rom through p1 (t = 0) and p2 (t = 1). */
  cplx a0 = -0.5 * p0 + 1.5 * p1 - 1.5 * p2 + 0.5 * p3;
  cplx a1 = p0 - 2.5 * p1 + 2.0 * p2 - 0.5 * p3;
  cplx a2 = -0.5 * p0 + 0.5 * p2;
  return ((a0 * t + a1) * t + a2) * t + p1;
}

static cplx bicubic_at(const cplx* grid, int nw2, int Nx, int Ny, double u, double v, int o) {
  double x = u * Nx, y = v * Ny;
  int ix = (int)floor(x), iy = (int)floor(y);
  double tx = x - (double)ix, ty = y - (double)iy;
  cplx row[4];
  for (int b = -1; b <= 2; ++b) {
    cplx col[4];
    for (int a = -1; a <= 2; ++a) {
      int xi = wrap((long)ix + a, Nx), yi = wrap((long)iy + b, Ny);
      col[a + 1] = grid[((size_t)yi * Nx + xi) * nw2 + o];
    }
    row[b + 1] = cubic_at(col[0], col[1], col[2], col[3], tx);
  }
  return cubic_at(row[0], row[1], row[2], row[3], ty);
}

int oracle_run_kspace_steps(const char* tb, const oracle_settings* s, int nsteps, double* t, double* Jout) {
  tb_model m;
  if (tb_parse(tb, &m)) return -1;
  tb_apply_flags(&m, s->tb_flags);
  placed_grid g;
  if (grid_place(&m, s, &g)) {
    tb_free(&m);
    return -3;
  }
  const int nt = oracle_nt(s);
  if (nt < 2) {
    grid_free(&g);
    tb_free(&m);
    return -4;
  }
  const int nw = g.nw, nw2 = g.nw2, N1 = g.N1, N2 = g.N2, Nk = g.Nk;
  const double A2au = 1.0 / 0.5291772;
  double* E = malloc(sizeof(double) * 3 * nt);
  double* A = malloc(sizeof(double) * 3 * nt);
  oracle_fields(tb, s, t, E, A);
  const double dt = t[1] - t[0];
  double b[3][3], lat[3][3];
  memcpy(lat, m.lat, sizeof lat);
  oracle_reciprocal(lat, b);
  double bau[3][3];
  for (int r = 0; r < 3; ++r)
    for (int q = 0; q < 3; ++q) bau[r][q] = b[r][q] / A2au;
  double* bm[3] = {bau[0], bau[1], bau[2]};

  cell_ref* sup;
  int ns = list_support(&g, &sup);
  cplx* vw = malloc(sizeof(cplx) * 3 * 16 * nw2);
  velocity_window(&m, &g, vw);
  cplx *T1 = twiddles(N1), *T2 = twiddles(N2);
  /* H0(k) and r_a(k) on the grid (au). */
  cplx* h0g = calloc((size_t)Nk * nw2, sizeof(cplx));
  cplx* rg = calloc(3 * (size_t)Nk * nw2, sizeof(cplx));
  for (int k = 0; k < Nk; ++k) {
    const int m1 = k / N2, m2 = k % N2;
    for (int q = 0; q < ns; ++q) {
      cplx f = T1[wrap((long)m1 * sup[q].n1, N1)] * T2[wrap((long)m2 * sup[q].n2, N2)];
      const size_t st = (size_t)sup[q].site * nw2;
      for (int o = 0; o < nw2; ++o) {
        h0g[(size_t)k * nw2 + o] += f * (m.hop[st + o] * (1.0 / 27.2114));
        for (int a = 0; a < 3; ++a) rg[((size_t)a * Nk + k) * nw2 + o] += f * (-m.bc[a][st + o] * A2au);
      }
    }
  }
  /* Windowed velocity W_a(k) (constant: no phase in this solver). */
  cplx* Wk = calloc(3 * (size_t)Nk * nw2, sizeof(cplx));
  for (int k = 0; k < Nk; ++k) {
    const int m1 = k / N2, m2 = k % N2;
    for (int w = 0; w < 16; ++w) {
      cplx f = T1[wrap((long)m1 * (w / 4 - 2), N1)] * T2[wrap((long)m2 * (w % 4 - 2), N2)];
      for (int a = 0; a < 3; ++a)
        for (int o = 0; o < nw2; ++o) Wk[((size_t)a * Nk + k) * nw2 + o] += f * vw[((size_t)a * 16 + w) * nw2 + o];
    }
  }
  cplx* rho = malloc(sizeof(cplx) * (size_t)Nk * nw2);
  {
    cplx* Hk = malloc(sizeof(cplx) * nw2);
    cplx* U = malloc(sizeof(cplx) * nw2);
    double* w = malloc(sizeof(double) * nw);
    for (int k = 0; k < Nk; ++k) rho0_at(&m, sup, ns, T1, T2, N1, N2, k / N2, k % N2, Hk, U, w, rho + (size_t)k * nw2);
    free(Hk);
    free(U);
    free(w);
  }
  cplx* heff = malloc(sizeof(cplx) * (size_t)Nk * nw2);
  cplx* kn[4];
  for (int n = 0; n < 4; ++n) kn[n] = malloc(sizeof(cplx) * (size_t)Nk * nw2);
  cplx* Hs = malloc(sizeof(cplx) * nw2);
  cplx* X = malloc(sizeof(cplx) * nw2);
  cplx* J = (cplx*)Jout;
  for (int i = 0; i < 3 * nt; ++i) J[i] = 0;
  const int nrun = (nsteps < 0 || nsteps > nt) ? nt : nsteps;
  for (int ti = 0; ti < nrun; ++ti) {
    /* src/solver_kspace.cpp:168-229: E and A at t, their end-point mean, t + dt (clamped). */
    double Es[3][3], As[3][3];
    for (int a = 0; a < 3; ++a) {
      const double* Ea = E + (size_t)a * nt;
      const double* Aa = A + (size_t)a * nt;
      if (ti < nt - 1) {
        Es[0][a] = Ea[ti];
        Es[1][a] = 0.5 * Ea[ti] + 0.5 * Ea[ti + 1];
        Es[2][a] = Ea[ti + 1];
        As[0][a] = Aa[ti];
        As[1][a] = 0.5 * Aa[ti] + 0.5 * Aa[ti + 1];
        As[2][a] = Aa[ti + 1];
      } else {
        Es[0][a] = Es[1][a] = Es[2][a] = Ea[nt - 1];
        As[0][a] = As[1][a] = As[2][a] = Aa[nt - 1];
      }
    }
    static const double cstage[4] = {0.0, 0.5, 0.5, 1.0};
    static const int point_of_stage[4] = {0, 1, 1, 2};
    for (int n = 0; n < 4; ++n) {
      const int f = point_of_stage[n];
      for (size_t q = 0; q < (size_t)Nk * nw2; ++q)
        heff[q] = h0g[q] + Es[f][0] * rg[q] + Es[f][1] * rg[(size_t)Nk * nw2 + q] + Es[f][2] * rg[2 * (size_t)Nk * nw2 + q];
      for (int k = 0; k < Nk; ++k) {
        double kv[3], c[3];
        for (int a = 0; a < 3; ++a) kv[a] = g.K[3 * k + a] / A2au - As[f][a];
        oracle_cramer3(bm, kv, c);
        for (int o = 0; o < nw2; ++o) {
          Hs[o] = bicubic_at(heff, nw2, N1, N2, c[0], c[1], o);
          X[o] = n == 0 ? rho[(size_t)k * nw2 + o] : rho[(size_t)k * nw2 + o] + cstage[n] * dt * kn[n - 1][(size_t)k * nw2 + o];
        }
        rk_stage(nw, Hs, X, kn[n] + (size_t)k * nw2);
      }
    }
    cplx jsum[3] = {0, 0, 0};
    for (int k = 0; k < Nk; ++k) {
      cplx* r = rho + (size_t)k * nw2;
      for (int o = 0; o < nw2; ++o) {
        const size_t q = (size_t)k * nw2 + o;
        r[o] = r[o] + (0.1666666666666 * dt) * (kn[0][q] + 2.0 * kn[1][q] + 2.0 * kn[2][q] + kn[3][q]);
      }
      for (int a = 0; a < 3; ++a)
        for (int o = 0; o < nw2; ++o) jsum[a] += Wk[((size_t)a * Nk + k) * nw2 + o] * conj(r[o]);
    }
    for (int a = 0; a < 3; ++a) J[(size_t)a * nt + ti] = jsum[a] / (double)Nk;
  }
  free(heff);
  for (int n = 0; n < 4; ++n) free(kn[n]);
  free(Hs);
  free(X);
  free(rho);
  free(Wk);
  free(h0g);
  free(rg);
  free(T1);
  free(T2);
  free(vw);
  free(E);
  free(A);
  free(sup);
  grid_free(&g);
  tb_free(&m);
  return nt;
}
