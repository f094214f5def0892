// Probe over the reference's own objects (test infrastructure; built only by oracle/Makefile).
//
// SWESim keeps its operators private (include/swe.h:7-24), so this file rebuilds the same objects
// in the order of SWESim::_init (src/swe.cpp:49-93) and copies intermediate arrays out, so that
// the tests can pin each setup stage of the restatement and of the product separately.
#include <complex>
#include <cstring>
#include <string>

#include "berry_connection.h"
#include "efield.h"
#include "grid.h"
#include "hamiltonian.h"
#include "matrix_field.h"
#include "observable.h"
#include "rdm.h"
#include "settings.h"
#include "solver_kspace.h"
#include "velocity.h"
#include "wannier_tb.h"

namespace {
Settings* make_settings(int n1, int n2, double tmax, double dt, double intensity, double lambda_nm,
                        double tmax_field, const double* pol, const double* phi) {
  Settings* s = new Settings();
  s->nr1 = n1;
  s->nr2 = n2;
  s->nr3 = 1;
  s->tmax = tmax;
  s->dt = dt;
  s->intensity_wcm2 = intensity;
  s->lambda_nm = lambda_nm;
  s->tmax_field = tmax_field;
  s->sx = pol[0];
  s->sy = pol[1];
  s->sz = pol[2];
  s->phi_x = phi[0];
  s->phi_y = phi[1];
  s->phi_z = phi[2];
  return s;
}
void copy_field(Operator* op, int npts, int nw2, cdouble* dst) {
  for (int i = 0; i < npts; ++i)
    for (int o = 0; o < nw2; ++o) dst[(size_t)i * nw2 + o] = op->data_ptr()[i][o];
}
}  // namespace

extern "C" {

// Number of time steps the reference derives from the settings (src/swe.cpp:52).
int probe_nt(double tmax, double dt) {
  Settings s;
  s.tmax = tmax;
  s.dt = dt;
  s.nt = s.tmax / s.dt;
  return s.nt;
}

// t (au), E and A (au, [3][nt]) as built by Efield::init_fields after the au conversion.
int probe_fields(const char* tb, int n1, int n2, double tmax, double dt, double intensity, double lambda_nm,
                 double tmax_field, const double* pol, const double* phi, double* t, double* E, double* A) {
  Settings* s = make_settings(n1, n2, tmax, dt, intensity, lambda_nm, tmax_field, pol, phi);
  WannierTB* w = new WannierTB(tb);
  s->nt = s->tmax / s->dt;
  s->num_orb = w->num_orb;
  s->num_sites = w->num_sites;
  Grid* g = new Grid(s, w);
  Efield* f = new Efield(s, g, SI);
  w->convert_to_au();
  g->convert_to_au();
  f->convert_to_au();
  f->init_fields();
  int nt = s->nt;
  for (int i = 0; i < nt; ++i) {
    t[i] = g->t()[i];
    E[i] = f->E_x[i];
    E[nt + i] = f->E_y[i];
    E[2 * nt + i] = f->E_z[i];
    A[i] = f->A_x[i];
    A[nt + i] = f->A_y[i];
    A[2 * nt + i] = f->A_z[i];
  }
  delete f;
  delete g;
  delete w;
  delete s;
  return nt;
}

// Placed operators in R space and SI units, in the reference's AoS layout [n1*n2][nw*nw]:
// H (eV), r_a = -x_bc (Angstrom) and v_a (eV*Angstrom, built in SI, src/swe.cpp:66-68).
int probe_operators(const char* tb, int n1, int n2, cdouble* H, cdouble* r3, cdouble* v3) {
  const double pol[3] = {0, 1, 0}, phi[3] = {0, 0, 0};
  Settings* s = make_settings(n1, n2, 1.0, 0.5, 1e12, 3000.0, 80.0, pol, phi);
  WannierTB* w = new WannierTB(tb);
  s->nt = s->tmax / s->dt;
  s->num_orb = w->num_orb;
  s->num_sites = w->num_sites;
  Grid* g = new Grid(s, w);
  Hamiltonian* h = new Hamiltonian(s, g, w, WGAUGE, RSPACE);
  BerryConnection* r[3];
  Velocity* v[3];
  for (int a = 0; a < 3; ++a) r[a] = new BerryConnection(s, g, w, WGAUGE, RSPACE, a);
  for (int a = 0; a < 3; ++a) {
    v[a] = new Velocity(s, g, w, WGAUGE, RSPACE);
    v[a]->setup(h, r[a], a);
  }
  const int npts = n1 * n2, nw2 = w->num_orb * w->num_orb;
  copy_field(h, npts, nw2, H);
  for (int a = 0; a < 3; ++a) {
    copy_field(r[a], npts, nw2, r3 + (size_t)a * npts * nw2);
    copy_field(v[a], npts, nw2, v3 + (size_t)a * npts * nw2);
  }
  int nw = w->num_orb;
  for (int a = 0; a < 3; ++a) {
    delete v[a];
    delete r[a];
  }
  delete h;
  delete g;
  delete w;
  delete s;
  return nw;
}

// Equilibrium density matrix in k space, W gauge (after src/swe.cpp:85-86), plus H(k) in the W
// gauge (au) that was diagonalised (src/swe.cpp:82-83), both [n1*n2][nw*nw].
int probe_rho0(const char* tb, int n1, int n2, cdouble* rho_k, cdouble* Hk) {
  const double pol[3] = {0, 1, 0}, phi[3] = {0, 0, 0};
  Settings* s = make_settings(n1, n2, 1.0, 0.5, 1e12, 3000.0, 80.0, pol, phi);
  WannierTB* w = new WannierTB(tb);
  s->nt = s->tmax / s->dt;
  s->num_orb = w->num_orb;
  s->num_sites = w->num_sites;
  Grid* g = new Grid(s, w);
  Hamiltonian* h = new Hamiltonian(s, g, w, WGAUGE, RSPACE);
  RDM* rho = new RDM(s, g, w, WGAUGE, RSPACE);
  MatrixField* U = new MatrixField(s, w);
  w->convert_to_au();
  g->convert_to_au();
  h->convert_to_au();
  rho->convert_to_au();
  h->convert_to_k();
  const int npts = n1 * n2, nw2 = w->num_orb * w->num_orb;
  copy_field(h, npts, nw2, Hk);
  h->diagonalization_W_KSPACE(U);
  rho->convert_to_k();
  h->convert_w_to_h(U);
  rho->convert_w_to_h(U);
  rho->calculate_equilibrium(h);
  rho->convert_h_to_w(U);
  copy_field(rho, npts, nw2, rho_k);
  int nw = w->num_orb;
  delete U;
  delete rho;
  delete h;
  delete g;
  delete w;
  delete s;
  return nw;
}

// The reference's k-space RK4 solver (src/solver_kspace.cpp), which no reference entry point
// reaches, driven the way SWESim drives its real-space solver: SWESim::_init's setup
// (src/swe.cpp:49-93), Solver_kspace::init, then per step step_rk4(ti) followed by the three
// Observables of src/swe.cpp:203-205 on the real-space rho it leaves behind (no Peierls phase:
// this solver has none).  First nsteps steps; t (au, nt) and J ([3][nt], zero after nsteps).
int probe_kspace_run(const char* tb, int n1, int n2, double tmax, double dt, double intensity, double lambda_nm,
                     double tmax_field, const double* pol, const double* phi, int nsteps, double* t, cdouble* J) {
  Settings* s = make_settings(n1, n2, tmax, dt, intensity, lambda_nm, tmax_field, pol, phi);
  WannierTB* w = new WannierTB(tb);
  s->nt = s->tmax / s->dt;
  s->num_orb = w->num_orb;
  s->num_sites = w->num_sites;
  Grid* g = new Grid(s, w);
  Hamiltonian* h = new Hamiltonian(s, g, w, WGAUGE, RSPACE);
  RDM* rho = new RDM(s, g, w, WGAUGE, RSPACE);
  BerryConnection* r[3];
  Velocity* v[3];
  for (int a = 0; a < 3; ++a) r[a] = new BerryConnection(s, g, w, WGAUGE, RSPACE, a);
  for (int a = 0; a < 3; ++a) v[a] = new Velocity(s, g, w, WGAUGE, RSPACE);
  for (int a = 0; a < 3; ++a) v[a]->setup(h, r[a], a);
  MatrixField* U = new MatrixField(s, w);
  Efield* f = new Efield(s, g, SI);
  Observable* obs[3];
  for (int a = 0; a < 3; ++a) obs[a] = new Observable(s, g, rho, v[a]);
  w->convert_to_au();
  g->convert_to_au();
  h->convert_to_au();
  rho->convert_to_au();
  for (int a = 0; a < 3; ++a) r[a]->convert_to_au();
  f->convert_to_au();
  for (int a = 0; a < 3; ++a) v[a]->convert_to_au();
  f->init_fields();
  h->convert_to_k();
  h->diagonalization_W_KSPACE(U);
  rho->convert_to_k();
  h->convert_w_to_h(U);
  rho->convert_w_to_h(U);
  rho->calculate_equilibrium(h);
  h->convert_h_to_w(U);
  h->convert_to_r();
  rho->convert_h_to_w(U);
  rho->convert_to_r();
  Solver_kspace* ks = new Solver_kspace(s, g, h, rho, r, f, w);
  ks->init();
  const int nt = s->nt;
  const int nrun = (nsteps < 0 || nsteps > nt) ? nt : nsteps;
  for (int ti = 0; ti < nrun; ++ti) {
    ks->step_rk4(ti);
    for (int a = 0; a < 3; ++a) obs[a]->calculate();
  }
  for (int i = 0; i < nt; ++i) {
    t[i] = g->t()[i];
    for (int a = 0; a < 3; ++a) J[(size_t)a * nt + i] = i < nrun ? obs[a]->get_ptr()[i] : cdouble(0.0, 0.0);
  }
  delete ks;
  for (int a = 0; a < 3; ++a) {
    delete obs[a];
    delete v[a];
    delete r[a];
  }
  delete f;
  delete U;
  delete rho;
  delete h;
  delete g;
  delete w;
  delete s;
  return nt;
}

// The same k-space drive, split for timing: setup once, then batches of steps (the reference's CPU
// cost per RK4 step of this solver, without its setup).
struct KspaceRun {
  Settings* s;
  WannierTB* w;
  Grid* g;
  Hamiltonian* h;
  RDM* rho;
  BerryConnection* r[3];
  Velocity* v[3];
  MatrixField* U;
  Efield* f;
  Observable* obs[3];
  Solver_kspace* ks;
  int ti;
};

void* probe_kspace_new(const char* tb, int n1, int n2, double tmax, double dt, double intensity, double lambda_nm,
                       double tmax_field, const double* pol, const double* phi) {
  KspaceRun* k = new KspaceRun();
  k->s = make_settings(n1, n2, tmax, dt, intensity, lambda_nm, tmax_field, pol, phi);
  Settings* s = k->s;
  k->w = new WannierTB(tb);
  s->nt = s->tmax / s->dt;
  s->num_orb = k->w->num_orb;
  s->num_sites = k->w->num_sites;
  k->g = new Grid(s, k->w);
  k->h = new Hamiltonian(s, k->g, k->w, WGAUGE, RSPACE);
  k->rho = new RDM(s, k->g, k->w, WGAUGE, RSPACE);
  for (int a = 0; a < 3; ++a) k->r[a] = new BerryConnection(s, k->g, k->w, WGAUGE, RSPACE, a);
  for (int a = 0; a < 3; ++a) k->v[a] = new Velocity(s, k->g, k->w, WGAUGE, RSPACE);
  for (int a = 0; a < 3; ++a) k->v[a]->setup(k->h, k->r[a], a);
  k->U = new MatrixField(s, k->w);
  k->f = new Efield(s, k->g, SI);
  for (int a = 0; a < 3; ++a) k->obs[a] = new Observable(s, k->g, k->rho, k->v[a]);
  k->w->convert_to_au();
  k->g->convert_to_au();
  k->h->convert_to_au();
  k->rho->convert_to_au();
  for (int a = 0; a < 3; ++a) k->r[a]->convert_to_au();
  k->f->convert_to_au();
  for (int a = 0; a < 3; ++a) k->v[a]->convert_to_au();
  k->f->init_fields();
  k->h->convert_to_k();
  k->h->diagonalization_W_KSPACE(k->U);
  k->rho->convert_to_k();
  k->h->convert_w_to_h(k->U);
  k->rho->convert_w_to_h(k->U);
  k->rho->calculate_equilibrium(k->h);
  k->h->convert_h_to_w(k->U);
  k->h->convert_to_r();
  k->rho->convert_h_to_w(k->U);
  k->rho->convert_to_r();
  k->ks = new Solver_kspace(s, k->g, k->h, k->rho, k->r, k->f, k->w);
  k->ks->init();
  k->ti = 0;
  return k;
}

// nsteps more steps (the step index wraps before the end of the pulse).
void probe_kspace_steps(void* handle, int nsteps) {
  KspaceRun* k = static_cast<KspaceRun*>(handle);
  for (int i = 0; i < nsteps; ++i) {
    k->ks->step_rk4(k->ti);
    for (int a = 0; a < 3; ++a) k->obs[a]->calculate();
    k->ti = (k->ti + 1) % (k->s->nt - 1);
  }
}

void probe_kspace_delete(void* handle) {
  KspaceRun* k = static_cast<KspaceRun*>(handle);
  delete k->ks;
  for (int a = 0; a < 3; ++a) {
    delete k->obs[a];
    delete k->v[a];
    delete k->r[a];
  }
  delete k->f;
  delete k->U;
  delete k->rho;
  delete k->h;
  delete k->g;
  delete k->w;
  delete k->s;
  delete k;
}
}
