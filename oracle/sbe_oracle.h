/* CPU restatement of the reference's SBE propagation path -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load this library, and only
 * as the checker.  It restates, in plain C and FP64, the algorithm of rodrigomarher/HHG-Solids:
 *   src/wannier_tb.cpp:15-113   TB file parse (H_mn stored at [n][m], degeneracies ignored)
 *   src/grid.cpp:27-111         lattice, reciprocal vectors, centred supercell, time grid
 *   src/vec3_util.cpp:13-36     Cramer solve used to place X_R on grid cells ((int) truncation)
 *   src/hamiltonian.cpp:8-39, src/berry_connection.cpp:7-50   placement (r = -x_bc)
 *   src/velocity.cpp:41-115     v_a(R) = i (R_a H(R) - [r_a, H]_conv(R)), built in SI units
 *   src/efield.cpp:30-50        E(t) with float sinf/sqrtf, A by left-rectangle integration
 *   src/hamiltonian.cpp:70-101, src/operator.cpp:165-280, src/rdm.cpp:23-38   rho0 = U f U^+
 *   src/swe.cpp:183-233, src/solver.cpp:86-181,1411-1726, src/observable.cpp:16-30   RK4 + J
 * The propagation is restated in the k-space-resident form that the real-space FFT-convolution
 * solver is equivalent to for even N1, N2:
 *   H_s(k) = sum_R e^{-ik.R} e^{iA_i.R} (H0_R + E_s . r_R),  k_n = -i [H_s(k), rho(k) + c_n k_{n-1}],
 *   rho += 0.1666666666666 dt (k1 + 2 k2 + 2 k3 + k4),
 *   J_a(t_i) = (1/Nk) sum_k sum_ij W_a,ij(k) conj(rho_ij(k)),  W_a(k) = sum_{R in 4x4} e^{-ik.R} e^{iA_i.R} v_a(R).
 * Parity of this restatement is pinned against the reference itself, compiled from its own sources
 * (oracle/Makefile -> _ref/libwannier.so); the fixtures it produced live in tests/golden/. */
#ifndef HHG_SBE_ORACLE_H
#define HHG_SBE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nr1, nr2, nr3;
  double tmax, dt, intensity, lambda_nm, tmax_field;
  double pol[3], phi[3];
  int tb_flags; /* 0: read the TB file as the reference does; bit 0: divide by the degeneracies;
                   bit 1: keep the file's orbital order (an option the reference does not have) */
} oracle_settings;

/* nt = (int)(tmax / dt)  (src/swe.cpp:52). */
int oracle_nt(const oracle_settings* s);
/* Number of orbitals and R sites of a TB file; returns 0 on success. */
int oracle_model_info(const char* tb, int* nw, int* nsites);
/* t (au, nt), E and A (au, [3][nt]) exactly as the reference computes them. */
int oracle_fields(const char* tb, const oracle_settings* s, double* t, double* E, double* A);
/* Dense placed operators in SI, layout [nr1*nr2][nw*nw] complex (interleaved re,im):
 * H (eV), r_a = -x_bc (Angstrom, [3][...]) ; returns nw or < 0 on error. */
int oracle_place(const char* tb, const oracle_settings* s, double* H, double* r3);
/* Velocity v_a(R) on the 4x4 cell window n in {-2,-1,0,1}^2, [3][16][nw*nw] complex, eV*Angstrom;
 * window cell w = (n1+2)*4 + (n2+2). */
int oracle_velocity_window(const char* tb, const oracle_settings* s, double* v3w);
/* Equilibrium rho(k) in the W gauge, [nr1*nr2][nw*nw] complex. */
int oracle_rho0(const char* tb, const oracle_settings* s, double* rho_k);
/* Full propagation restricted to k-points [k_begin, k_end) of the flattened grid (m1*nr2 + m2):
 * t (au, nt) and the partial current J (complex, [3][nt]) normalised by the FULL nr1*nr2, so that
 * partial currents over a partition of the k-grid add up to the full current. Returns nt. */
int oracle_run(const char* tb, const oracle_settings* s, int k_begin, int k_end, double* t, double* J);
/* As oracle_run, but only the first nsteps steps (fields still built for the full nt, so the
 * samples equal the first nsteps samples of the full run); J entries after nsteps stay zero. */
int oracle_run_steps(const char* tb, const oracle_settings* s, int k_begin, int k_end, int nsteps, double* t,
                     double* J);

/* The reference's k-space solver (src/solver_kspace.cpp, never reached by the reference's own
 * entry points) driven step by step like the real-space one, without a Peierls phase: per stage,
 * H0(k) + E_s . r(k) interpolated at k - A_s by the Catmull-Rom bicubic of src/interpolation.cpp
 * (with its index order), full commutator, RK4; J from the 4x4 window with no phase.  All k-points,
 * first nsteps steps (< 0: all); t (au) and J ([3][nt]) as in oracle_run.  Returns nt. */
int oracle_run_kspace_steps(const char* tb, const oracle_settings* s, int nsteps, double* t, double* J);

#ifdef __cplusplus
}
#endif
#endif
