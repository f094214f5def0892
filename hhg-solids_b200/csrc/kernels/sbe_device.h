// Host <-> device interface of the SBE propagation kernels (plain structs, no torch types).
#pragma once
#include <cuda_runtime.h>

namespace hhg {

constexpr int kMaxOrb = 16;       // largest nw the kernels take
constexpr int kWindow = 16;       // 4x4 current window of the reference observable

// Per time step, precomputed on the host in FP64.
struct StepParams {
  double es[3][3];   // field samples [t, t+dt/2, t+dt][axis] (src/solver.cpp:109-148), au
  double2 p1, p2;    // e^{i A(t_i).a1}, e^{i A(t_i).a2}: Peierls phase per unit cell step
};

// One solve's device-resident tables.
struct SolveTables {
  int nw, nw2, N1, N2, Nk, nt;
  int ncell;                 // support cells of H0 / r
  const int2* cell_n;        // [ncell] (n1, n2)
  const double2* H0;         // [ncell][nw2] Hartree
  int nax;                   // field axes with a non-zero polarisation component
  int ax_id[3];
  const double2* R;          // [nax][ncell][nw2] bohr (r = -x_bc)
  int nj;                    // current axes with a non-zero velocity window
  int j_id[3];
  const double2* V;          // [nj][16][nw2] velocity on the window cells
  const double2* T1;         // [N1] e^{-2 pi i m/N1}
  const double2* T2;         // [N2] e^{-2 pi i m/N2}
  const StepParams* steps;   // [nt]
  double dt;                 // au
  int hermitian;             // placed H0 and r are Hermitian-symmetric on the grid: [H,X] = HX - (HX)^+
};

struct LaunchShape {
  int k_per_cta;   // k-points (element groups) per CTA
  int group;       // threads per k-point (power of two <= 32, or a multiple of 32)
  int ctas;        // grid size (persistent CTAs)
  size_t smem;     // dynamic shared memory bytes
};

// Picks the launch shape for a solve on the current device; returns false if nw/ncell don't fit.
bool plan_propagate(const SolveTables& t, int sm_count, LaunchShape* out, char* why, int why_len);

// rho[Nk][nw2] in/out (k-space, W gauge). Jpart[ctas][nt][3] is accumulated (zero it first);
// J[3][nt] receives the reduced, 1/Nk-normalised current. Returns the number of launches.
// If `after_propagate` is non-null it is recorded between the propagation and the reduction.
int launch_propagate_fp64(const SolveTables& t, const LaunchShape& s, double2* rho, double2* Jpart, double2* J,
                          cudaStream_t stream, cudaEvent_t after_propagate = nullptr);

// rho0(k) = U f U^+ of H(k) = sum_cells e^{-ik.R} H0 (no field), one k-point per thread.
int launch_rho0_fp64(const SolveTables& t, double2* rho, cudaStream_t stream);

// FMA-chain throughput probe (TFLOP/s) on the current device.
int measure_fma_peaks(double* fp64_tflops, double* fp32_tflops);

}  // namespace hhg
