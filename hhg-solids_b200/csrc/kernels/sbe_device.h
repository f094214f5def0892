// Host <-> device interface of the SBE propagation kernels (plain structs, no torch types).
#pragma once
#include <cuda_runtime.h>

namespace hhg {

constexpr int kMaxOrb = 16;   // largest nw the kernels take
constexpr int kWindow = 16;   // 4x4 current window of the reference observable (n in {-2,-1,0,1}^2)
constexpr int kRing = 32;     // time steps per staged chunk (field table in, current partials out)

// One solve's device-resident tables (all pointers are device memory).
struct SolveTables {
  int nw, nw2, N1, N2, Nk, nt;
  int row0, row1;    // k-grid rows m1 in [row0, row1) are propagated (a slab of a sharded solve);
                     // J is still normalised by the full Nk, so slab currents add up

  int step0, step1;  // one launch propagates steps [step0, step1); 0 and nt for the whole pulse.  A pulse run
                     // as consecutive chunks gives the same rho and current bit for bit.

  int kmode;         // 0: the real-space solver (src/solver.cpp); 1: the k-space solver (src/solver_kspace.cpp),
                     // whose stages see H at three points per step (t, t + dt/2, t + dt): Q and P are then
                     // tables of evaluation points 0 .. 2 nt (point 2i + s/2 for stage s of step i) and the
                     // window carries no phase

  int hermitian;     // placed H0 and r are Hermitian-symmetric on the grid: [H,X] = HX - (HX)^+
  double dt;         // au
  int nax, ax_id[3]; // field axes with a non-zero polarisation component
  int nj, j_id[3];   // current axes with a non-zero velocity window
  const double* es;  // [nt][3 stages (t, t+dt/2, t+dt)][3 axes] field samples (src/solver.cpp:109-148)

  // Sparse form (thread-per-k kernel): occupied cells and non-zero window cells.
  int ncell;
  const int2* cell_n;   // [ncell] (n1, n2)
  const double2* H0;    // [ncell][nw2] Hartree
  const double2* R;     // [nax][ncell][nw2] bohr (r = -x_bc)
  int nwin;
  const int2* win_n;    // [nwin]
  const double2* V;     // [nj][nwin][nw2] velocity on the window cells
  const double2* Q;     // [nt][ncell + nwin] Peierls phase e^{i A(t_i).R_c} of each listed cell (k-space
                        // solver: [2 nt + 1][ncell + nwin] interpolation multipliers, window entries 1)

  // Bounding box of the occupied cells (element-group kernel, tables in GroupTables).
  int b1lo, b1n, b2lo, b2n;
  int np;               // |n| range of the P tables

  const double2* T1;    // [N1] e^{-2 pi i m/N1}
  const double2* T2;    // [N2] e^{-2 pi i m/N2}
};

// Tables of the element-group kernel in both precisions: box [1+nax][b1n][b2n][nw2] (H0 then the
// field-coupled r), window velocity [nj][4][4][nw2], P [nt][2][2np+1] = e^{i n A(t_i).a_1|2}, twiddles.
struct GroupTables {
  const double2 *Xbox64, *Xwin64, *P64, *T1_64, *T2_64;
  const float2 *Xbox32, *Xwin32, *P32, *T1_32, *T2_32;
  void* pre;  // scratch of LaunchShape::pre_bytes for precomputed inner sums (shapes with pre_chunk > 0)
};

struct LaunchShape {
  int kernel;      // 0: thread per k-point (FP64, nw <= 2, Hermitian); 1: element groups FP64; 2: element groups mixed;
                   // 3: column tiles, thread per k-point (FP64, nw <= 2, Hermitian); 4: tensor-core fragment
                   // kernel (mixed, 11 or 12 orbitals; variant indexes its shape table); 5: FP64 tensor-core
                   // fragment kernel (plain form, 11 or 12 orbitals); 6: tile kernel (mixed, 11 or 12 orbitals,
                   // half a warp per k-point)
  int k_per_cta;   // k-points per CTA
  int group;       // threads per k-point
  int threads;     // threads per CTA
  int ctas;        // grid size (persistent physical CTAs, <= vctas)
  int vctas;       // virtual CTAs: fixed work split and current-partial rows (result independent of ctas)
  int ntiles;      // work tiles
  int box_sm, win_sm;  // element groups: cell tables staged in shared memory
  int ept;             // element groups: matrix elements per thread
  int variant;         // element groups: compiled shape (-1: runtime-shaped instance); column tiles: 1 when
                       // the box rows are Hermitian-halved
  int kmode;           // instance for the k-space solver (SolveTables::kmode)
  size_t smem;     // dynamic shared memory bytes
  int pre_chunk;     // element groups: > 0 when the inner Wannier sums of every column are precomputed
                     // by a separate kernel, this many steps per launch pair
  size_t pre_bytes;  // scratch those sums need (GroupTables::pre)
};

// One solve of a batched element-group launch (device memory).
struct BatchDesc {
  SolveTables t;
  GroupTables gt;
  int B, G, box_sm, win_sm, vctas, pad;
  double2* rho;
  double2* Jpart;
};

// Picks kernel and launch shape for a solve on the current device; false (with a reason) if it
// cannot run it.  precision 0: plain FP64; 1: mixed (FP32 commutators and Wannier sums, FP64 state,
// RK accumulation and current sum).
// tile_hint > 0 asks for smaller tiles than the default (element groups: k-points per CTA; column
// tiles: parts per column); the autotuner of swe.cpp passes the measured best.  Result bits depend
// on the tile shape only through the order of the final k-sum.
bool plan_propagate(const SolveTables& t, int precision, int sm_count, LaunchShape* out, char* why, int why_len,
                    int tile_hint = 0);
bool plan_group(const SolveTables& t, int precision, int sm_count, LaunchShape* out, char* why, int why_len,
                int tile_hint = 0);
int launch_group(const SolveTables& t, const GroupTables& gt, const LaunchShape& s, double2* rho, double2* Jpart,
                 cudaStream_t stream);
// Column-tile kernel (nw <= 2, Hermitian, FP64): false if the solve does not suit it.
bool plan_kcol(const SolveTables& t, int sm_count, LaunchShape* out, size_t smem_max, int parts_hint = 0);
void launch_kcol(const SolveTables& t, const GroupTables& gt, const LaunchShape& s, double2* rho, double2* Jpart,
                 cudaStream_t stream);
// Persistent work-stealing launch over (solve, virtual CTA) items of solves sharing the kernel shape of
// `s` (same variant, threads); smem = the largest member's.  Returns the grid size.
int launch_group_batch(const LaunchShape& s, const BatchDesc* descs, const int2* items, int nitems, int* counter,
                       size_t smem, int sm_count, cudaStream_t stream);

// rho[Nk][nw2] in/out (k-space, W gauge). Jpart[vctas][nt][3] is accumulated (zero it first);
// J[3][nt] receives the reduced, 1/Nk-normalised current.  Returns the number of launches.
// If `after_propagate` is non-null it is recorded between the propagation and the reduction.
int launch_propagate(const SolveTables& t, const GroupTables& gt, const LaunchShape& s, double2* rho, double2* Jpart,
                     double2* J, cudaStream_t stream, cudaEvent_t after_propagate = nullptr);
// Records `ev` on `stream`, as a graph node that records it when the graph runs if the stream is being
// captured.
cudaError_t record_event(cudaEvent_t ev, cudaStream_t stream);
// The propagation launches alone (steps [t.step0, t.step1)), without the reduction; returns their number.
int launch_propagate_steps(const SolveTables& t, const GroupTables& gt, const LaunchShape& s, double2* rho,
                           double2* Jpart, cudaStream_t stream);

// Same as launch_propagate, with the current partials in a fixed device array owned by the
// library instead of a caller buffer (see noalloc.cu).  Returns 0, or -1 with a reason in `why`.
int propagate_static_scratch(const SolveTables& t, const GroupTables& gt, const LaunchShape& s, double2* rho,
                             double2* J, cudaStream_t stream, char* why, int why_len);
size_t static_scratch_capacity();

// J[3][nt] = (1/Nk) sum over the vctas rows of Jpart, in row order.
void launch_reduce_current(const double2* Jpart, int vctas, int nt, int Nk, double2* J, cudaStream_t stream);

// rho0(k) = U f U^+ of H(k) = sum_cells e^{-ik.R} H0 (no field), one warp per k-point.
int launch_rho0_fp64(const SolveTables& t, double2* rho, cudaStream_t stream);

// S[b] = fftshift(fft(ifftshift(gradient(J[b], h)))) for `count` signals of length n (device
// buffers; scratch holds count*n values).  Returns the number of FFT passes, or -1.
int spectrum_device(const double2* J, int n, int count, double h, double2* S, double2* scratch, cudaStream_t stream);
// I[b][(h-1)/2], h = 1, 3, ..., 2 nh - 1: |S|^2 summed over the harmonic-order window (h - 1/2, h + 1/2)
// of the order axis linspace(-n pi/tmax, n pi/tmax, n) / (2 pi 300 / lambda_nm).
int harmonics_device(const double2* S, int n, int count, double tmax, double lambda_nm, int nh, double* I,
                     cudaStream_t stream);

// Per-step factor tables on the device (tables.cu).  A [3][nt] (au), Rc [ncw][3] (bohr), lat the first
// two lattice vectors (bohr): Q [nt][ncw] Peierls phases, P [nt][2][2np+1] separable powers.
void launch_peierls_tables(const double* A, const double* Rc, const double lat[2][3], int nt, int ncw, int np,
                           double2* Q, double2* P, cudaStream_t stream);
// k-space solver: x0 [npts][2] stencil offsets -N u_d; P [npts][2][2np+1] interpolation factors,
// Q [npts][ncw] their products on the (transposed) cells, 1 on the window cells.
void launch_interp_tables(const double* x0, int N, int np, int npts, const int2* cellp, int ncell, int ncw, double2* P,
                          double2* Q, cudaStream_t stream);
void launch_to_float2(const double2* in, size_t n, float2* out, cudaStream_t stream);

// FMA-chain throughput probe (TFLOP/s) on the current device.
int measure_fma_peaks(double* fp64_tflops, double* fp32_tflops);

}  // namespace hhg
