/* hhg-b200: B200-native drop-in for the SBE time propagation of rodrigomarher/HHG-Solids.
 *
 * The first block re-exports, with the same names, signatures and argument meaning, the C-linkage
 * surface that the reference's ctypes wrapper (pySWE/pyswe.py:13-35,65-98) binds, declared in the
 * reference's src/cwrapper.cpp:5-28.  Each entry cites the line it replaces.  A `SWESim` here owns
 * GPU state; `Settings` is opaque to callers exactly as in the reference.
 *
 * Differences in error behaviour: the reference throws through extern "C" or calls exit() on bad
 * input (src/wannier_tb.cpp:18, src/operator.cpp:167-168).  Here no entry point throws or exits:
 * a failure records a message, leaves the object in a defined state, and SWESim_last_error() /
 * HHG_last_error() return it (NULL when the last call on that object succeeded).
 *
 * The second block holds additions with no counterpart in the reference (precision and solver
 * selection, device-resident timing, the batched API); the reference-facing block does not
 * depend on them. */
#ifndef HHG_SWE_H
#define HHG_SWE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct SWESim SWESim;
typedef struct Settings Settings;
typedef struct SWEBatch SWEBatch;
typedef struct SWEServer SWEServer;
/* std::complex<double> / numpy complex128 layout: {re, im}. */
typedef struct hhg_cdouble {
  double re, im;
} hhg_cdouble;

/* ---- reference C ABI (src/cwrapper.cpp) -------------------------------------------------- */

/* src/cwrapper.cpp:7   SWESim* SWESim_new()                       caller owns; free with SWESim_delete */
SWESim* SWESim_new(void);
/* src/cwrapper.cpp:8   void SWESim_run_simulation(SWESim*)        propagates nt RK4 steps, records J(t) */
void SWESim_run_simulation(SWESim* swe);
/* src/cwrapper.cpp:9   void SWESim_test_files(SWESim*)            text dumps into test/ and fields/ */
void SWESim_test_files(SWESim* swe);
/* src/cwrapper.cpp:10  void SWESim_set_path_tb(SWESim*, char*)   path is copied */
void SWESim_set_path_tb(SWESim* swe, char* path_tb);
/* src/cwrapper.cpp:11  void SWESim_set_settings(SWESim*, Settings*)   borrowed: must outlive the SWESim */
void SWESim_set_settings(SWESim* swe, Settings* settings);
/* src/cwrapper.cpp:12  void SWESim_init(SWESim*)                 full setup (src/swe.cpp:49-93) */
void SWESim_init(SWESim* swe);
/* src/cwrapper.cpp:13  void SWESim_restart(SWESim*)              setup again from scratch */
void SWESim_restart(SWESim* swe);
/* src/cwrapper.cpp:14  void SWESim_get_current(SWESim*, double* t, cdouble* jx, cdouble* jy, cdouble* jz)
 * caller-allocated arrays of nt entries; t in atomic units. */
void SWESim_get_current(SWESim* swe, double* t, hhg_cdouble* jx, hhg_cdouble* jy, hhg_cdouble* jz);
/* src/cwrapper.cpp:15  void SWESim_delete(SWESim*) */
void SWESim_delete(SWESim* swe);

/* src/cwrapper.cpp:17  Settings* Settings_new()   defaults of include/settings.h:8-22 */
Settings* Settings_new(void);
/* src/cwrapper.cpp:18-20  grid sizes */
void Settings_set_nr1(Settings* s, int val);
void Settings_set_nr2(Settings* s, int val);
void Settings_set_nr3(Settings* s, int val);
/* src/cwrapper.cpp:21-25  tmax (fs), dt (fs), intensity (W/cm^2), lambda (nm), tmax_field (fs) */
void Settings_set_tmax(Settings* s, double val);
void Settings_set_dt(Settings* s, double val);
void Settings_set_intensity(Settings* s, double val);
void Settings_set_lambda(Settings* s, double val);
void Settings_set_tmax_field(Settings* s, double val);
/* src/cwrapper.cpp:26-27  polarisation vector and CEP phases, 3 doubles each */
void Settings_set_pol_vec(Settings* s, double* val);
void Settings_set_phi_vec(Settings* s, double* val);

/* ---- additions (no counterpart in the reference) ----------------------------------------- */

/* Message of the last failed call on `swe` (NULL if it succeeded); valid until the next call. */
const char* SWESim_last_error(SWESim* swe);
/* Message of the last failed call in this thread on any object (NULL if none). */
const char* HHG_last_error(void);
/* Frees a Settings made by Settings_new (the reference never frees them). */
void Settings_delete(Settings* s);
/* Number of time steps nt = (int)(tmax/dt) (src/swe.cpp:52), -1 before SWESim_init. */
int SWESim_get_nt(SWESim* swe);
/* Orbitals per k-point, -1 before SWESim_init. */
int SWESim_get_num_orb(SWESim* swe);
/* CUDA device ordinal used by the next SWESim_init (default: the current device). */
void SWESim_set_device(SWESim* swe, int device);
/* Device time in milliseconds of the last SWESim_run_simulation's propagation kernels. */
double SWESim_last_kernel_ms(SWESim* swe);
/* Device time in milliseconds of the last run's propagation kernel alone (without the J reduction). */
double SWESim_last_propagate_ms(SWESim* swe);
/* Bytes copied host->device by the last SWESim_init (model tables, twiddles, field table). */
long long SWESim_h2d_bytes(SWESim* swe);
/* Launch shape chosen for the propagation kernel; returns -1 before SWESim_init. */
int SWESim_launch_shape(SWESim* swe, int* ctas, int* threads, int* k_per_cta, long long* smem);
/* Number of kernel launches issued by the last SWESim_run_simulation. */
int SWESim_last_launches(SWESim* swe);
/* Arithmetic of the next SWESim_init: 0 = plain FP64 (default, the reference's arithmetic to
 * 1e-10); 1 = mixed: Wannier sums, field coupling and RK4 commutators in complex FP32, the state,
 * the RK4 accumulation and the current's k-sum in FP64 (error against plain FP64 reported by the
 * tests and bench). */
void SWESim_set_precision(SWESim* swe, int mode);
/* Autotuning of the tile shape (no counterpart in the reference): when on (or with the environment
 * variable HHG_AUTOTUNE=1), SWESim_init times the first steps of the pulse under a few candidate tile
 * shapes (k-points per CTA, rows per column tile) and keeps the fastest; the choice is cached per
 * device and solve shape for the rest of the process.  Results change only by the rounding of the
 * current's k-sum order.  Takes effect at the next SWESim_init. */
void SWESim_set_autotune(SWESim* swe, int on);
/* TB-file reading (no counterpart in the reference, which always transposes each block and ignores
 * the degeneracy line, src/wannier_tb.cpp:36-49,74,102): flags 0 (default) read as the reference
 * does; bit 0 divides each R block (H and positions) by its degeneracy, as Wannier90 defines the
 * file; bit 1 stores line "m n" at [m-1][n-1].  Takes effect at the next SWESim_init. */
void SWESim_set_tb_convention(SWESim* swe, int flags);
/* Solver (no counterpart in the reference's C ABI, which always drives the real-space solver):
 * 0 (default) the real-space solver of src/solver.cpp as SWESim::run_simulation drives it;
 * 1 the k-space solver of src/solver_kspace.cpp (compiled in the reference but reached by none of
 * its entry points), driven the same way step by step with J taken from the 4x4 window without a
 * Peierls phase.  The k-space solver needs nr1 == nr2.  Takes effect at the next SWESim_init. */
void SWESim_set_solver(SWESim* swe, int mode);
/* Restrict the next SWESim_init to k-grid rows m1 in [row0, row1) (row1 = -1: to the end): one
 * slab of a solve split over several GPUs.  The current stays normalised by the full grid, so the
 * currents of a partition of the rows add up to the full current. */
void SWESim_set_k_rows(SWESim* swe, int row0, int row1);
/* Put rho back to the equilibrium rho0 and clear the recorded current, keeping the setup
 * (a fresh propagation without re-running SWESim_init). */
void SWESim_reset(SWESim* swe);
/* Copy the k-space density matrix, [nr1*nr2][nw*nw] complex (W gauge), to host memory. */
void SWESim_get_rho_k(SWESim* swe, hhg_cdouble* out);
/* Fields the propagation uses: t (au, nt), E and A (au, [3][nt]). */
void SWESim_get_fields(SWESim* swe, double* t, double* E, double* A);

/* Allocation-free propagation.  No counterpart in the reference.
 *
 * For callers that cannot allocate GPU memory while they run: code whose device memory is owned
 * by another framework's pool (a PyTorch or JAX process, a simulation code with its own arena),
 * where a foreign cudaMalloc fragments that pool and a cudaFree stalls every stream on the device
 * because it synchronises the whole GPU; and latency-critical loops that cannot take those stalls.
 *
 * Does what SWESim_run_simulation does with the tables SWESim_init put on the device, but the
 * caller supplies the state and the result, both in device memory on the SWESim's device:
 *   rho_k    [nr1*nr2][nw*nw] complex, in: the starting density matrix (e.g. the equilibrium that
 *            SWESim_get_rho_k returns before any run), out: the state after nt steps;
 *   current  [3][nt] complex, out: J(t) (no record is added to SWESim_get_current's history).
 * Work is queued on `stream` (a cudaStream_t, NULL for the default stream) and the call returns
 * without waiting; it makes the SWESim's device current.
 *
 * It calls no cudaMalloc / cudaFree: the current partials go to a fixed 32 MiB array of device
 * memory that the library holds on each device it is used on until the process exits.  Solves
 * that need more (virtual CTAs x nt x 48 bytes > 32 MiB: an element-group solve on 148 CTAs up to nt of about
 * 4700; a 200x200 2-orbital solve on 400 column tiles up to about 1740) are
 * rejected with -1 and a message.  Each call looks up that array's device address (a call made
 * while the stream is being captured into a graph reuses the address of an earlier call on the same
 * device, so make one call before capturing).  All calls on a device share the array and clear it
 * at their start: calls whose work overlaps on the GPU (different streams, or different host
 * threads) corrupt each other's result.
 * The queued work also reads the SWESim's own device tables and, for solves whose kernel takes
 * precomputed inner Wannier sums (models of 6, 11 or 12 orbitals), writes the SWESim's own buffer
 * of those sums.  So synchronise `stream` before another SWESim_run_simulation or
 * SWESim_run_simulation_noalloc, SWESim_restart, SWESim_init or SWESim_delete on the same SWESim.
 * Returns 0, or -1 (message in SWESim_last_error). */
int SWESim_run_simulation_noalloc(SWESim* swe, hhg_cdouble* rho_k, hhg_cdouble* current, void* stream);

/* Batches: several initialised solves (each after SWESim_init, all on one device) propagated
 * together, each from its equilibrium, with kernels running side by side and the launch sequence
 * captured in a CUDA graph.  Every solve's current is bit for bit what it gives alone; read it with
 * SWESim_get_current.  The SWESim objects stay owned by the caller and must outlive the batch. */
SWEBatch* SWEBatch_new(void);
/* Appends a solve; returns its index in the batch, or -1. */
int SWEBatch_add(SWEBatch* batch, SWESim* swe);
/* Propagates every solve of the batch; returns 0, or -1 (message in SWEBatch_last_error). */
int SWEBatch_run(SWEBatch* batch);
/* Device time in milliseconds of the last SWEBatch_run (all solves, first launch to last copy). */
double SWEBatch_last_ms(SWEBatch* batch);
const char* SWEBatch_last_error(SWEBatch* batch);
void SWEBatch_delete(SWEBatch* batch);

/* Serving (no counterpart in the reference, whose pol_scan script runs one solve per MPI rank):
 * a request loop with continuous batching on one device.  A request is a SWESim with its TB path,
 * settings and precision set; SWESim_init is optional (the server sets it up when it admits it).
 * Requests are admitted in arrival order while their device memory (an upper bound before setup,
 * the exact figure after) fits in hbm_budget_bytes beside the running ones and fewer than max_active
 * are running; a request larger than the budget runs when nothing else does.  Running solves advance
 * together in chunks of chunk_steps RK4 steps, newly admitted ones joining at the next chunk.  When a
 * solve finishes, its current is readable with SWESim_get_current and its device memory is returned
 * (SWESim_init again to reuse the object).  Each result equals, bit for bit, what the same solve
 * gives alone.  The SWESim and its Settings must outlive the request. */
/* device: CUDA ordinal; hbm_budget_bytes 0: 80 % of the device memory free at creation. NULL on error (HHG_last_error). */
SWEServer* SWEServer_new(int device, long long hbm_budget_bytes, int max_active, int chunk_steps);
/* Queues a request; returns its ticket (>= 0), or -1 (HHG_last_error). */
long long SWEServer_submit(SWEServer* srv, SWESim* swe);
/* Blocks until the ticket completes or timeout_s passes (< 0: no limit).
 * 1 done, -1 failed (SWEServer_ticket_error), 0 timed out, -2 unknown ticket. */
int SWEServer_wait(SWEServer* srv, long long ticket, double timeout_s);
/* 0 queued, 1 setting up, 2 running, 3 done, -1 failed, -2 unknown. */
int SWEServer_status(SWEServer* srv, long long ticket);
/* Seconds since the server started: submitted, admitted, first chunk, done (0 if not yet). Returns the status. */
int SWEServer_times(SWEServer* srv, long long ticket, double* out4);
const char* SWEServer_ticket_error(SWEServer* srv, long long ticket);
/* Fills up to n of: completed, failed, chunks, GPU ms in chunks, peak running solves, peak reserved
 * bytes, budget bytes, queued, admitted, GPU ms between chunks, host ms setting up admitted solves,
 * host ms completing finished ones; returns the count written. */
int SWEServer_stats(SWEServer* srv, double* out, int n);
/* Serves every request already submitted, then stops the scheduler and frees the server. */
void SWEServer_delete(SWEServer* srv);

/* HHG spectra on the device (the post-processing of the reference's scripts/pol_scan.py:34-40, which
 * runs it in numpy; no C counterpart).  S = fftshift(fft(ifftshift(gradient(J, spacing)))) with
 * numpy's conventions, from a batched mixed-radix FFT kernel (any length). */
/* Spectra of the solve's current as SWESim_get_current returns it (x, y, z; nt values each; NULL
 * skips an axis); spacing <= 0 takes the settings' dt in fs, as pol_scan does. */
void SWESim_get_spectrum(SWESim* swe, double spacing, hhg_cdouble* sx, hhg_cdouble* sy, hhg_cdouble* sz);
/* count signals of n samples each (host arrays [count][n]); returns 0 or -1 (HHG_last_error). */
int HHG_spectrum(const hhg_cdouble* J, int n, int count, double spacing, hhg_cdouble* S);
/* I[count][nh]: |S|^2 summed over each odd harmonic order h = 1, 3, ..., 2 nh - 1, within
 * (h - 1/2, h + 1/2) on pol_scan's order axis linspace(-n pi/tmax, n pi/tmax, n) / (2 pi 300 / lambda_nm). */
int HHG_harmonic_intensities(const hhg_cdouble* S, int n, int count, double tmax_fs, double lambda_nm, int nh,
                             double* I);

/* FP64 FMA / FP32 FMA chain throughput of the current device (TFLOP/s), for roofline denominators. */
int HHG_measure_peaks(double* fp64_tflops, double* fp32_tflops);

#ifdef __cplusplus
}
#endif
#endif
