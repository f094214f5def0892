// Host-side state of one propagation (SWESim) and the helpers shared by the host sources.
#pragma once
#include <cuda_runtime.h>

#include <complex>
#include <stdexcept>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../kernels/sbe_device.h"
#include "hhg_swe.h"
#include "tb_model.hpp"

// Defaults of include/settings.h:8-22 of the reference.
struct Settings {
  int nr1 = 400, nr2 = 400, nr3 = 1;
  double tmax = 90.0;
  double dt = 10.98e-3 / 0.5;
  int nt = (int)(90.0 / (10.98e-3 / 0.5));
  double lambda_nm = 3000;
  double tmax_field = 80.0;
  double intensity_wcm2 = 5e10;
  double sx = 0.96, sy = 0.25, sz = 0.0;
  double phi_x = 0.0, phi_y = 0.0, phi_z = 0.0;
};

namespace hhg {

// A named range on the profiler timeline (NVTX; costs nothing without a profiler attached).
struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  size_t cap = 0;
  // Set: allocations are stream-ordered on this stream, from the device's memory pool (no device-wide
  // synchronisation, so a server can set solves up and retire them while others run).  The buffer
  // may then be used on other streams only after the host has synchronised with this one.
  cudaStream_t astream = nullptr;
  bool pooled = false;
  // Keeps the current allocation when it is large enough (re-initialisation reuses buffers).
  void alloc(size_t count) {
    if (count == 0) count = 1;
    if (p && count <= cap) {
      n = count;
      return;
    }
    release();
    if (astream) {
      check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&p), count * sizeof(T), astream), "cudaMallocAsync");
      pooled = true;
    } else {
      check_cuda(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
      pooled = false;
    }
    n = cap = count;
  }
  void upload(const std::vector<T>& v, cudaStream_t s) {
    alloc(v.size());
    if (!v.empty()) check_cuda(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s), "H2D");
  }
  // A pooled buffer is returned in the order of its stream: every use of it on any stream must have
  // completed (the owners release only after synchronising).
  void release() {
    if (p) {
      if (pooled)
        cudaFreeAsync(p, astream);
      else
        cudaFree(p);
    }
    p = nullptr;
    n = cap = 0;
    pooled = false;
  }
  ~DevBuf() { release(); }
};

inline double2 d2(cd z) { return make_double2(z.real(), z.imag()); }

// Records a failure for HHG_last_error (per host thread).
void set_thread_error(const std::string& msg);

}  // namespace hhg

struct SWESim {
  std::string path_tb;
  Settings* settings = nullptr;
  int device = -1;
  int req_row0 = 0, req_row1 = -1;  // k-grid row slab requested with SWESim_set_k_rows (-1: all)
  std::string err;
  bool has_err = false;
  bool ready = false;

  hhg::TBModel model;
  int N1 = 0, N2 = 0, Nk = 0, nw = 0, nw2 = 0, nt = -1;
  double lat_au[3][3] = {};
  std::vector<double> Rgrid;  // [Nk][3] Angstrom
  std::vector<int> site_of_cell;
  std::vector<double> t, E, A;
  std::vector<double> es;          // [nt][3][3]
  std::vector<int2> cell_n, win_n;
  std::vector<double2> H0, Rtab, V, Xbox, Vd, T1, T2;
  std::vector<double> Rc, x0_;  // listed cells' positions (bohr); k-space stencil offsets
  int npts_ = 0, ncw_ = 0;      // evaluation points, listed cells
  int precision = 0;  // 0 plain FP64, 1 mixed
  int solver = 0;     // 0 the real-space solver (src/solver.cpp), 1 the k-space solver (src/solver_kspace.cpp)
  bool autotune = false;  // time candidate tile shapes at SWESim_init (also HHG_AUTOTUNE=1)
  int tb_flags = 0;   // TB reading: 0 as the reference; bit 0 divide by the degeneracies, bit 1 keep the file's
                      // orbital order (line "m n" at [m-1][n-1])
  std::vector<int2> cellp;  // cell coordinates the propagation sums over (transposed for the k-space solver)
  unsigned generation = 0;  // bumped by every successful SWESim_init (batches re-capture on change)
  int nax = 0, ax_id[3] = {0, 0, 0}, nj = 0, j_id[3] = {0, 0, 0};

  cudaStream_t stream = nullptr;
  int stream_device = -1;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evm = nullptr;
  hhg::DevBuf<int2> d_cell, d_cellp, d_win;
  hhg::DevBuf<double2> d_H0, d_R, d_V, d_Q, d_Xbox, d_Vd, d_P, d_T1, d_T2, d_rho0, d_rho, d_Jpart, d_J;
  hhg::DevBuf<double2> d_pre;  // precomputed inner sums (element-group shapes with pre_chunk > 0)
  hhg::DevBuf<float2> d_Xbox32, d_Vd32, d_P32, d_T1_32, d_T2_32;
  hhg::GroupTables gtab{};
  hhg::DevBuf<double> d_es, d_A, d_Rc, d_x0;
  hhg::SolveTables tab{};
  hhg::LaunchShape shape{};
  double2* h_J = nullptr;  // pinned [3][nt] (host_J())
  size_t h_J_cap = 0;
  std::vector<hhg::cd> Jhist[3];
  float last_ms = 0.f, last_prop_ms = 0.f;
  // run()'s launch sequence (clear, propagate, reduce, copy the current out) captured once per setup
  // and replayed; rebuilt when a new setup or a new pinned buffer changes what it points at.
  cudaGraphExec_t run_graph = nullptr;
  unsigned run_graph_gen = 0;
  const double2* run_graph_hJ = nullptr;
  int graph_launches = 0;  // kernel launches inside run_graph
  void drop_run_graph() {
    if (run_graph) cudaGraphExecDestroy(run_graph);
    run_graph = nullptr;
  }
  size_t h2d_bytes = 0;
  int last_launches = 0;

  ~SWESim() { release(); }

  // Forget the previous setup but keep device buffers, stream, events and the pinned host
  // buffer for reuse: a restart then costs no cudaFree / cudaFreeHost (both synchronise).
  void invalidate() {
    drop_run_graph();
    ready = false;
    for (auto& j : Jhist) j.clear();
  }

  // Stream-ordered allocation of every device buffer on `s` (nullptr: plain cudaMalloc).
  void bind_buffers(cudaStream_t s) {
    for (auto* b : {&d_cell, &d_cellp, &d_win}) b->astream = s;
    for (auto* b : {&d_H0, &d_R, &d_V, &d_Q, &d_Xbox, &d_Vd, &d_P, &d_T1, &d_T2, &d_rho0, &d_rho, &d_Jpart, &d_J, &d_pre})
      b->astream = s;
    for (auto* b : {&d_Xbox32, &d_Vd32, &d_P32, &d_T1_32, &d_T2_32}) b->astream = s;
    for (auto* b : {&d_es, &d_A, &d_Rc, &d_x0}) b->astream = s;
  }
  void release() {
    drop_run_graph();
    d_cell.release();
    d_cellp.release();
    d_win.release();
    for (auto* b : {&d_H0, &d_R, &d_V, &d_Q, &d_Xbox, &d_Vd, &d_P, &d_T1, &d_T2, &d_rho0, &d_rho, &d_Jpart, &d_J})
      b->release();
    for (auto* b : {&d_Xbox32, &d_Vd32, &d_P32, &d_T1_32, &d_T2_32}) b->release();
    d_es.release();
    d_A.release();
    d_Rc.release();
    d_x0.release();
    d_pre.release();
    bind_buffers(nullptr);
    if (h_J) cudaFreeHost(h_J);
    h_J = nullptr;
    h_J_cap = 0;
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (evm) cudaEventDestroy(evm);
    ev0 = ev1 = evm = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
    ready = false;
    for (auto& j : Jhist) j.clear();
  }

  // Finished by a SWEServer: the device state was returned, the current record stays readable.
  bool served = false;
  // Device memory this object holds now.
  size_t device_bytes() const;
  // Upper bound of the device memory init() allocates for the current settings (parses the TB file).
  size_t footprint_estimate() const;
  // Keeps J[3][nt] as the current record (as run() does) and returns every device buffer.
  double2* host_J();
  void finish_served(const double2* J);

  void tune_tiles(int sms);
  void init();
  void run();
  void reset_state();
  void test_files();
  void write_fields_files(const std::string& dir);
};

