// SWESim / Settings: the C-linkage surface of rodrigomarher/HHG-Solids (src/cwrapper.cpp:5-28)
// over a GPU propagation.
//
// Setup (SWESim::_init, src/swe.cpp:49-93) runs on the host where it is bookkeeping and its
// rounding must follow the reference: TB parse, supercell, (int)-Cramer placement, field,
// velocity on the current window.  Everything per k-point (Wannier sums, eigensolve, rho0, the
// nt RK4 steps and the current) runs in the CUDA kernels of ../kernels.  There is no CPU path:
// without a CUDA device, SWESim_init fails with a message.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <map>
#include <mutex>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "swe_sim.hpp"

namespace hhg {
namespace refarith {
void cramer3(double** rows, double* v, double* c);
void supercell(int N1, int N2, int N3, double lat[3][3], double* R);
void time_grid(int nt, double dt_fs, double* t);
void efield(int nt, const double* t, double lambda_nm, double tmax_field_fs, double intensity, const double* s,
            const double* phi, double* E, double* A);
}  // namespace refarith
}  // namespace hhg

using hhg::cd;
using hhg::check_cuda;
using hhg::d2;
using hhg::DevBuf;

namespace {

// Setup phase timer, printed to stderr when the environment sets HHG_TRACE=1.
struct PhaseTrace {
  bool on = false;
  std::chrono::steady_clock::time_point t0, last;
  std::string line;
  PhaseTrace() {
    const char* e = std::getenv("HHG_TRACE");
    on = e && e[0] && e[0] != '0';
    t0 = last = std::chrono::steady_clock::now();
  }
  void mark(const char* name) {
    nvtxMarkA(name);
    if (!on) return;
    const auto now = std::chrono::steady_clock::now();
    char buf[96];
    snprintf(buf, sizeof buf, " %s=%.2fms", name, std::chrono::duration<double, std::milli>(now - last).count());
    line += buf;
    last = now;
  }
  ~PhaseTrace() {
    if (on)
      fprintf(stderr, "[hhg] init%s total=%.2fms\n", line.c_str(),
              std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
  }
};
constexpr double kEv2Ha = 1.0 / 27.2114;       // include/constants.h:10
constexpr double kA2Bohr = 1.0 / 0.5291772;    // include/constants.h:6

thread_local std::string g_last_error;
thread_local bool g_has_error = false;


}  // namespace

namespace {

// Placement of src/hamiltonian.cpp:8-39: site index per grid cell (first matching TB cell), -1 if none.
void place_sites(const hhg::TBModel& m, int N1, int N2, const std::vector<double>& R, std::vector<int>& site) {
  std::map<std::tuple<int, int, int>, int> first;
  for (int s = 0; s < m.nsites; ++s) {
    auto key = std::make_tuple(m.R[3 * s], m.R[3 * s + 1], m.R[3 * s + 2]);
    if (!first.count(key)) first[key] = s;
  }
  double rows[3][3];
  std::memcpy(rows, m.lattice, sizeof rows);
  double* mat[3] = {rows[0], rows[1], rows[2]};
  const int Nk = N1 * N2;
  site.assign(Nk, -1);
  for (int c = 0; c < Nk; ++c) {
    double v[3] = {R[3 * c], R[3 * c + 1], R[3 * c + 2]};
    double coef[3];
    hhg::refarith::cramer3(mat, v, coef);
    auto it = first.find(std::make_tuple((int)coef[0], (int)coef[1], (int)coef[2]));
    if (it != first.end()) site[c] = it->second;
  }
}

inline int wrapi(long x, int n) {
  long r = x % n;
  return (int)(r < 0 ? r + n : r);
}

}  // namespace

namespace {

bool autotune_env() {
  const char* e = std::getenv("HHG_AUTOTUNE");
  return e && e[0] == '1';
}

// Tile hints measured by tune_tiles, per device and solve shape: every solve of the same shape in
// this process uses the same tiles (so batches and servers stay bit-identical to solo runs).
std::mutex g_tune_mutex;
std::map<std::vector<int>, int> g_tune_cache;

}  // namespace

// Autotuner: times the propagation of the first steps under each candidate tile shape and keeps
// the fastest (element-group kernels: k-points per CTA from the largest that fits down to half of
// it; column tiles: 1 to 3 parts per column).  The state is reset to rho0 afterwards.
void SWESim::tune_tiles(int sms) {
  const std::vector<int> key = {device, shape.kernel, shape.variant, precision, nw, tab.nax, tab.nj, N1, N2,
                                tab.row1 - tab.row0, tab.kmode, tab.hermitian, tab.b1n, tab.b2n};
  int hint = -1;
  {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) hint = it->second;
  }
  char why[256] = {0};
  if (hint < 0) {
    std::vector<int> hints;
    if (shape.kernel == 3) {
      hints = {1, 2, 3};
    } else if (shape.kernel == 4) {
      hints = {16, 8};  // fragment kernel: 16 or 8 k-points per CTA
    } else if (shape.kernel == 1 || shape.kernel == 2) {
      const int B = shape.k_per_cta;
      for (int b : {B, (3 * B + 3) / 4, (2 * B + 2) / 3, (B + 1) / 2}) hints.push_back(b);
    }
    const int steps = std::min(nt, 128);
    DevBuf<double2> scratch;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
    float best_ms = 0.f;
    std::vector<std::pair<int, int>> seen;  // (k_per_cta, threads) already timed
    for (int h : hints) {
      hhg::LaunchShape cand{};
      if (!hhg::plan_propagate(tab, precision, sms, &cand, why, sizeof why, h)) continue;
      bool dup = false;
      for (auto& p : seen) dup = dup || (p.first == cand.k_per_cta && p.second == cand.threads);
      if (dup) continue;
      seen.emplace_back(cand.k_per_cta, cand.threads);
      scratch.alloc((size_t)cand.vctas * nt * 3);
      hhg::SolveTables tt = tab;
      tt.step1 = steps;
      float ms = 0.f;
      for (int rep = 0; rep < 3; ++rep) {
        check_cuda(cudaMemcpyAsync(d_rho.p, d_rho0.p, sizeof(double2) * (size_t)Nk * nw2, cudaMemcpyDeviceToDevice,
                                   stream), "D2D");
        check_cuda(cudaEventRecord(e0, stream), "event");
        hhg::launch_propagate_steps(tt, gtab, cand, d_rho.p, scratch.p, stream);
        check_cuda(cudaEventRecord(e1, stream), "event");
        check_cuda(cudaEventSynchronize(e1), "autotune");
        float m = 0.f;
        check_cuda(cudaEventElapsedTime(&m, e0, e1), "event time");
        if (rep > 0) ms = rep == 1 ? m : std::min(ms, m);  // first run warms up
      }
      check_cuda(cudaGetLastError(), "autotune launch");
      if (hint < 0 || ms < best_ms) {
        best_ms = ms;
        hint = h;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (hint < 0) hint = 0;
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    g_tune_cache.emplace(key, hint);  // the first measurement of a shape wins
    hint = g_tune_cache[key];
  }
  if (hint > 0) {
    hhg::LaunchShape tuned{};
    if (hhg::plan_propagate(tab, precision, sms, &tuned, why, sizeof why, hint)) shape = tuned;
  }
  d_Jpart.alloc((size_t)shape.vctas * nt * 3);
  check_cuda(cudaMemcpyAsync(d_rho.p, d_rho0.p, sizeof(double2) * (size_t)Nk * nw2, cudaMemcpyDeviceToDevice, stream),
             "D2D");
  check_cuda(cudaStreamSynchronize(stream), "autotune");
}

void SWESim::init() {
  hhg::TraceRange range("hhg SWESim_init");
  PhaseTrace trace;
  invalidate();
  served = false;
  if (!settings) throw std::runtime_error("SWESim_init: settings not set (call SWESim_set_settings first)");
  if (path_tb.empty()) throw std::runtime_error("SWESim_init: TB path not set (call SWESim_set_path_tb first)");
  model = hhg::parse_tb(path_tb);
  // Optional Wannier90 reading (off by default, where the model is read exactly as the reference
  // reads it, src/wannier_tb.cpp:36-49,74,102): the file's orbital order and the degeneracy weights.
  if (tb_flags & 2)
    for (int st = 0; st < model.nsites; ++st) {
      auto transpose = [&](std::vector<cd>& v) {
        for (int i = 0; i < model.nw; ++i)
          for (int j = i + 1; j < model.nw; ++j)
            std::swap(v[((size_t)st * model.nw + i) * model.nw + j], v[((size_t)st * model.nw + j) * model.nw + i]);
      };
      transpose(model.hop);
      for (auto& b : model.bc) transpose(b);
    }
  if (tb_flags & 1)
    for (int st = 0; st < model.nsites; ++st) {
      const int dg = model.degeneracy[st];
      if (dg <= 0) throw std::runtime_error("SWESim_init: degeneracy " + std::to_string(dg) + " in the TB file");
      const size_t nwsq = (size_t)model.nw * model.nw;
      for (size_t o = 0; o < nwsq; ++o) {
        model.hop[st * nwsq + o] /= (double)dg;
        for (auto& b : model.bc) b[st * nwsq + o] /= (double)dg;
      }
    }
  trace.mark("parse");
  Settings& s = *settings;
  nt = (int)(s.tmax / s.dt);
  s.nt = nt;
  N1 = s.nr1;
  N2 = s.nr2;
  nw = model.nw;
  nw2 = nw * nw;
  if (s.nr3 != 1) throw std::runtime_error("SWESim_init: only 2D grids (nr3 = 1) are supported");
  if (N1 < 4 || N2 < 4 || (N1 % 2) || (N2 % 2))
    throw std::runtime_error(
        "SWESim_init: nr1 and nr2 must be even and >= 4 (odd sizes shift the reference's fftshift/ifftshift pair "
        "by one cell; sizes below 4 put its 4x4 current window outside the grid)");
  if (nt < 2) throw std::runtime_error("SWESim_init: tmax/dt must give at least 2 time steps");
  if (solver == 1 && N1 != N2)
    throw std::runtime_error(
        "SWESim_init: the k-space solver needs nr1 == nr2 (its interpolation reads the grid as data[yi*nr1 + xi] "
        "with yi along the second axis, src/interpolation.cpp:36-37, which scrambles a non-square grid)");
  if (nw > hhg::kMaxOrb) throw std::runtime_error("SWESim_init: more than 16 orbitals is not supported");
  if ((long)N1 * N2 > (1L << 30)) throw std::runtime_error("SWESim_init: grid too large");
  Nk = N1 * N2;

  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    throw std::runtime_error("SWESim_init: no CUDA device (this library has no CPU path)");
  if (device < 0) check_cuda(cudaGetDevice(&device), "cudaGetDevice");
  if (stream && device != stream_device) release();  // device changed: start over
  check_cuda(cudaSetDevice(device), "cudaSetDevice");
  if (!stream) {
    // Highest priority: a solve set up while a server runs others gets its table and rho0 kernels
    // onto the SMs as soon as blocks of the running launches retire, instead of behind them.
    int least = 0, greatest = 0;
    check_cuda(cudaDeviceGetStreamPriorityRange(&least, &greatest), "cudaDeviceGetStreamPriorityRange");
    check_cuda(cudaStreamCreateWithPriority(&stream, cudaStreamNonBlocking, greatest), "cudaStreamCreate");
    // Device buffers come from the device's stream-ordered pool, which keeps freed memory for reuse.
    cudaMemPool_t pool = nullptr;
    check_cuda(cudaDeviceGetDefaultMemPool(&pool, device), "cudaDeviceGetDefaultMemPool");
    uint64_t keep = UINT64_MAX;
    check_cuda(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
    bind_buffers(stream);
    check_cuda(cudaEventCreate(&ev0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&ev1), "cudaEventCreate");
    check_cuda(cudaEventCreate(&evm), "cudaEventCreate");
    stream_device = device;
  }
  trace.mark("cuda_objects");

  // Supercell and placement (src/grid.cpp:64-111, src/hamiltonian.cpp:8-39, src/berry_connection.cpp:7-50).
  Rgrid.assign((size_t)Nk * 3, 0.0);
  hhg::refarith::supercell(N1, N2, 1, model.lattice, Rgrid.data());
  place_sites(model, N1, N2, Rgrid, site_of_cell);
  trace.mark("placement");
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) lat_au[a][b] = model.lattice[a][b] * kA2Bohr;

  // Fields (src/efield.cpp:30-50) and the per-step table (src/solver.cpp:109-148, src/swe.cpp:192-196).
  t.assign(nt, 0.0);
  E.assign((size_t)3 * nt, 0.0);
  A.assign((size_t)3 * nt, 0.0);
  hhg::refarith::time_grid(nt, s.dt, t.data());
  const double pol[3] = {s.sx, s.sy, s.sz}, phi[3] = {s.phi_x, s.phi_y, s.phi_z};
  hhg::refarith::efield(nt, t.data(), s.lambda_nm, s.tmax_field, s.intensity_wcm2, pol, phi, E.data(), A.data());
  nax = 0;
  for (int a = 0; a < 3; ++a)
    if (pol[a] != 0.0) ax_id[nax++] = a;
  es.assign((size_t)nt * 9, 0.0);
  for (int ti = 0; ti < nt; ++ti) {
    double* p = es.data() + (size_t)ti * 9;
    for (int a = 0; a < 3; ++a) {
      const double* Ea = E.data() + (size_t)a * nt;
      if (ti < nt - 1) {
        p[0 * 3 + a] = Ea[ti];
        p[1 * 3 + a] = 0.5 * Ea[ti] + 0.5 * Ea[ti + 1];
        p[2 * 3 + a] = Ea[ti + 1];
      } else {
        p[0 * 3 + a] = p[1 * 3 + a] = p[2 * 3 + a] = Ea[nt - 1];
      }
    }
  }

  trace.mark("fields");
  // Support cells: placed cells whose H0 or field-coupled r block is non-zero (zero blocks add exact zeros).
  cell_n.clear();
  H0.clear();
  std::vector<std::vector<double2>> Rax(nax);
  for (int c = 0; c < Nk; ++c) {
    const int st = site_of_cell[c];
    if (st < 0) continue;
    bool nz = false;
    for (int o = 0; o < nw2 && !nz; ++o) {
      nz = model.hop[(size_t)st * nw2 + o] != cd(0, 0);
      for (int a = 0; a < nax && !nz; ++a) nz = model.bc[ax_id[a]][(size_t)st * nw2 + o] != cd(0, 0);
    }
    if (!nz) continue;
    cell_n.push_back(make_int2(c / N2 - N1 / 2, c % N2 - N2 / 2));
    for (int o = 0; o < nw2; ++o) {
      H0.push_back(d2(model.hop[(size_t)st * nw2 + o] * kEv2Ha));
      for (int a = 0; a < nax; ++a) Rax[a].push_back(d2(-model.bc[ax_id[a]][(size_t)st * nw2 + o] * kA2Bohr));
    }
  }
  const int ncell = (int)cell_n.size();
  Rtab.clear();
  for (int a = 0; a < nax; ++a) Rtab.insert(Rtab.end(), Rax[a].begin(), Rax[a].end());

  // Velocity on the 4x4 window (src/velocity.cpp:41-115, evaluated in SI with the to-au factor 1.0 of
  // include/constants.h:13): v_a(n) = i (R_a(n) H(n) - sum_n' [r(n') H(n - n') - H(n') r(n - n')]),
  // with the cyclic convolution of the reference's FFT product taken directly.
  auto cell_of = [&](int n1, int n2) { return wrapi((long)n1 + N1 / 2, N1) * N2 + wrapi((long)n2 + N2 / 2, N2); };
  std::vector<int> placed;
  for (int c = 0; c < Nk; ++c)
    if (site_of_cell[c] >= 0) placed.push_back(c);
  std::vector<cd> vw((size_t)3 * hhg::kWindow * nw2, cd(0, 0));
  bool r_nonzero_of[3];  // an axis without position elements has no convolution term
  for (int a = 0; a < 3; ++a) {
    r_nonzero_of[a] = false;
    for (const cd& z : model.bc[a]) r_nonzero_of[a] = r_nonzero_of[a] || z != cd(0, 0);
  }
  // One task per (axis, window cell), each with its own sum in a fixed order: the tasks run on host
  // threads and give the same bits on any number of them.
  auto window_cell = [&](int a, int w) {
      const bool r_nonzero = r_nonzero_of[a];
      const int n1 = w / 4 - 2, n2 = w % 4 - 2;
      const int c = cell_of(n1, n2);
      std::vector<cd> acc(nw2, cd(0, 0));
      for (int q : placed) {
        if (!r_nonzero) break;
        const int q1 = q / N2 - N1 / 2, q2 = q % N2 - N2 / 2;
        const int d = cell_of(n1 - q1, n2 - q2);
        const int sd = site_of_cell[d];
        if (sd < 0) continue;
        const int sq = site_of_cell[q];
        const cd* rq = model.bc[a].data() + (size_t)sq * nw2;
        const cd* Hq = model.hop.data() + (size_t)sq * nw2;
        const cd* rd = model.bc[a].data() + (size_t)sd * nw2;
        const cd* Hd = model.hop.data() + (size_t)sd * nw2;
        // The products written out: the same arithmetic as std::complex's operator* on finite
        // values, without its out-of-line NaN handling.
        auto mul = [](cd x, cd y) { return cd(x.real() * y.real() - x.imag() * y.imag(), x.real() * y.imag() + x.imag() * y.real()); };
        for (int i = 0; i < nw; ++i)
          for (int j = 0; j < nw; ++j) {
            cd sum(0, 0);
            for (int k = 0; k < nw; ++k) sum += mul(-rq[i * nw + k], Hd[k * nw + j]) - mul(Hq[i * nw + k], -rd[k * nw + j]);
            acc[i * nw + j] += sum;
          }
      }
      const int sc = site_of_cell[c];
      const double Ra = Rgrid[3 * (size_t)c + a];
      for (int o = 0; o < nw2; ++o) {
        const cd h = sc >= 0 ? model.hop[(size_t)sc * nw2 + o] : cd(0, 0);
        vw[((size_t)a * hhg::kWindow + w) * nw2 + o] = cd(0, 1) * (Ra * h - acc[o]);
      }
  };
  {
    const int ntask = 3 * hhg::kWindow;
    // (threads only where the sums are large: for small models starting them costs more than the sums)
    const double work = (double)ntask * (double)placed.size() * nw * nw * nw;
    const int nthr = work < 2e5 ? 1 : std::max(1, std::min<int>(ntask, (int)std::thread::hardware_concurrency()));
    std::atomic<int> next{0};
    auto worker = [&] {
      for (int k = next++; k < ntask; k = next++) window_cell(k / hhg::kWindow, k % hhg::kWindow);
    };
    std::vector<std::thread> pool;
    for (int i = 1; i < nthr; ++i) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
  }
  nj = 0;
  for (int a = 0; a < 3; ++a) {
    bool nz = false;
    for (size_t o = 0; o < (size_t)hhg::kWindow * nw2 && !nz; ++o) nz = vw[(size_t)a * hhg::kWindow * nw2 + o] != cd(0, 0);
    if (nz) j_id[nj++] = a;  // otherwise J_a is exactly zero, as in the reference
  }
  // Window cells with a non-zero velocity on some current axis (sparse form) ...
  win_n.clear();
  V.clear();
  std::vector<int> win_w;
  for (int w = 0; w < hhg::kWindow; ++w) {
    bool nz = false;
    for (int a = 0; a < nj && !nz; ++a)
      for (int o = 0; o < nw2 && !nz; ++o) nz = vw[((size_t)j_id[a] * hhg::kWindow + w) * nw2 + o] != cd(0, 0);
    if (nz) {
      win_w.push_back(w);
      win_n.push_back(make_int2(w / 4 - 2, w % 4 - 2));
    }
  }
  for (int a = 0; a < nj; ++a)
    for (int w : win_w)
      for (int o = 0; o < nw2; ++o) V.push_back(d2(vw[((size_t)j_id[a] * hhg::kWindow + w) * nw2 + o]));
  // ... and dense over the 4x4 window (separable form).
  Vd.assign((size_t)nj * hhg::kWindow * nw2, make_double2(0.0, 0.0));
  for (int a = 0; a < nj; ++a)
    for (int w = 0; w < hhg::kWindow; ++w)
      for (int o = 0; o < nw2; ++o) Vd[((size_t)a * hhg::kWindow + w) * nw2 + o] = d2(vw[((size_t)j_id[a] * hhg::kWindow + w) * nw2 + o]);
  const int nwin = (int)win_n.size();

  // Coordinates the propagation sums over.  The k-space solver interpolates H_eff(k - A) from the
  // grid read as data[yi*N + xi] with xi along the first fractional coordinate (src/interpolation.cpp:
  // 17-43): on a square grid that evaluates the model with its cells transposed, n -> (n2, n1).
  cellp = cell_n;
  if (solver == 1)
    for (auto& n : cellp) std::swap(n.x, n.y);
  const int ncw = ncell + nwin;
  // Per-cell factors of every evaluation point.  Real-space solver: the Peierls phase
  // e^{i A(t_i).R_c} of step i (src/swe.cpp:225-233), R_c the cell's supercell position in bohr.
  // k-space solver: the bicubic interpolation at k - A_s (src/solver_kspace.cpp:286-305) acts on the
  // cell (n1', n2') as the factor Cx(n1') Cy(n2'), Cx(q) = sum_a w_a(tx) e^{-2 pi i (ox + a) q / N}
  // over the Catmull-Rom weights w of the stencil offsets a = -1..2 (src/interpolation.cpp:8-14),
  // where ox + tx = -N u_A and u_A is the first fractional coordinate of A_s (Cramer solve against
  // the reciprocal vectors, src/vec3_util.cpp:13-36); Cy likewise from the second.  Points 2i, 2i+1,
  // 2i+2 are A(t_i), the mean of A(t_i) and A(t_i+1), A(t_i+1) (clamped at the last step).
  const int npts = solver == 1 ? 2 * nt + 1 : nt;
  int np_ = 2;
  for (int c = 0; c < ncell; ++c) np_ = std::max(np_, std::max(std::abs(cellp[c].x), std::abs(cellp[c].y)));
  std::vector<double> x0;  // k-space solver: [npts][2] stencil offsets -N u_d(A_j)
  if (solver == 1) {
    double bA[3][3];  // reciprocal vectors (1/Angstrom, src/grid.cpp:27-46), then in au
    {
      const double(*a)[3] = model.lattice;
      double cr[3][3];
      for (int r = 0; r < 3; ++r) {
        const int p = (r + 1) % 3, q = (r + 2) % 3;
        cr[r][0] = a[p][1] * a[q][2] - a[p][2] * a[q][1];
        cr[r][1] = a[p][2] * a[q][0] - a[p][0] * a[q][2];
        cr[r][2] = a[p][0] * a[q][1] - a[p][1] * a[q][0];
      }
      const double vol = a[0][0] * cr[0][0] + a[0][1] * cr[0][1] + a[0][2] * cr[0][2];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) bA[r][c] = 2.0 * M_PI / vol * cr[r][c] / kA2Bohr;
    }
    double* brows[3] = {bA[0], bA[1], bA[2]};
    x0.assign((size_t)npts * 2, 0.0);
    const int N = N1;
    for (int j = 0; j < npts; ++j) {
      const int i = std::min(j / 2, nt - 1);
      double Aj[3];
      for (int a = 0; a < 3; ++a) {
        const double* Aa = A.data() + (size_t)a * nt;
        if (j == 2 * nt || (j % 2 == 1 && i == nt - 1))
          Aj[a] = Aa[nt - 1];
        else if (j % 2 == 1)
          Aj[a] = 0.5 * Aa[i] + 0.5 * Aa[i + 1];
        else
          Aj[a] = Aa[j / 2];
      }
      double crd[3];
      hhg::refarith::cramer3(brows, Aj, crd);
      for (int d = 0; d < 2; ++d) x0[(size_t)2 * j + d] = -crd[d] * (double)N;  // stencil offset o + t
    }
  }
  // (The tables themselves are built on the device below, from A, the cell positions Rc and the
  // stencil offsets x0.)
  Rc.assign((size_t)ncw * 3, 0.0);
  for (int c = 0; c < ncw; ++c) {
    const int2 n = c < ncell ? cell_n[c] : win_n[c - ncell];
    const int cc = cell_of(n.x, n.y);
    for (int a = 0; a < 3; ++a) Rc[3 * c + a] = Rgrid[3 * (size_t)cc + a] * kA2Bohr;
  }

  // Dense bounding box of the support cells for the separable Wannier sum.
  int b1lo = 0, b1hi = 0, b2lo = 0, b2hi = 0;
  for (int c = 0; c < ncell; ++c) {
    if (c == 0 || cellp[c].x < b1lo) b1lo = cellp[c].x;
    if (c == 0 || cellp[c].x > b1hi) b1hi = cellp[c].x;
    if (c == 0 || cellp[c].y < b2lo) b2lo = cellp[c].y;
    if (c == 0 || cellp[c].y > b2hi) b2hi = cellp[c].y;
  }
  const int b1n = ncell ? b1hi - b1lo + 1 : 1, b2n = ncell ? b2hi - b2lo + 1 : 1;
  // Box table [1 + nax][b1n][b2n][nw2]: H0, then the field-coupled r of each active axis.
  Xbox.assign((size_t)(1 + nax) * b1n * b2n * nw2, make_double2(0.0, 0.0));
  for (int c = 0; c < ncell; ++c) {
    const size_t box = (size_t)(cellp[c].x - b1lo) * b2n + (cellp[c].y - b2lo);
    for (int o = 0; o < nw2; ++o) {
      Xbox[box * nw2 + o] = H0[(size_t)c * nw2 + o];
      for (int a = 0; a < nax; ++a)
        Xbox[((size_t)(1 + a) * b1n * b2n + box) * nw2 + o] = Rtab[((size_t)a * ncell + c) * nw2 + o];
    }
  }
  npts_ = npts;
  ncw_ = ncw;
  x0_ = std::move(x0);
  tab.nwin = nwin;
  tab.b1lo = b1lo;
  tab.b1n = b1n;
  tab.b2lo = b2lo;
  tab.b2n = b2n;
  tab.np = np_;

  // Hermitian symmetry of the placed operators on the grid: block(-n) == block(n)^+ for every cell.
  // It fails when the grid is smaller than the model's R range or a misplacement is one-sided; the
  // kernel then forms the full HX - XH instead of HX - (HX)^+.
  bool herm = true;
  for (int c = 0; c < Nk && herm; ++c) {
    const int n1 = c / N2 - N1 / 2, n2 = c % N2 - N2 / 2;
    const int st = site_of_cell[c], sm = site_of_cell[cell_of(-n1, -n2)];
    if (st < 0 && sm < 0) continue;
    auto blk = [&](const std::vector<cd>& v, int s, int i, int j) { return s < 0 ? cd(0, 0) : v[(size_t)s * nw2 + i * nw + j]; };
    for (int i = 0; i < nw && herm; ++i)
      for (int j = 0; j < nw && herm; ++j) {
        herm = blk(model.hop, st, i, j) == std::conj(blk(model.hop, sm, j, i));
        for (int a = 0; a < nax && herm; ++a)
          herm = blk(model.bc[ax_id[a]], st, i, j) == std::conj(blk(model.bc[ax_id[a]], sm, j, i));
      }
  }

  T1.resize(N1);
  T2.resize(N2);
  for (int m = 0; m < N1; ++m) {
    const double ang = 2.0 * M_PI * (double)m / (double)N1;
    T1[m] = make_double2(std::cos(ang), -std::sin(ang));
  }
  for (int m = 0; m < N2; ++m) {
    const double ang = 2.0 * M_PI * (double)m / (double)N2;
    T2[m] = make_double2(std::cos(ang), -std::sin(ang));
  }

  trace.mark("tables");
  // Device tables.
  h2d_bytes = sizeof(int2) * (cell_n.size() + cellp.size() + win_n.size()) +
              sizeof(double2) * (H0.size() + Rtab.size() + V.size() + Xbox.size() + Vd.size() + T1.size() + T2.size()) +
              sizeof(double) * (es.size() + A.size() + Rc.size() + x0_.size());
  d_cell.upload(cell_n, stream);
  d_cellp.upload(cellp, stream);
  d_win.upload(win_n, stream);
  d_H0.upload(H0, stream);
  d_R.upload(Rtab, stream);
  d_V.upload(V, stream);
  // Factor tables of every evaluation point, built on the device.
  {
    const int npw = 2 * tab.np + 1;
    d_A.upload(A, stream);
    d_Rc.upload(Rc, stream);
    d_Q.alloc((size_t)npts_ * ncw_);
    d_P.alloc((size_t)npts_ * 2 * npw);
    if (solver == 1) {
      d_x0.upload(x0_, stream);
      hhg::launch_interp_tables(d_x0.p, N1, tab.np, npts_, d_cellp.p, (int)cellp.size(), ncw_, d_P.p, d_Q.p, stream);
    } else {
      hhg::launch_peierls_tables(d_A.p, d_Rc.p, lat_au, nt, ncw_, tab.np, d_Q.p, d_P.p, stream);
    }
    check_cuda(cudaGetLastError(), "table kernels");
  }
  d_Xbox.upload(Xbox, stream);
  d_Vd.upload(Vd, stream);
  d_T1.upload(T1, stream);
  d_T2.upload(T2, stream);
  d_es.upload(es, stream);
  if (precision == 1) {
    // FP32 copies for the mixed form (Wannier sums and commutators in complex FP32).
    auto to32 = [](const std::vector<double2>& v) {
      std::vector<float2> o(v.size());
      for (size_t q = 0; q < v.size(); ++q) o[q] = make_float2((float)v[q].x, (float)v[q].y);
      return o;
    };
    d_Xbox32.upload(to32(Xbox), stream);
    d_Vd32.upload(to32(Vd), stream);
    d_P32.alloc(d_P.n);
    hhg::launch_to_float2(d_P.p, d_P.n, d_P32.p, stream);
    d_T1_32.upload(to32(T1), stream);
    d_T2_32.upload(to32(T2), stream);
    h2d_bytes += sizeof(float2) * (Xbox.size() + Vd.size() + T1.size() + T2.size());
    check_cuda(cudaStreamSynchronize(stream), "H2D");  // the host vectors above are temporaries
  }
  gtab = hhg::GroupTables{d_Xbox.p, d_Vd.p, d_P.p, d_T1.p, d_T2.p,
                          d_Xbox32.p, d_Vd32.p, d_P32.p, d_T1_32.p, d_T2_32.p, nullptr};
  d_rho0.alloc((size_t)Nk * nw2);
  d_rho.alloc((size_t)Nk * nw2);
  d_J.alloc((size_t)3 * nt);
  const int row0 = req_row0, row1 = req_row1 < 0 ? N1 : req_row1;
  if (row0 < 0 || row1 > N1 || row0 >= row1)
    throw std::runtime_error("SWESim_init: k-row slab [" + std::to_string(row0) + ", " + std::to_string(row1) +
                             ") is not inside the grid's " + std::to_string(N1) + " rows");
  tab.row0 = row0;
  tab.row1 = row1;
  tab.nw = nw;
  tab.nw2 = nw2;
  tab.N1 = N1;
  tab.N2 = N2;
  tab.Nk = Nk;
  tab.nt = nt;
  tab.step0 = 0;
  tab.step1 = nt;
  tab.hermitian = herm ? 1 : 0;
  tab.dt = t[1] - t[0];
  tab.nax = nax;
  tab.nj = nj;
  for (int a = 0; a < 3; ++a) {
    tab.ax_id[a] = ax_id[a];
    tab.j_id[a] = j_id[a];
  }
  tab.es = d_es.p;
  tab.ncell = ncell;
  tab.cell_n = d_cellp.p;
  tab.kmode = solver;
  tab.H0 = d_H0.p;
  tab.R = d_R.p;
  tab.win_n = d_win.p;
  tab.V = d_V.p;
  tab.Q = d_Q.p;
  tab.T1 = d_T1.p;
  tab.T2 = d_T2.p;

  int sms = 0;
  check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
  char why[256] = {0};
  trace.mark("upload");
  if (!hhg::plan_propagate(tab, precision, sms, &shape, why, sizeof why)) throw std::runtime_error(std::string("SWESim_init: ") + why);
  trace.mark("plan");
  d_Jpart.alloc((size_t)shape.vctas * nt * 3);
  // Scratch of the precomputed inner sums (independent of the tile shape, so autotuning keeps it).
  gtab.pre = nullptr;
  if (shape.pre_bytes > 0) {
    d_pre.alloc((shape.pre_bytes + sizeof(double2) - 1) / sizeof(double2));
    gtab.pre = d_pre.p;
  }

  // Equilibrium density matrix (src/swe.cpp:82-90) on the GPU.
  {
    hhg::SolveTables t0 = tab;  // the model's own cell coordinates
    t0.cell_n = d_cell.p;
    hhg::launch_rho0_fp64(t0, d_rho0.p, stream);
  }
  check_cuda(cudaGetLastError(), "rho0 launch");
  check_cuda(cudaMemcpyAsync(d_rho.p, d_rho0.p, sizeof(double2) * (size_t)Nk * nw2, cudaMemcpyDeviceToDevice, stream),
             "D2D");
  check_cuda(cudaStreamSynchronize(stream), "init");
  trace.mark("rho0");
  if (autotune || autotune_env()) {
    tune_tiles(sms);
    trace.mark("autotune");
  }
  ready = true;
  ++generation;
}

size_t SWESim::device_bytes() const {
  size_t b = (d_cell.cap + d_cellp.cap + d_win.cap) * sizeof(int2) +
             (d_es.cap + d_A.cap + d_Rc.cap + d_x0.cap) * sizeof(double);
  for (const auto* x : {&d_H0, &d_R, &d_V, &d_Q, &d_Xbox, &d_Vd, &d_P, &d_T1, &d_T2, &d_rho0, &d_rho, &d_Jpart, &d_J,
                        &d_pre})
    b += x->cap * sizeof(double2);
  for (const auto* x : {&d_Xbox32, &d_Vd32, &d_P32, &d_T1_32, &d_T2_32}) b += x->cap * sizeof(float2);
  return b;
}

size_t SWESim::footprint_estimate() const {
  if (!settings) throw std::runtime_error("SWESim: settings not set (call SWESim_set_settings first)");
  if (path_tb.empty()) throw std::runtime_error("SWESim: TB path not set (call SWESim_set_path_tb first)");
  const hhg::TBModel m = hhg::parse_tb(path_tb);
  const Settings& s = *settings;
  const size_t nt_ = (size_t)std::max(2, (int)(s.tmax / s.dt));
  const size_t N1_ = (size_t)std::max(1, s.nr1), N2_ = (size_t)std::max(1, s.nr2);
  const size_t w2 = (size_t)m.nw * m.nw, ns = (size_t)std::max(1, m.nsites);
  int np_ = 2;
  for (int c = 0; c < m.nsites; ++c) np_ = std::max(np_, std::max(std::abs(m.R[3 * c]), std::abs(m.R[3 * c + 1])));
  const size_t box = (size_t)(2 * np_ + 1) * (2 * np_ + 1);
  int dev = device, sms = 148;
  if (dev < 0) cudaGetDevice(&dev);
  if (dev >= 0) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t c16 = sizeof(double2);
  size_t b = 2 * N1_ * N2_ * w2 * c16;                            // rho, rho0
  b += 4 * (size_t)sms * nt_ * 3 * c16;                           // current partials (up to 4 CTAs per SM)
  b += nt_ * (3 * c16 + 9 * sizeof(double));                      // J, field table
  b += nt_ * (ns + hhg::kWindow) * c16;                           // Peierls phases of the listed cells
  b += nt_ * 2 * (2 * np_ + 1) * c16 * 3 / 2;                     // P, FP64 and FP32
  b += (4 * box + 4 * ns + 6 * hhg::kWindow) * w2 * c16 * 3 / 2;  // cell tables, both precisions
  b += (N1_ + N2_) * c16 * 3 / 2 + (size_t(1) << 20);
  // Precomputed inner sums: 64 steps (2 x 64 + 1 points for the k-space solver) x N2 columns x (box
  // rows of H0 and r_a, window rows) x nw2.
  const size_t pre_pts = solver == 1 ? 2 * std::min<size_t>(64, nt_) + 1 : std::min<size_t>(64, nt_);
  b += pre_pts * N2_ * ((size_t)4 * (np_ + 1) + 12) * w2 * c16;
  return b;
}

// The pinned [3][nt] host copy of the current, allocated at the first run rather than at setup: a
// solve set up by a server while others run never needs it (page-locking allocations can wait for
// the device).
double2* SWESim::host_J() {
  if (!h_J || h_J_cap < (size_t)3 * nt) {
    if (h_J) cudaFreeHost(h_J);
    h_J = nullptr;
    check_cuda(cudaMallocHost(&h_J, sizeof(double2) * 3 * (size_t)nt), "cudaMallocHost");
    h_J_cap = (size_t)3 * nt;
  }
  return h_J;
}

void SWESim::finish_served(const double2* J) {
  std::vector<cd> keep[3];
  for (int a = 0; a < 3; ++a)
    for (int ti = 0; ti < nt; ++ti) keep[a].push_back(cd(J[(size_t)a * nt + ti].x, J[(size_t)a * nt + ti].y));
  release();
  for (int a = 0; a < 3; ++a) Jhist[a] = std::move(keep[a]);
  served = true;
}

void SWESim::reset_state() {
  if (!ready) throw std::runtime_error("SWESim_reset: SWESim_init has not succeeded");
  check_cuda(cudaMemcpyAsync(d_rho.p, d_rho0.p, sizeof(double2) * (size_t)Nk * nw2, cudaMemcpyDeviceToDevice, stream),
             "D2D");
  check_cuda(cudaStreamSynchronize(stream), "reset");
  for (auto& j : Jhist) j.clear();
}

namespace {
bool run_graphs_enabled() {
  const char* e = std::getenv("HHG_GRAPH");  // HHG_GRAPH=0: launch the sequence directly (measurements)
  return !(e && e[0] == '0');
}
}  // namespace

void SWESim::run() {
  hhg::TraceRange range("hhg SWESim_run_simulation");
  if (!ready) throw std::runtime_error("SWESim_run_simulation: SWESim_init has not succeeded");
  check_cuda(cudaSetDevice(device), "cudaSetDevice");
  double2* hJ = host_J();
  // The time loop (src/swe.cpp:183-223) as one launch sequence: clear the current partials, the
  // propagation launches (a pair per chunk of steps for precomputed-sum shapes), the reduction and the
  // copy of J to pinned host memory.  It is captured into a CUDA graph at the first run of a setup and
  // replayed afterwards, so a run costs one graph launch.
  auto enqueue = [&] {
    // (external event records: inside a captured graph they record when the graph runs)
    check_cuda(cudaMemsetAsync(d_Jpart.p, 0, sizeof(double2) * d_Jpart.n, stream), "memset");
    check_cuda(hhg::record_event(ev0, stream), "event");
    const int n = hhg::launch_propagate(tab, gtab, shape, d_rho.p, d_Jpart.p, d_J.p, stream, evm);
    check_cuda(cudaGetLastError(), "propagate launch");
    check_cuda(hhg::record_event(ev1, stream), "event");
    check_cuda(cudaMemcpyAsync(hJ, d_J.p, sizeof(double2) * 3 * (size_t)nt, cudaMemcpyDeviceToHost, stream), "D2H");
    return n;
  };
  if (!run_graphs_enabled()) {
    drop_run_graph();
    last_launches = enqueue();
  } else {
    if (run_graph && (run_graph_gen != generation || run_graph_hJ != hJ)) drop_run_graph();
    if (!run_graph) {
      cudaGraph_t g = nullptr;
      check_cuda(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
      int n = 0;
      try {
        n = enqueue();
      } catch (...) {
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      check_cuda(cudaStreamEndCapture(stream, &g), "end capture");
      const cudaError_t e = cudaGraphInstantiate(&run_graph, g, 0);
      cudaGraphDestroy(g);
      check_cuda(e, "graph instantiate");
      run_graph_gen = generation;
      run_graph_hJ = hJ;
      graph_launches = n;
    }
    check_cuda(cudaGraphLaunch(run_graph, stream), "graph launch");
    last_launches = graph_launches;
  }
  check_cuda(cudaStreamSynchronize(stream), "run_simulation");
  check_cuda(cudaEventElapsedTime(&last_ms, ev0, ev1), "event time");
  check_cuda(cudaEventElapsedTime(&last_prop_ms, ev0, evm), "event time");
  // The reference appends one sample per step to each Observable (src/observable.cpp:29);
  // SWESim_get_current returns the first nt of them.
  for (int a = 0; a < 3; ++a)
    for (int ti = 0; ti < nt; ++ti) Jhist[a].push_back(cd(hJ[(size_t)a * nt + ti].x, hJ[(size_t)a * nt + ti].y));
}

namespace {

void write_matrix_field(const std::string& path, const char* unit, int npts, int nw2,
                        const std::function<cd(int, int)>& get) {
  std::ofstream f(path);
  if (!f) return;
  f << unit << "\n";
  for (int i = 0; i < npts; ++i)
    for (int o = 0; o < nw2; ++o) {
      const cd z = get(i, o);
      f << i << " " << std::abs(z) << " " << std::atan2(z.imag(), z.real()) << "\n";
    }
}

}  // namespace

// src/efield.cpp:91-113: fields/efield.dat and fields/afield.dat, "t E_x E_y E_z" per line.
void SWESim::write_fields_files(const std::string& dir) {
  std::filesystem::create_directories(dir);
  std::ofstream fe(dir + "/efield.dat"), fa(dir + "/afield.dat");
  fe << 1 << "\n";
  fa << 1 << "\n";
  for (int i = 0; i < nt; ++i) {
    fe << t[i] << " " << E[i] << " " << E[nt + i] << " " << E[2 * (size_t)nt + i] << "\n";
    fa << t[i] << " " << A[i] << " " << A[nt + i] << " " << A[2 * (size_t)nt + i] << "\n";
  }
}

// Debug dumps in the text format of src/matrix_field.cpp:28-53 ("index |z| arg z"), following
// src/swe.cpp:131-181: supercell and k vectors (SI and AU), the placed Hamiltonian (SI and AU),
// the equilibrium rho(k) (W gauge, AU), the Berry connections and the fields.
void SWESim::test_files() {
  if (!ready) throw std::runtime_error("SWESim_test_files: SWESim_init has not succeeded");
  std::filesystem::create_directories("test");
  double b[3][3];
  {
    const double(*a)[3] = model.lattice;
    double cr[3][3];
    for (int r = 0; r < 3; ++r) {
      const int p = (r + 1) % 3, q = (r + 2) % 3;
      cr[r][0] = a[p][1] * a[q][2] - a[p][2] * a[q][1];
      cr[r][1] = a[p][2] * a[q][0] - a[p][0] * a[q][2];
      cr[r][2] = a[p][0] * a[q][1] - a[p][1] * a[q][0];
    }
    const double vol = a[0][0] * cr[0][0] + a[0][1] * cr[0][1] + a[0][2] * cr[0][2];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) b[r][c] = 2.0 * M_PI / vol * cr[r][c];
  }
  for (int au = 0; au < 2; ++au) {
    const double lf = au ? kA2Bohr : 1.0;
    const char* tag = au ? "AU" : "SI";
    std::ofstream fr(std::string("test/Rvecs_") + tag + ".dat"), fk(std::string("test/Kvecs_") + tag + ".dat");
    fr << "_" << tag << "_\n";
    fk << "_" << tag << "_\n";
    for (int c = 0; c < Nk; ++c) {
      const int m1 = c / N2, m2 = c % N2;
      fr << Rgrid[3 * c] * lf << " " << Rgrid[3 * c + 1] * lf << " " << Rgrid[3 * c + 2] * lf << "\n";
      double k[3];
      for (int x = 0; x < 3; ++x) k[x] = ((double)m1 / N1 * b[0][x] + (double)m2 / N2 * b[1][x]) / lf;
      fk << k[0] << " " << k[1] << " " << k[2] << "\n";
    }
    const double ef = au ? kEv2Ha : 1.0;
    write_matrix_field(std::string("test/hamiltonian_") + tag + ".dat", au ? "_AU_" : "_SI_", Nk, nw2,
                       [&](int c, int o) {
                         const int st = site_of_cell[c];
                         return st >= 0 ? model.hop[(size_t)st * nw2 + o] * ef : cd(0, 0);
                       });
  }
  std::vector<double2> rho((size_t)Nk * nw2);
  check_cuda(cudaMemcpy(rho.data(), d_rho0.p, sizeof(double2) * rho.size(), cudaMemcpyDeviceToHost), "D2H");
  write_matrix_field("test/rho_k_W_AU.dat", "_AU_", Nk, nw2,
                     [&](int c, int o) { return cd(rho[(size_t)c * nw2 + o].x, rho[(size_t)c * nw2 + o].y); });
  const char* names[3] = {"test/x_bc.dat", "test/y_bc.dat", "test/z_bc.dat"};
  for (int a = 0; a < 3; ++a)
    write_matrix_field(names[a], "_AU_", Nk, nw2, [&](int c, int o) {
      const int st = site_of_cell[c];
      return st >= 0 ? -model.bc[a][(size_t)st * nw2 + o] * kA2Bohr : cd(0, 0);
    });
  write_fields_files("fields");
}

// ------------------------------------------------------------------------------------- C ABI

namespace {

void set_error(SWESim* swe, const std::string& msg) {
  g_last_error = msg;
  g_has_error = true;
  if (swe) {
    swe->err = msg;
    swe->has_err = true;
  }
}

void clear_error(SWESim* swe) {
  g_has_error = false;
  if (swe) swe->has_err = false;
}

template <typename F>
void guarded(SWESim* swe, const char* name, F&& f) {
  if (!swe) {
    set_error(nullptr, std::string(name) + ": null SWESim");
    return;
  }
  try {
    clear_error(swe);
    f();
  } catch (const std::exception& e) {
    set_error(swe, e.what());
  } catch (...) {
    set_error(swe, std::string(name) + ": unknown error");
  }
}

}  // namespace

extern "C" {

SWESim* SWESim_new(void) {
  try {
    clear_error(nullptr);
    return new SWESim();
  } catch (...) {
    set_error(nullptr, "SWESim_new: out of memory");
    return nullptr;
  }
}

void SWESim_run_simulation(SWESim* swe) { guarded(swe, "SWESim_run_simulation", [&] { swe->run(); }); }

void SWESim_test_files(SWESim* swe) { guarded(swe, "SWESim_test_files", [&] { swe->test_files(); }); }

void SWESim_set_path_tb(SWESim* swe, char* path_tb) {
  guarded(swe, "SWESim_set_path_tb", [&] { swe->path_tb = path_tb ? std::string(path_tb) : std::string(); });
}

void SWESim_set_settings(SWESim* swe, Settings* settings) {
  guarded(swe, "SWESim_set_settings", [&] { swe->settings = settings; });
}

void SWESim_init(SWESim* swe) { guarded(swe, "SWESim_init", [&] { swe->init(); }); }

void SWESim_restart(SWESim* swe) { guarded(swe, "SWESim_restart", [&] { swe->init(); }); }

void SWESim_get_current(SWESim* swe, double* t, hhg_cdouble* jx, hhg_cdouble* jy, hhg_cdouble* jz) {
  guarded(swe, "SWESim_get_current", [&] {
    if (!swe->ready && !swe->served) throw std::runtime_error("SWESim_get_current: SWESim_init has not succeeded");
    if ((int)swe->Jhist[0].size() < swe->nt)
      throw std::runtime_error("SWESim_get_current: run_simulation has not been called");
    hhg_cdouble* out[3] = {jx, jy, jz};
    for (int ti = 0; ti < swe->nt; ++ti) {
      if (t) t[ti] = swe->t[ti];
      for (int a = 0; a < 3; ++a)
        if (out[a]) out[a][ti] = hhg_cdouble{swe->Jhist[a][ti].real(), swe->Jhist[a][ti].imag()};
    }
  });
}

void SWESim_delete(SWESim* swe) {
  try {
    delete swe;
  } catch (...) {
  }
}

Settings* Settings_new(void) { return new Settings(); }
void Settings_delete(Settings* s) { delete s; }
void Settings_set_nr1(Settings* s, int v) { if (s) s->nr1 = v; }
void Settings_set_nr2(Settings* s, int v) { if (s) s->nr2 = v; }
void Settings_set_nr3(Settings* s, int v) { if (s) s->nr3 = v; }
void Settings_set_tmax(Settings* s, double v) { if (s) s->tmax = v; }
void Settings_set_dt(Settings* s, double v) { if (s) s->dt = v; }
void Settings_set_intensity(Settings* s, double v) { if (s) s->intensity_wcm2 = v; }
void Settings_set_lambda(Settings* s, double v) { if (s) s->lambda_nm = v; }
void Settings_set_tmax_field(Settings* s, double v) { if (s) s->tmax_field = v; }
void Settings_set_pol_vec(Settings* s, double* v) {
  if (s && v) {
    s->sx = v[0];
    s->sy = v[1];
    s->sz = v[2];
  }
}
void Settings_set_phi_vec(Settings* s, double* v) {
  if (s && v) {
    s->phi_x = v[0];
    s->phi_y = v[1];
    s->phi_z = v[2];
  }
}

const char* SWESim_last_error(SWESim* swe) { return (swe && swe->has_err) ? swe->err.c_str() : nullptr; }
const char* HHG_last_error(void) { return g_has_error ? g_last_error.c_str() : nullptr; }
int SWESim_get_nt(SWESim* swe) { return (swe && (swe->ready || swe->served)) ? swe->nt : -1; }
int SWESim_get_num_orb(SWESim* swe) { return (swe && swe->ready) ? swe->nw : -1; }
void SWESim_set_device(SWESim* swe, int device) {
  guarded(swe, "SWESim_set_device", [&] { swe->device = device; });
}
double SWESim_last_kernel_ms(SWESim* swe) { return swe ? (double)swe->last_ms : -1.0; }
double SWESim_last_propagate_ms(SWESim* swe) { return swe ? (double)swe->last_prop_ms : -1.0; }
long long SWESim_h2d_bytes(SWESim* swe) { return swe ? (long long)swe->h2d_bytes : -1; }
int SWESim_launch_shape(SWESim* swe, int* ctas, int* threads, int* k_per_cta, long long* smem) {
  if (!swe || !swe->ready) return -1;
  if (ctas) *ctas = swe->shape.ctas;
  if (threads) *threads = swe->shape.threads;
  if (k_per_cta) *k_per_cta = swe->shape.k_per_cta;
  if (smem) *smem = (long long)swe->shape.smem;
  return swe->shape.kernel;
}
int SWESim_last_launches(SWESim* swe) { return swe ? swe->last_launches : -1; }

void SWESim_get_rho_k(SWESim* swe, hhg_cdouble* out) {
  guarded(swe, "SWESim_get_rho_k", [&] {
    if (!swe->ready) throw std::runtime_error("SWESim_get_rho_k: SWESim_init has not succeeded");
    check_cuda(cudaMemcpy(out, swe->d_rho.p, sizeof(double2) * (size_t)swe->Nk * swe->nw2, cudaMemcpyDeviceToHost),
               "D2H");
  });
}

void SWESim_get_fields(SWESim* swe, double* t, double* E, double* A) {
  guarded(swe, "SWESim_get_fields", [&] {
    if (!swe->ready) throw std::runtime_error("SWESim_get_fields: SWESim_init has not succeeded");
    if (t) std::copy(swe->t.begin(), swe->t.end(), t);
    if (E) std::copy(swe->E.begin(), swe->E.end(), E);
    if (A) std::copy(swe->A.begin(), swe->A.end(), A);
  });
}

void SWESim_set_precision(SWESim* swe, int mode) {
  guarded(swe, "SWESim_set_precision", [&] {
    if (mode != 0 && mode != 1) throw std::runtime_error("SWESim_set_precision: mode must be 0 (plain FP64) or 1 (mixed)");
    swe->precision = mode;
  });
}

void SWESim_set_autotune(SWESim* swe, int on) {
  guarded(swe, "SWESim_set_autotune", [&] { swe->autotune = on != 0; });
}

void SWESim_set_tb_convention(SWESim* swe, int flags) {
  guarded(swe, "SWESim_set_tb_convention", [&] {
    if (flags < 0 || flags > 3) throw std::runtime_error("SWESim_set_tb_convention: flags must be in 0..3");
    swe->tb_flags = flags;
  });
}

void SWESim_set_solver(SWESim* swe, int mode) {
  guarded(swe, "SWESim_set_solver", [&] {
    if (mode != 0 && mode != 1)
      throw std::runtime_error("SWESim_set_solver: mode must be 0 (real-space solver) or 1 (k-space solver)");
    swe->solver = mode;
  });
}

void SWESim_set_k_rows(SWESim* swe, int row0, int row1) {
  guarded(swe, "SWESim_set_k_rows", [&] {
    swe->req_row0 = row0;
    swe->req_row1 = row1;
  });
}

void SWESim_reset(SWESim* swe) { guarded(swe, "SWESim_reset", [&] { swe->reset_state(); }); }

// Allocation-free variant of SWESim_run_simulation; see include/hhg_swe.h.
int SWESim_run_simulation_noalloc(SWESim* swe, hhg_cdouble* rho_k, hhg_cdouble* current, void* stream) {
  int rc = -1;
  guarded(swe, "SWESim_run_simulation_noalloc", [&] {
    if (!swe->ready) throw std::runtime_error("SWESim_run_simulation_noalloc: SWESim_init has not succeeded");
    if (!rho_k || !current) throw std::runtime_error("SWESim_run_simulation_noalloc: null rho_k or current pointer");
    check_cuda(cudaSetDevice(swe->device), "cudaSetDevice");
    char why[512] = {0};
    if (hhg::propagate_static_scratch(swe->tab, swe->gtab, swe->shape, reinterpret_cast<double2*>(rho_k),
                                           reinterpret_cast<double2*>(current), static_cast<cudaStream_t>(stream), why,
                                           sizeof why) != 0)
      throw std::runtime_error(std::string("SWESim_run_simulation_noalloc: ") + why);
    rc = 0;
  });
  return rc;
}

int HHG_measure_peaks(double* fp64_tflops, double* fp32_tflops) {
  try {
    return hhg::measure_fma_peaks(fp64_tflops, fp32_tflops);
  } catch (...) {
    return -1;
  }
}

}  // extern "C"

namespace hhg {
void set_thread_error(const std::string& msg) {
  g_last_error = msg;
  g_has_error = true;
}
}  // namespace hhg
