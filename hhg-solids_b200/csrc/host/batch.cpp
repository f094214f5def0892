// Several solves on one GPU: SWEBatch (a fixed set, propagated together from equilibrium) and
// SWEServer (a request loop with continuous batching).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>

#include "swe_sim.hpp"

using hhg::cd;
using hhg::check_cuda;
using hhg::DevBuf;

// ------------------------------------------------------------------------------------- batches

// Several initialised solves propagated together.  By default every solve keeps its own launch (the
// same kernel, shape and parameters as alone) on its own stream, and the hardware block scheduler
// packs the CTAs of the concurrent launches onto the SMs.  With HHG_BATCH=persistent, solves that
// run the element-group kernel are instead grouped by kernel shape into one persistent launch per
// shape whose CTAs take (solve, virtual CTA) items from a packed work list (longest first).  Measured
// on B200, the persistent form runs about 12 % more instructions per step (the solve descriptor lives
// in registers rather than in the constant bank of a launch's parameters): C2 mixed 843 vs 718 ms per
// solve in a batch of four, the 64-solve scan 32.3 vs 27.2 s; so the stream form is the default.
// Either way a solve keeps the tile shape and virtual-CTA split it has alone, so its current is bit
// for bit the one it gives alone.  The launch sequence (reset to rho0, clear, propagate, reduce,
// copy the current out) is captured once into a CUDA graph and replayed.
namespace {
bool persistent_batch_mode() {
  const char* mode = std::getenv("HHG_BATCH");
  return mode && std::strcmp(mode, "persistent") == 0;
}
}  // namespace

struct SWEBatch {
  int device = -1;
  std::vector<SWESim*> sims;
  std::vector<int> launches;  // per solve: kernel launches of one run (propagation and reduction)
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> done;
  cudaStream_t master = nullptr;
  cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr;
  cudaGraphExec_t graph = nullptr;
  DevBuf<hhg::BatchDesc> d_desc;
  DevBuf<int2> d_items;
  DevBuf<int> d_counters;
  std::vector<unsigned> generations;
  bool dirty = true;
  float last_ms = 0.f;
  int groups = 0, separate = 0;
  std::string err;
  bool has_err = false;

  ~SWEBatch() { release(); }
  void release() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
    for (auto st : streams) cudaStreamDestroy(st);
    streams.clear();
    for (auto e : done) cudaEventDestroy(e);
    done.clear();
    for (auto* e : {&fork, &ev0, &ev1})
      if (*e) cudaEventDestroy(*e);
    fork = ev0 = ev1 = nullptr;
    if (master) cudaStreamDestroy(master);
    master = nullptr;
  }

  void prepare() {
    if (sims.empty()) throw std::runtime_error("SWEBatch_run: empty batch");
    for (SWESim* sim : sims)
      if (!sim->ready) throw std::runtime_error("SWEBatch_run: a solve of the batch is not initialised");
    device = sims[0]->device;
    for (SWESim* sim : sims)
      if (sim->device != device) throw std::runtime_error("SWEBatch_run: all solves of a batch must be on one device");
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    release();
    int sms = 0;
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");

    const bool streams_only = !persistent_batch_mode();
    // Kernel-shape classes of the element-group solves; the others run alone.
    std::map<std::tuple<int, int, int, int, int, int, int, int, int>, std::vector<int>> classes;
    std::vector<int> alone;
    for (int i = 0; i < (int)sims.size(); ++i) {
      const hhg::LaunchShape& sh = sims[i]->shape;
      if (sh.kernel == 0 || sh.kernel == 3 || sh.pre_chunk > 0 || streams_only) {
        alone.push_back(i);
      } else {
        const hhg::SolveTables& t = sims[i]->tab;
        classes[std::make_tuple(sh.kernel, sh.variant, sh.ept, sh.threads, sh.group, sh.kmode, t.nw, t.nax, t.nj)].push_back(i);
      }
    }
    groups = (int)classes.size();
    separate = (int)alone.size();
    // Descriptors and items (per class: solves by decreasing item cost, all items of a solve).
    std::vector<hhg::BatchDesc> descs(sims.size());
    std::vector<int2> items;
    std::vector<std::pair<size_t, size_t>> ranges;  // per class: [first item, end)
    for (int i = 0; i < (int)sims.size(); ++i) {
      SWESim* sim = sims[i];
      hhg::BatchDesc& d = descs[i];
      std::memset(&d, 0, sizeof d);
      d.t = sim->tab;
      d.gt = sim->gtab;
      d.B = sim->shape.k_per_cta;
      d.G = sim->shape.group;
      d.box_sm = sim->shape.box_sm;
      d.win_sm = sim->shape.win_sm;
      d.vctas = sim->shape.vctas;
      d.rho = sim->d_rho.p;
      d.Jpart = sim->d_Jpart.p;
    }
    for (auto& kv : classes) {
      std::vector<int> members = kv.second;
      auto cost = [&](int i) {
        const hhg::LaunchShape& sh = sims[i]->shape;
        return (double)sh.ntiles / std::max(1, sh.vctas);  // tiles per item
      };
      std::stable_sort(members.begin(), members.end(), [&](int a, int b) { return cost(a) > cost(b); });
      const size_t first = items.size();
      for (int i : members)
        for (int v = 0; v < sims[i]->shape.vctas; ++v) items.push_back(make_int2(i, v));
      ranges.emplace_back(first, items.size());
    }
    d_desc.alloc(descs.size());
    check_cuda(cudaMemcpy(d_desc.p, descs.data(), sizeof(hhg::BatchDesc) * descs.size(), cudaMemcpyHostToDevice), "H2D");
    d_items.alloc(std::max<size_t>(1, items.size()));
    if (!items.empty())
      check_cuda(cudaMemcpy(d_items.p, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice), "H2D");
    d_counters.alloc(std::max<size_t>(1, classes.size()));

    check_cuda(cudaStreamCreateWithFlags(&master, cudaStreamNonBlocking), "cudaStreamCreate");
    for (auto* e : {&fork, &ev0, &ev1}) check_cuda(cudaEventCreate(e), "cudaEventCreate");
    const size_t nstreams = classes.size() + alone.size();
    streams.resize(nstreams);
    done.resize(nstreams);
    for (size_t q = 0; q < nstreams; ++q) {
      check_cuda(cudaStreamCreateWithFlags(&streams[q], cudaStreamNonBlocking), "cudaStreamCreate");
      check_cuda(cudaEventCreateWithFlags(&done[q], cudaEventDisableTiming), "cudaEventCreate");
    }

    auto reset_and_clear = [&](SWESim* sim, cudaStream_t st) {
      check_cuda(cudaMemcpyAsync(sim->d_rho.p, sim->d_rho0.p, sizeof(double2) * (size_t)sim->Nk * sim->nw2,
                                 cudaMemcpyDeviceToDevice, st), "D2D");
      check_cuda(cudaMemsetAsync(sim->d_Jpart.p, 0, sizeof(double2) * (size_t)sim->shape.vctas * sim->nt * 3, st),
                 "memset");
    };
    auto reduce_and_copy = [&](SWESim* sim, cudaStream_t st) {
      hhg::launch_reduce_current(sim->d_Jpart.p, sim->shape.vctas, sim->nt, sim->Nk, sim->d_J.p, st);
      check_cuda(cudaMemcpyAsync(sim->host_J(), sim->d_J.p, sizeof(double2) * 3 * (size_t)sim->nt, cudaMemcpyDeviceToHost, st),
                 "D2H");
    };

    launches.assign(sims.size(), 0);
    for (SWESim* sim : sims) sim->host_J();  // pinned current buffers, before the capture
    cudaGraph_t g = nullptr;
    check_cuda(cudaStreamBeginCapture(master, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture");
    check_cuda(cudaEventRecord(fork, master), "event");
    size_t q = 0;
    int ci = 0;
    for (auto& kv : classes) {
      cudaStream_t st = streams[q];
      check_cuda(cudaStreamWaitEvent(st, fork, 0), "cudaStreamWaitEvent");
      size_t smem = 0;
      for (int i : kv.second) {
        reset_and_clear(sims[i], st);
        smem = std::max(smem, sims[i]->shape.smem);
      }
      check_cuda(cudaMemsetAsync(d_counters.p + ci, 0, sizeof(int), st), "memset");
      const auto& rg = ranges[ci];
      hhg::launch_group_batch(sims[kv.second[0]]->shape, d_desc.p, d_items.p + rg.first, (int)(rg.second - rg.first),
                              d_counters.p + ci, smem, sms, st);
      for (int i : kv.second) launches[i] = 2;  // the shared launch and the solve's reduction
      for (int i : kv.second) reduce_and_copy(sims[i], st);
      check_cuda(cudaEventRecord(done[q], st), "event");
      check_cuda(cudaStreamWaitEvent(master, done[q], 0), "cudaStreamWaitEvent");
      ++q;
      ++ci;
    }
    for (int i : alone) {
      cudaStream_t st = streams[q];
      SWESim* sim = sims[i];
      check_cuda(cudaStreamWaitEvent(st, fork, 0), "cudaStreamWaitEvent");
      reset_and_clear(sim, st);
      launches[i] = hhg::launch_propagate(sim->tab, sim->gtab, sim->shape, sim->d_rho.p, sim->d_Jpart.p, sim->d_J.p, st);
      check_cuda(cudaMemcpyAsync(sim->host_J(), sim->d_J.p, sizeof(double2) * 3 * (size_t)sim->nt, cudaMemcpyDeviceToHost, st),
                 "D2H");
      check_cuda(cudaEventRecord(done[q], st), "event");
      check_cuda(cudaStreamWaitEvent(master, done[q], 0), "cudaStreamWaitEvent");
      ++q;
    }
    check_cuda(cudaStreamEndCapture(master, &g), "cudaStreamEndCapture");
    const cudaError_t ie = cudaGraphInstantiate(&graph, g, 0);
    cudaGraphDestroy(g);
    check_cuda(ie, "cudaGraphInstantiate");
    generations.clear();
    for (SWESim* sim : sims) generations.push_back(sim->generation);
    dirty = false;
  }

  // Every solve from its equilibrium rho0; each SWESim then holds its current as after
  // SWESim_reset + SWESim_run_simulation.
  void run() {
    for (size_t i = 0; i < sims.size() && !dirty; ++i) dirty = !sims[i]->ready || generations[i] != sims[i]->generation;
    if (dirty) prepare();
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    check_cuda(cudaEventRecord(ev0, master), "event");
    check_cuda(cudaGraphLaunch(graph, master), "cudaGraphLaunch");
    check_cuda(cudaEventRecord(ev1, master), "event");
    check_cuda(cudaStreamSynchronize(master), "SWEBatch_run");
    check_cuda(cudaEventElapsedTime(&last_ms, ev0, ev1), "event time");
    for (size_t i = 0; i < sims.size(); ++i) {
      SWESim* sim = sims[i];
      for (auto& j : sim->Jhist) j.clear();
      for (int a = 0; a < 3; ++a)
        for (int ti = 0; ti < sim->nt; ++ti)
          sim->Jhist[a].push_back(cd(sim->h_J[(size_t)a * sim->nt + ti].x, sim->h_J[(size_t)a * sim->nt + ti].y));
      sim->last_launches = launches[i];
    }
  }
};


// ------------------------------------------------------------------------------------- serving

// A request loop with continuous batching.  Requests (SWESim objects with settings and TB path set)
// queue in arrival order.  A scheduler thread admits the queue head when the device memory it will
// take (an upper bound computed before any allocation, replaced by the exact figure once set up) fits
// in the budget beside the solves already admitted and fewer than max_active are admitted, sets it up
// (SWESim_init on its own stream) while the GPU runs the current chunk, and adds it to the next chunk.
// A chunk advances every running solve by up to chunk_steps RK4 steps: each solve's own launch (step
// range [step, step + chunk_steps)) on a stream of a pool, so the block scheduler interleaves them
// (or, with HHG_BATCH=persistent, one persistent work-stealing launch per kernel shape over the
// running solves' (solve, virtual CTA) items; see SWEBatch for the measured comparison).  A solve that reaches nt is reduced, its current copied out, its
// device memory returned, and its ticket completed; the others continue with the next chunk, joined
// by the newly admitted.  A pulse run in chunks gives the same state and current bit for bit as in
// one launch, and a solve's tile shape and work split do not depend on the others, so every result
// equals, bit for bit, the one the same solve gives alone.
namespace {

using Clock = std::chrono::steady_clock;

struct Ticket {
  long long id = 0;
  SWESim* sim = nullptr;
  int state = 0;  // 0 queued, 1 setting up, 2 running, 3 done, -1 failed
  std::string err;
  double t_submit = 0, t_admit = 0, t_start = 0, t_done = 0;  // seconds since the server started
  size_t estimate = 0, reserved = 0;
  int step = 0, step1 = 0;
};

}  // namespace

struct SWEServer {
  int device = 0;
  size_t budget = 0;
  int max_active = 32;
  int chunk = 256;
  Clock::time_point t0 = Clock::now();

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Ticket*> queue;
  std::map<long long, std::unique_ptr<Ticket>> tickets;
  long long next_id = 0;
  bool stopping = false;
  size_t used = 0;    // bytes reserved by admitted, unfinished solves
  int admitted = 0;   // admitted, unfinished solves
  std::string fatal;

  // Scheduler-thread state.
  std::vector<Ticket*> active, joining;
  std::thread thr;
  cudaStream_t master = nullptr;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> stream_done;
  cudaEvent_t chunk_begin = nullptr, chunk_end = nullptr, uploaded = nullptr;
  cudaEvent_t ends[2] = {nullptr, nullptr};  // chunk_end alternates between these (GPU gaps between chunks)
  bool have_prev_end = false;
  DevBuf<hhg::BatchDesc> d_desc;
  DevBuf<int2> d_items;
  DevBuf<int> d_counters;
  DevBuf<double2> d_J;
  std::vector<hhg::BatchDesc> h_desc;
  std::vector<int2> h_items;
  double2* h_J = nullptr;
  size_t h_J_cap = 0;
  // Statistics.
  long long chunks = 0, completed = 0, failed = 0;
  int peak_active = 0;
  size_t peak_bytes = 0;
  double gpu_ms = 0.0;
  double gap_ms = 0.0;    // GPU time between the end of a chunk and the start of the next one
  double setup_ms = 0.0;  // host time setting up admitted solves
  double finish_ms = 0.0; // host time completing finished solves

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

  void start() {
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    if (budget == 0) {
      size_t fr = 0, tot = 0;
      check_cuda(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo");
      budget = fr / 10 * 8;
    }
    check_cuda(cudaStreamCreateWithFlags(&master, cudaStreamNonBlocking), "cudaStreamCreate");
    check_cuda(cudaEventCreate(&chunk_begin), "cudaEventCreate");
    for (auto* e : {&ends[0], &ends[1]}) check_cuda(cudaEventCreateWithFlags(e, cudaEventBlockingSync), "cudaEventCreate");
    chunk_end = ends[0];
    check_cuda(cudaEventCreateWithFlags(&uploaded, cudaEventDisableTiming), "cudaEventCreate");
    thr = std::thread([this] { loop(); });
  }

  ~SWEServer() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stopping = true;
    }
    cv_work.notify_all();
    if (thr.joinable()) thr.join();
    for (auto st : streams) cudaStreamDestroy(st);
    for (auto e : stream_done) cudaEventDestroy(e);
    for (auto e : {chunk_begin, ends[0], ends[1], uploaded})
      if (e) cudaEventDestroy(e);
    if (master) cudaStreamDestroy(master);
    if (h_J) cudaFreeHost(h_J);
  }

  long long submit(SWESim* sim) {
    std::lock_guard<std::mutex> lk(mu);
    if (stopping) throw std::runtime_error("SWEServer_submit: server is shutting down");
    for (const auto& kv : tickets)
      if (kv.second->sim == sim && kv.second->state >= 0 && kv.second->state < 3)
        throw std::runtime_error("SWEServer_submit: this SWESim is already queued or running");
    auto t = std::make_unique<Ticket>();
    t->id = next_id++;
    t->sim = sim;
    t->t_submit = now();
    queue.push_back(t.get());
    const long long id = t->id;
    tickets[id] = std::move(t);
    cv_work.notify_all();
    return id;
  }

  void fail(Ticket* t, const std::string& msg) {
    std::lock_guard<std::mutex> lk(mu);
    t->state = -1;
    t->err = msg;
    t->t_done = now();
    ++failed;
    cv_done.notify_all();
  }

  // Admits and sets up the queue head if it fits; false when nothing was admitted.
  bool admit_one() {
    Ticket* t = nullptr;
    {
      std::lock_guard<std::mutex> lk(mu);
      if (queue.empty() || admitted >= max_active) return false;
      t = queue.front();
    }
    SWESim* sim = t->sim;
    if (t->estimate == 0) {
      try {
        if (sim->ready && sim->device != device)
          throw std::runtime_error("SWEServer: the SWESim is initialised on another device");
        t->estimate = sim->ready ? sim->device_bytes() : sim->footprint_estimate();
      } catch (const std::exception& e) {
        {
          std::lock_guard<std::mutex> lk(mu);
          queue.pop_front();
        }
        fail(t, e.what());
        return true;
      }
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      if (admitted > 0 && used + t->estimate > budget) return false;  // wait for memory
      queue.pop_front();
      used += t->estimate;
      ++admitted;
      t->reserved = t->estimate;
      t->state = 1;
      t->t_admit = now();
    }
    const auto s0 = Clock::now();
    try {
      if (!sim->ready) {
        sim->device = device;
        sim->init();
      } else {
        sim->reset_state();
      }
      check_cuda(cudaSetDevice(device), "cudaSetDevice");
      check_cuda(cudaMemsetAsync(sim->d_Jpart.p, 0, sizeof(double2) * sim->d_Jpart.n, sim->stream), "memset");
      check_cuda(cudaStreamSynchronize(sim->stream), "setup");
      for (auto& j : sim->Jhist) j.clear();
      const size_t actual = sim->device_bytes();
      setup_ms += std::chrono::duration<double, std::milli>(Clock::now() - s0).count();
      std::lock_guard<std::mutex> lk(mu);
      used = used - t->reserved + actual;
      t->reserved = actual;
      peak_bytes = std::max(peak_bytes, used);
      t->state = 2;
    } catch (const std::exception& e) {
      {
        std::lock_guard<std::mutex> lk(mu);
        used -= t->reserved;
        --admitted;
      }
      try {
        sim->release();
      } catch (...) {
      }
      fail(t, e.what());
      check_cuda(cudaSetDevice(device), "cudaSetDevice");
      return true;
    }
    t->step = 0;
    joining.push_back(t);
    return true;
  }

  cudaStream_t stream_at(size_t q) {
    while (streams.size() <= q) {
      cudaStream_t st;
      cudaEvent_t e;
      check_cuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
      check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
      streams.push_back(st);
      stream_done.push_back(e);
    }
    return streams[q];
  }

  void launch_chunk() {
    hhg::TraceRange range("hhg SWEServer chunk");
    const bool persistent = persistent_batch_mode();
    int sms = 0;
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
    std::map<std::tuple<int, int, int, int, int, int, int, int, int>, std::vector<int>> classes;
    std::vector<int> alone;
    h_desc.assign(active.size(), hhg::BatchDesc{});
    for (int i = 0; i < (int)active.size(); ++i) {
      Ticket* t = active[i];
      SWESim* sim = t->sim;
      if (t->step == 0) t->t_start = now();
      t->step1 = std::min(sim->nt, t->step + chunk);
      hhg::BatchDesc& d = h_desc[i];
      d.t = sim->tab;
      d.t.step0 = t->step;
      d.t.step1 = t->step1;
      d.gt = sim->gtab;
      d.B = sim->shape.k_per_cta;
      d.G = sim->shape.group;
      d.box_sm = sim->shape.box_sm;
      d.win_sm = sim->shape.win_sm;
      d.vctas = sim->shape.vctas;
      d.rho = sim->d_rho.p;
      d.Jpart = sim->d_Jpart.p;
      const hhg::LaunchShape& sh = sim->shape;
      if (sh.kernel == 0 || sh.kernel == 3 || sh.pre_chunk > 0 || !persistent)
        alone.push_back(i);
      else
        classes[std::make_tuple(sh.kernel, sh.variant, sh.ept, sh.threads, sh.group, sh.kmode, sim->tab.nw,
                                sim->tab.nax, sim->tab.nj)].push_back(i);
    }
    h_items.clear();
    std::vector<std::pair<size_t, size_t>> ranges;
    for (auto& kv : classes) {
      std::vector<int>& m = kv.second;
      auto cost = [&](int i) {
        const hhg::LaunchShape& sh = active[i]->sim->shape;
        return (double)sh.ntiles / std::max(1, sh.vctas) * (active[i]->step1 - active[i]->step);
      };
      std::stable_sort(m.begin(), m.end(), [&](int a, int c) { return cost(a) > cost(c); });
      const size_t first = h_items.size();
      for (int i : m)
        for (int v = 0; v < active[i]->sim->shape.vctas; ++v) h_items.push_back(make_int2(i, v));
      ranges.emplace_back(first, h_items.size());
    }
    d_desc.alloc(h_desc.size());
    d_items.alloc(h_items.size());
    d_counters.alloc(std::max<size_t>(1, classes.size()));
    check_cuda(cudaEventRecord(chunk_begin, master), "event");
    check_cuda(cudaMemcpyAsync(d_desc.p, h_desc.data(), sizeof(hhg::BatchDesc) * h_desc.size(), cudaMemcpyHostToDevice,
                               master), "H2D");
    if (!h_items.empty())
      check_cuda(cudaMemcpyAsync(d_items.p, h_items.data(), sizeof(int2) * h_items.size(), cudaMemcpyHostToDevice,
                                 master), "H2D");
    check_cuda(cudaMemsetAsync(d_counters.p, 0, sizeof(int) * d_counters.n, master), "memset");
    check_cuda(cudaEventRecord(uploaded, master), "event");
    size_t q = 0;
    int ci = 0;
    std::vector<size_t> used_streams;
    for (auto& kv : classes) {
      cudaStream_t st = stream_at(q);
      check_cuda(cudaStreamWaitEvent(st, uploaded, 0), "cudaStreamWaitEvent");
      size_t smem = 0;
      for (int i : kv.second) smem = std::max(smem, active[i]->sim->shape.smem);
      const auto& rg = ranges[ci];
      hhg::launch_group_batch(active[kv.second[0]]->sim->shape, d_desc.p, d_items.p + rg.first,
                              (int)(rg.second - rg.first), d_counters.p + ci, smem, sms, st);
      used_streams.push_back(q);
      ++q;
      ++ci;
    }
    // Solves launched on their own: one stream each, from a pool (the block scheduler interleaves them).
    const size_t pool = std::min<size_t>(alone.size(), (size_t)std::max(1, max_active));
    for (size_t a = 0; a < alone.size(); ++a) {
      const size_t qs = q + a % std::max<size_t>(1, pool);
      cudaStream_t st = stream_at(qs);
      if (a < pool) check_cuda(cudaStreamWaitEvent(st, uploaded, 0), "cudaStreamWaitEvent");
      SWESim* sim = active[alone[a]]->sim;
      hhg::launch_propagate_steps(h_desc[alone[a]].t, sim->gtab, sim->shape, sim->d_rho.p, sim->d_Jpart.p, st);
      if (a < pool) used_streams.push_back(qs);
    }
    q += pool;
    check_cuda(cudaGetLastError(), "chunk launch");
    for (size_t u : used_streams) {
      check_cuda(cudaEventRecord(stream_done[u], streams[u]), "event");
      check_cuda(cudaStreamWaitEvent(master, stream_done[u], 0), "cudaStreamWaitEvent");
    }
    chunk_end = ends[chunks % 2];
    check_cuda(cudaEventRecord(chunk_end, master), "event");
    ++chunks;
  }

  void finish_chunk() {
    hhg::TraceRange range("hhg SWEServer finish");
    check_cuda(cudaEventSynchronize(chunk_end), "chunk");
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, chunk_begin, chunk_end) == cudaSuccess) gpu_ms += ms;
    const cudaEvent_t prev_end = chunk_end == ends[0] ? ends[1] : ends[0];
    if (have_prev_end && cudaEventElapsedTime(&ms, prev_end, chunk_begin) == cudaSuccess) gap_ms += ms;
    have_prev_end = true;
    const auto f0 = Clock::now();
    struct AddFinish {
      double& acc;
      Clock::time_point t;
      ~AddFinish() { acc += std::chrono::duration<double, std::milli>(Clock::now() - t).count(); }
    } add_finish{finish_ms, f0};
    std::vector<Ticket*> finished, still;
    for (Ticket* t : active) {
      t->step = t->step1;
      (t->step >= t->sim->nt ? finished : still).push_back(t);
    }
    active.swap(still);
    if (finished.empty()) return;
    size_t total = 0;
    for (Ticket* t : finished) total += (size_t)3 * t->sim->nt;
    d_J.alloc(total);
    if (!h_J || h_J_cap < total) {
      if (h_J) cudaFreeHost(h_J);
      h_J = nullptr;
      check_cuda(cudaMallocHost(&h_J, sizeof(double2) * total), "cudaMallocHost");
      h_J_cap = total;
    }
    size_t off = 0;
    for (Ticket* t : finished) {
      SWESim* sim = t->sim;
      hhg::launch_reduce_current(sim->d_Jpart.p, sim->shape.vctas, sim->nt, sim->Nk, d_J.p + off, master);
      off += (size_t)3 * sim->nt;
    }
    check_cuda(cudaMemcpyAsync(h_J, d_J.p, sizeof(double2) * total, cudaMemcpyDeviceToHost, master), "D2H");
    check_cuda(cudaStreamSynchronize(master), "current");
    off = 0;
    for (Ticket* t : finished) {
      SWESim* sim = t->sim;
      const size_t n = (size_t)3 * sim->nt;
      sim->finish_served(h_J + off);
      off += n;
      check_cuda(cudaSetDevice(device), "cudaSetDevice");
      std::lock_guard<std::mutex> lk(mu);
      used -= t->reserved;
      --admitted;
      t->state = 3;
      t->t_done = now();
      ++completed;
    }
    cv_done.notify_all();
  }

  void fail_all_running(const std::string& msg) {
    std::vector<Ticket*> all = active;
    all.insert(all.end(), joining.begin(), joining.end());
    active.clear();
    joining.clear();
    for (Ticket* t : all) {
      try {
        t->sim->release();
      } catch (...) {
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        used -= t->reserved;
        --admitted;
      }
      fail(t, msg);
    }
  }

  void loop() {
    try {
      check_cuda(cudaSetDevice(device), "cudaSetDevice");
      for (;;) {
        // Nothing running: admit what fits, or sleep until a request arrives.
        if (active.empty() && joining.empty()) {
          if (admit_one()) continue;
          std::unique_lock<std::mutex> lk(mu);
          if (stopping && queue.empty()) break;
          if (queue.empty()) cv_work.wait(lk, [&] { return stopping || !queue.empty(); });
          continue;
        }
        active.insert(active.end(), joining.begin(), joining.end());
        joining.clear();
        if (active.empty()) continue;
        peak_active = std::max(peak_active, (int)active.size());
        launch_chunk();
        // While the chunk runs: set up queued requests (they join the next chunk).
        while (cudaEventQuery(chunk_end) == cudaErrorNotReady)
          if (!admit_one()) break;
        finish_chunk();
      }
    } catch (const std::exception& e) {
      std::string msg = std::string("SWEServer: ") + e.what();
      {
        std::lock_guard<std::mutex> lk(mu);
        fatal = msg;
      }
      fail_all_running(msg);
      // Fail what is still queued; later submissions fail at once.
      std::unique_lock<std::mutex> lk(mu);
      stopping = true;
      while (!queue.empty()) {
        Ticket* t = queue.front();
        queue.pop_front();
        t->state = -1;
        t->err = msg;
        t->t_done = now();
        ++failed;
      }
      cv_done.notify_all();
    }
  }

  // 1 done, -1 failed, 0 timed out, -2 unknown ticket.
  int wait(long long id, double timeout_s) {
    std::unique_lock<std::mutex> lk(mu);
    auto it = tickets.find(id);
    if (it == tickets.end()) return -2;
    Ticket* t = it->second.get();
    auto done = [&] { return t->state == 3 || t->state == -1; };
    if (timeout_s < 0)
      cv_done.wait(lk, done);
    else if (!cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done))
      return 0;
    return t->state == 3 ? 1 : -1;
  }
};

extern "C" {

SWEBatch* SWEBatch_new(void) {
  try {
    return new SWEBatch();
  } catch (...) {
    return nullptr;
  }
}

void SWEBatch_delete(SWEBatch* b) {
  try {
    delete b;
  } catch (...) {
  }
}

int SWEBatch_add(SWEBatch* b, SWESim* swe) {
  if (!b || !swe) return -1;
  b->sims.push_back(swe);
  b->dirty = true;
  return (int)b->sims.size() - 1;
}

int SWEBatch_run(SWEBatch* b) {
  hhg::TraceRange range("hhg SWEBatch_run");
  if (!b) return -1;
  try {
    b->has_err = false;
    b->run();
    return 0;
  } catch (const std::exception& e) {
    b->err = e.what();
    b->has_err = true;
    hhg::set_thread_error(b->err);
    b->dirty = true;
    return -1;
  }
}

double SWEBatch_last_ms(SWEBatch* b) { return b ? (double)b->last_ms : -1.0; }
const char* SWEBatch_last_error(SWEBatch* b) { return (b && b->has_err) ? b->err.c_str() : nullptr; }


SWEServer* SWEServer_new(int device, long long hbm_budget_bytes, int max_active, int chunk_steps) {
  try {
    if (max_active < 1) throw std::runtime_error("SWEServer_new: max_active must be >= 1");
    if (chunk_steps < 1) throw std::runtime_error("SWEServer_new: chunk_steps must be >= 1");
    if (hbm_budget_bytes < 0) throw std::runtime_error("SWEServer_new: negative memory budget");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      throw std::runtime_error("SWEServer_new: no CUDA device (this library has no CPU path)");
    if (device < 0 || device >= ndev) throw std::runtime_error("SWEServer_new: no such device");
    auto srv = std::make_unique<SWEServer>();
    srv->device = device;
    srv->budget = (size_t)hbm_budget_bytes;
    srv->max_active = max_active;
    srv->chunk = chunk_steps;
    srv->start();
    return srv.release();
  } catch (const std::exception& e) {
    hhg::set_thread_error(e.what());
    return nullptr;
  }
}

long long SWEServer_submit(SWEServer* srv, SWESim* swe) {
  if (!srv || !swe) {
    hhg::set_thread_error("SWEServer_submit: null server or SWESim");
    return -1;
  }
  try {
    return srv->submit(swe);
  } catch (const std::exception& e) {
    hhg::set_thread_error(e.what());
    return -1;
  }
}

int SWEServer_wait(SWEServer* srv, long long ticket, double timeout_s) {
  return srv ? srv->wait(ticket, timeout_s) : -2;
}

int SWEServer_status(SWEServer* srv, long long ticket) {
  if (!srv) return -2;
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->tickets.find(ticket);
  return it == srv->tickets.end() ? -2 : it->second->state;
}

int SWEServer_times(SWEServer* srv, long long ticket, double* out4) {
  if (!srv || !out4) return -2;
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->tickets.find(ticket);
  if (it == srv->tickets.end()) return -2;
  const Ticket* t = it->second.get();
  out4[0] = t->t_submit;
  out4[1] = t->t_admit;
  out4[2] = t->t_start;
  out4[3] = t->t_done;
  return t->state;
}

const char* SWEServer_ticket_error(SWEServer* srv, long long ticket) {
  if (!srv) return nullptr;
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->tickets.find(ticket);
  if (it == srv->tickets.end() || it->second->state != -1) return nullptr;
  return it->second->err.c_str();
}

int SWEServer_stats(SWEServer* srv, double* out, int n) {
  if (!srv || !out) return -1;
  std::lock_guard<std::mutex> lk(srv->mu);
  const double v[12] = {(double)srv->completed, (double)srv->failed, (double)srv->chunks, srv->gpu_ms,
                        (double)srv->peak_active, (double)srv->peak_bytes, (double)srv->budget,
                        (double)srv->queue.size(), (double)srv->admitted, srv->gap_ms, srv->setup_ms,
                        srv->finish_ms};
  const int m = n < 12 ? n : 12;
  for (int i = 0; i < m; ++i) out[i] = v[i];
  return m;
}

void SWEServer_delete(SWEServer* srv) {
  try {
    delete srv;
  } catch (...) {
  }
}

}  // extern "C"
