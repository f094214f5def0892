// Propagation with library-owned scratch, for callers that must not allocate GPU memory.
//
// The propagation kernels accumulate the current in per-CTA partial sums ([ctas][nt][3] complex)
// before one reduction writes J.  SWESim_run_simulation keeps that scratch in a buffer it
// cudaMallocs at SWESim_init.  This file instead holds it in one fixed array of device global
// memory, g_current_scratch, which the CUDA driver reserves on every device where this library is
// used and keeps until the process exits.  A call therefore allocates nothing.
//
// Host code cannot use the array's name as a device address (on the host it names a stand-in
// object), so every call looks the address up with cudaGetSymbolAddress while the device is
// current.  The address is also kept per device for calls made while the stream is being captured
// into a graph, where the lookup (which may load the module) is not made: such a call needs an
// earlier call on the same device.  Looking it up again on every other call keeps the address
// right when the context was torn down and created again (cudaDeviceReset, or a framework that
// resets the primary context).  All calls on a device share the one array: it is cleared at the
// start of every call, and two calls whose work overlaps on the GPU (for example on two streams)
// corrupt each other's current.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "sbe_device.h"

namespace hhg {
namespace {

constexpr size_t kStaticScratchBytes = size_t(32) << 20;  // 32 MiB: [ctas][nt][3] complex128 partials
static __device__ __align__(256) unsigned char g_current_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void* g_scratch_address[kMaxDevices] = {};

}  // namespace

size_t static_scratch_capacity() { return kStaticScratchBytes; }

int propagate_static_scratch(const SolveTables& t, const GroupTables& gt, const LaunchShape& s, double2* rho,
                             double2* J, cudaStream_t stream, char* why, int why_len) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    snprintf(why, why_len, "no usable current CUDA device (%s)", cudaGetErrorString(e));
    return -1;
  }
  const size_t need = (size_t)s.vctas * (size_t)t.nt * 3 * sizeof(double2);
  if (need > kStaticScratchBytes) {
    snprintf(why, why_len,
             "this solve needs %zu bytes of scratch for its current partials (%d CTAs x %d steps x 3 axes); "
             "the allocation-free entry point has %zu bytes: use SWESim_run_simulation instead",
             need, s.vctas, t.nt, kStaticScratchBytes);
    return -1;
  }
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(stream, &capture);
  if (e != cudaSuccess) {
    snprintf(why, why_len, "cudaStreamIsCapturing failed: %s", cudaGetErrorString(e));
    return -1;
  }
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (capture == cudaStreamCaptureStatusNone) {
      void* addr = nullptr;
      e = cudaGetSymbolAddress(&addr, g_current_scratch);
      if (e != cudaSuccess || addr == nullptr) {
        snprintf(why, why_len, "cudaGetSymbolAddress of the static scratch failed on device %d: %s", dev,
                 cudaGetErrorString(e));
        return -1;
      }
      g_scratch_address[dev] = addr;
    } else if (!g_scratch_address[dev]) {
      snprintf(why, why_len,
               "the first allocation-free call on device %d is being captured into a graph: make one call on "
               "this device outside capture first, so that the scratch address is known", dev);
      return -1;
    }
    scratch = g_scratch_address[dev];
  }
  e = cudaMemsetAsync(scratch, 0, need, stream);
  if (e != cudaSuccess) {
    snprintf(why, why_len, "clearing the static scratch failed: %s", cudaGetErrorString(e));
    return -1;
  }
  launch_propagate(t, gt, s, rho, static_cast<double2*>(scratch), J, stream);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    snprintf(why, why_len, "propagation launch failed: %s", cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

}  // namespace hhg
