// noalloc.cu -- the fixed device workspace of the allocation-free GMRES entry
// point (spq_gmres_device_noalloc).
//
// The Krylov basis and the reduction scratch of that entry point live in one
// file-scope device array of kNoAllocDoubles doubles (48 MiB), sized for a
// preconditioned GMRES on 262,144 unknowns (the 64^3 grid) with up to 20
// iterations.  Its address is taken once per device with cudaGetSymbolAddress
// while that device is current; the first call on a device does this set-up,
// so that call should come before any stream capture on the device.  This
// file holds no kernel, so it compiles to a module of its own that CUDA 12.2+
// loads lazily, at that same first call: the 48 MiB are committed then, and
// the first call must come before a caller reserves the rest of device memory
// (or the process runs with CUDA_MODULE_LOADING=EAGER).  All
// trees on a device share the array: calls that overlap in time (other host
// threads, other streams) race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>

#include "noalloc.hpp"

namespace spq {
namespace {

static __device__ __align__(256) double g_noalloc_ws[kNoAllocDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_ws[kMaxDevices] = {};

}  // namespace

cudaError_t noalloc_workspace(double** ws) {
  *ws = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_ws[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_ws);
    if (e != cudaSuccess) return e;
    g_ws[dev] = static_cast<double*>(p);
  }
  *ws = g_ws[dev];
  return cudaSuccess;
}

}  // namespace spq
