// PCG solve whose scratch lives in a fixed device array of this library, for
// callers that cannot allocate device memory.
//
// Some hosts cannot call cudaMalloc (or any allocating routine) on the path
// that solves: for example a Monte Carlo driver that hands device pointers to
// a plugin while it is being captured into a CUDA graph or while it runs
// under an allocator it does not own, or an embedded caller with a fixed
// memory budget that must not grow.  For them qedf_pcg_solve_static takes the
// same inputs and outputs as qedf_pcg_solve but uses the file-scope array
// g_pcg_scratch below as the solver's workspace, so it allocates nothing.
//
// The array is QEDF_PCG_STATIC_SCRATCH_BYTES (64 MiB) per GPU and every GPU
// that loads the library keeps it until the process exits.  Problems whose
// workspace (qedf_pcg_workspace_bytes) is larger are rejected with
// QEDF_ERR_SIZE.  All calls on a device share the array: calls that overlap on
// the GPU (other streams, or other host threads) race on it and must be
// serialised by the caller.  The array keeps the previous call's contents;
// the solver's preparation kernel clears the accumulators and barrier words
// that must start at zero on every call, and every vector the solve reads is
// written by it first.
//
// In host code the name g_pcg_scratch is only a host-side stand-in, not a
// device address.  The device address is looked up with cudaGetSymbolAddress
// once per device, with that device current, by the first call on it; make
// that first call before any stream capture begins.  The address is cached for
// the life of the process, so it is stale after cudaDeviceReset (the module is
// loaded again in the new context, possibly elsewhere): a process that resets
// a device must not call this entry point afterwards.
#include <cstdint>
#include <mutex>

#include "qedf_internal.h"

namespace {

__device__ __align__(256) unsigned char g_pcg_scratch[QEDF_PCG_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

// device address of g_pcg_scratch on the current device (set up once per device)
int scratch_address(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return QEDF_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_pcg_scratch) != cudaSuccess || !ptr) return QEDF_ERR_CUDA;
    g_scratch_addr[dev] = ptr;
  }
  *out = g_scratch_addr[dev];
  return QEDF_OK;
}

}  // namespace

extern "C" int qedf_pcg_solve_static(const qedf_system* sys, int nsys, const void* boson, const void* b, void* x,
                                     int* iters, double* relres, int* status, const qedf_pcg_opts* opts,
                                     qedf_stream_t stream) {
  if (!sys || !opts) return QEDF_ERR_ARG;
  const int64_t need = qedf_pcg_workspace_bytes(sys, nsys, opts);
  if (need < 0) return QEDF_ERR_ARG;
  if (need > (int64_t)QEDF_PCG_STATIC_SCRATCH_BYTES) return QEDF_ERR_SIZE;
  void* scratch = nullptr;
  if (int e = scratch_address(&scratch)) return e;
  return qedf::pcg_solve_ws(sys, nsys, boson, b, x, iters, relres, status, scratch,
                            (int64_t)QEDF_PCG_STATIC_SCRATCH_BYTES, opts, stream);
}
