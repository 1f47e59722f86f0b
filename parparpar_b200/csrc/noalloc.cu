// Solve-and-reconstruct for callers that may not allocate device memory.
//
// Some callers cannot call cudaMalloc at the point where they need a repair
// solve: code running inside a memory pool owned by another allocator that
// leaves no free device memory, latency-critical loops where the implicit
// device-wide synchronisation of cudaMalloc/cudaFree is not acceptable, or
// services that must not fail with out-of-memory once they have started.
// pp_gf64_solve_and_reconstruct_noalloc serves them: the caller passes the
// matrix and right-hand-side blocks (device memory, modified in place) and a
// stream; the few words of working storage the solve needs (the elimination
// multipliers, the pivot record and a status word) live in the fixed array
// below, which is part of the library image and is therefore resident on
// every GPU that loads the library until the process exits.
//
// Limits and sharing:
//   * n <= PP_NOALLOC_SOLVE_MAX_N (4096); larger systems are rejected with
//     PP_ERR_TOO_LARGE before any work is enqueued.
//   * Every call uses the same array.  Calls whose work overlaps on the GPU
//     (for example on two different streams) race on it and give wrong
//     results; order such calls.
//   * The status word is cleared at the start of every call; the multiplier
//     column is fully rewritten by each pivot step before it is read, so the
//     previous call's contents do not matter.
//   * The device address of the array is looked up (cudaGetSymbolAddress) the
//     first time the entry point runs on a device, with that device current,
//     and cached; make that first call on each device before any stream
//     capture begins.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/parpar_b200.h"
#include "pp_internal.h"

namespace {

constexpr size_t kMaxN = PP_NOALLOC_SOLVE_MAX_N;
constexpr size_t kStatusSlot = kMaxN + 2;  // after n multipliers + 2 pivot words

// [0, n): multipliers, [n, n+2): pivot row and its inverse, [kStatusSlot]: status
static __device__ __align__(256) uint64_t g_solve_scratch[kMaxN + 4];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint64_t* g_scratch_dev[kMaxDevices] = {};

// Per-device set-up: the address of the fixed array as seen by device code,
// looked up with the device current.
int scratch_for_current_device(uint64_t** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return PP_ERR_NO_DEVICE;
  }
  if (dev < 0 || dev >= kMaxDevices) return PP_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> g(g_mu);
  if (!g_scratch_dev[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_solve_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return PP_ERR_CUDA;
    }
    g_scratch_dev[dev] = static_cast<uint64_t*>(p);
  }
  *out = g_scratch_dev[dev];
  return PP_OK;
}

// True when the kernels launched on device `dev` may dereference p: device
// memory of that very device, or managed memory.  Device memory of another GPU
// is refused: the scratch address and every launch belong to the current
// device, so such a buffer would be read across the link or fault.
bool on_device(const void* p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace

extern "C" PP_API int pp_gf64_solve_and_reconstruct_noalloc(uint64_t* A, uint64_t* rhs, size_t n,
                                                            size_t block_size64, void* cuda_stream) {
  if (n == 0) return PP_OK;
  if (n > kMaxN) return PP_ERR_TOO_LARGE;
  if (!A || (block_size64 && !rhs)) return PP_ERR_INVALID_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return PP_ERR_NO_DEVICE;
  }
  if (!on_device(A, dev) || (block_size64 && !on_device(rhs, dev))) return PP_ERR_INVALID_ARG;
  uint64_t* scratch = nullptr;
  if (int st = scratch_for_current_device(&scratch)) return st;
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  int* status = reinterpret_cast<int*>(scratch + kStatusSlot);
  if (cudaMemsetAsync(status, 0, sizeof(int), s) != cudaSuccess) {
    cudaGetLastError();
    return PP_ERR_CUDA;
  }
  if (pp::launch_gf64_solve(A, rhs, n, block_size64, scratch, status, s) != cudaSuccess) {
    cudaGetLastError();
    return PP_ERR_CUDA;
  }
  int h = 0;
  if (cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return PP_ERR_CUDA;
  }
  return h ? PP_ERR_SINGULAR : PP_OK;
}
