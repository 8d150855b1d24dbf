// Incident-line history without device allocation.
//
// fdtd_engine_add_aux_line precomputes the 1-D incident line of a TFSF plane
// wave for every step with a kernel whose running line state (E and H, n_e
// floats each) lives in scratch buffers that the engine allocates.  This file
// holds a variant of that kernel whose running state lives in a fixed
// file-scope device array instead, behind fdtd_op_aux_line_history_static: the
// caller passes every input and output buffer and the call allocates no device
// memory.
//
// Callers that need it: a process whose device memory is all held by its own
// caching pool (a framework allocator that reserved the free memory), where a
// cudaMalloc fails or forces the pool to release cached blocks; and a caller
// on a latency-critical stream, where cudaFree's device-wide synchronisation
// would stall the work queued on every other stream.
//
// Limits: n_e <= kAuxStaticMaxCells.  The scratch array is one per device and
// shared by all callers, so two calls whose kernels can overlap (different
// streams, or different host threads without ordering) race on it and both
// results are undefined; order such calls on one stream.
#include <cuda_runtime.h>

#include <string>

#include "../../include/fdtd_b200.h"
#include "common.cuh"

using namespace fdtdb200;

namespace {

constexpr int kAuxStaticMaxCells = FDTD_AUX_STATIC_MAX_CELLS;

// Running line state: E in [0, n_e), H in [kAuxStaticMaxCells, +n_e - 1).
// Every call clears the part it uses before its first step.
static __device__ __align__(256) float g_aux_line_scratch[2 * kAuxStaticMaxCells];


// One 256-thread block marches the line in time.  Same recurrence as the
// engine's history kernel (AuxiliaryGrid1D.advance_magnetic/advance_electric,
// witwin/maxwell/fdtd/excitation/spatial.py:443-462, sources.cu:803-839): the
// E row is recorded before the step, H is advanced and recorded, then E is
// advanced, the source cell overwritten and the last cell pinned to zero (a
// source on the last cell is overridden by the zero, as in the reference's
// update_auxiliary_electric_kernel).  A negative source index injects nothing.
// The last entry of each H row (no H cell there) is written as zero.
__global__ void aux_history_static_kernel(int ne, const float* __restrict__ e_decay, const float* __restrict__ e_curl,
                                          const float* __restrict__ h_decay, const float* __restrict__ h_curl,
                                          int src_index, const float* __restrict__ source, int n_steps,
                                          float* __restrict__ e_hist, float* __restrict__ h_hist,
                                          float* __restrict__ scratch, int h_offset) {
  float* e = scratch;
  float* h = scratch + h_offset;
  for (int x = threadIdx.x; x < ne; x += blockDim.x) {
    e[x] = 0.0f;
    if (x < ne - 1) h[x] = 0.0f;
  }
  __syncthreads();
  for (int n = 0; n < n_steps; ++n) {
    float* erow = e_hist + static_cast<int64_t>(n) * ne;
    float* hrow = h_hist + static_cast<int64_t>(n) * ne;
    for (int x = threadIdx.x; x < ne; x += blockDim.x) erow[x] = e[x];
    for (int x = threadIdx.x; x < ne - 1; x += blockDim.x) h[x] = h_decay[x] * h[x] - h_curl[x] * (e[x + 1] - e[x]);
    __syncthreads();
    for (int x = threadIdx.x; x < ne - 1; x += blockDim.x) hrow[x] = h[x];
    if (threadIdx.x == 0) hrow[ne - 1] = 0.0f;
    for (int x = threadIdx.x; x < ne; x += blockDim.x) {
      if (x >= 1 && x < ne - 1 && x != src_index) e[x] = e_decay[x] * e[x] - e_curl[x] * (h[x] - h[x - 1]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      // the source cell first, then the last cell pinned to zero: a source
      // placed on the last cell is overridden, as in the reference's op
      if (src_index >= 0 && src_index < ne) e[src_index] = source[n];
      e[ne - 1] = 0.0f;
    }
    __syncthreads();
  }
}

int static_fail(int code, const std::string& msg) {
  set_last_error(msg);
  return code;
}

// Device address of the scratch array on the current device.  Looked up on
// every call (cheap and allocation-free), so the address stays valid after the
// device's primary context is reset and this file's module is loaded again;
// the first call on a device may load the module, so make it before any
// stream capture.
int scratch_for_current_device(float** out) {
  float* ptr = nullptr;
  const cudaError_t err = cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), g_aux_line_scratch);
  if (err != cudaSuccess || !ptr)
    return static_fail(FDTD_ERR_CUDA, std::string("aux_line_history_static: cudaGetSymbolAddress: ") +
                                          cudaGetErrorString(err));
  *out = ptr;
  return 0;
}

}  // namespace

extern "C" int fdtd_op_aux_line_history_static(int n_e, const float* e_decay, const float* e_curl,
                                               const float* h_decay, const float* h_curl, int source_index,
                                               const float* source, int n_steps, float* e_hist, float* h_hist,
                                               void* stream) {
  if (n_e > kAuxStaticMaxCells)
    return static_fail(FDTD_ERR_INVALID_ARG, "aux_line_history_static: n_e = " + std::to_string(n_e) +
                                                 " exceeds the static scratch maximum of " +
                                                 std::to_string(kAuxStaticMaxCells) + " cells");
  if (n_e < 4 || n_steps <= 0 || !e_decay || !e_curl || !h_decay || !h_curl || !source || !e_hist || !h_hist)
    return static_fail(FDTD_ERR_INVALID_ARG, "aux_line_history_static: bad arguments");
  float* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  aux_history_static_kernel<<<1, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      n_e, e_decay, e_curl, h_decay, h_curl, source_index, source, n_steps, e_hist, h_hist, scratch,
      kAuxStaticMaxCells);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess)
    return static_fail(FDTD_ERR_CUDA, std::string("aux_line_history_static: ") + cudaGetErrorString(err));
  return 0;
}
