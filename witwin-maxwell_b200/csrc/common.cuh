// Shared device helpers for the B200 FDTD kernels.
//
// Field layout convention (same as the reference, witwin/maxwell/fdtd/cuda/kernels/common.cuh:61-63):
// C-contiguous [X][Y][Z] with z fastest.  Boundary codes follow
// witwin/maxwell/fdtd/boundary/common.py:5-10.
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

namespace fdtdb200 {

// Records the message returned by fdtd_last_error() for the calling thread.
void set_last_error(const std::string& msg);

constexpr int BND_NONE = 0;
constexpr int BND_PML = 1;
constexpr int BND_PERIODIC = 2;
constexpr int BND_BLOCH = 3;
constexpr int BND_PEC = 4;
constexpr int BND_PMC = 5;

__host__ __device__ __forceinline__ int64_t off3(int64_t i, int64_t j, int64_t k, int64_t ny, int64_t nz) {
  return (i * ny + j) * nz + k;
}

// Slab-compressed CPML index along one axis (witwin/maxwell/fdtd/cuda/kernels/common.cuh:65-78).
__host__ __device__ __forceinline__ int slab_local(int coord, int low, int hstart, int hlen) {
  if (coord < low) return coord;
  if (coord >= hstart && coord < hstart + hlen) return low + coord - hstart;
  return -1;
}

}  // namespace fdtdb200
