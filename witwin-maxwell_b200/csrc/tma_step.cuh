// Declarations of the TMA-fed fused step kernel (tma_kernel.cu).
#pragma once

#include <cuda.h>

#include "engine.cuh"

namespace fdtdb200 {

constexpr int kTmaRows = 8;                      // consumer warps (y rows) per CTA
constexpr int kTmaThreads = (kTmaRows + 1) * 32;  // + one producer warp
constexpr int kStages = 4;                       // plane tiles in flight per CTA

// Tensor maps of the current E^n and H^{n-1/2} component arrays (padded
// [NX][NY][P] float32 layout), boxes {36, rows, 1}.
struct TmaMaps {
  CUtensorMap e[3];
  CUtensorMap h[3];
};

template <bool kAnyCpml, bool kAnyCoef, bool kUniform>
__global__ void tma_step_kernel(const StepParams p, const __grid_constant__ TmaMaps maps, int n);

// Dynamic shared memory of one CTA.
size_t tma_smem_bytes();
// Encode the map of one field array; rows = tma_rows_e() for E, tma_rows_h() for H.
// Returns 0, -1 when the driver entry point is unavailable, or the CUresult.
int encode_field_map(CUtensorMap* map, const float* base, int NX, int NY, int P, int rows);
int tma_rows_e();
int tma_rows_h();

}  // namespace fdtdb200
