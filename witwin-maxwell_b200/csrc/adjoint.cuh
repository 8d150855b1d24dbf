// Adjoint state and launchers of the reverse-time step (adjoint.cu).
#pragma once

#include "engine.cuh"

namespace fdtdb200 {

// Permittivity-gradient box of one E component: [lo, hi) in that component's
// Yee index space, the replayed E history of the box ([slot][cells]) and the
// accumulated dL/deps (absolute permittivity, F/m) per box cell.
struct DesignBox {
  int lo[3], hi[3];
  int64_t cells;
  float* hist;
  float* grad;  // nullptr: no box for this component
};

struct AdjParams {
  float* gE[3];        // adjoint of E (padded layout)
  float* gH[3];        // adjoint of H
  float* gpsiE[3][2];  // adjoint CPML psi, same slab layout as the forward psi
  float* gpsiH[3][2];
  const float* seed_re;  // dL/d(accumulator), [n_freq][n_samples]; nullptr = no seeds
  const float* seed_im;
  int64_t n_samples;
  DesignBox design[3];
  int hist_slot;  // history slot of E^n for the reverse step of step n
  float inv_dt;
  // Adjoint ADE pole state, per pole id in the forward pole-state layout:
  // gpol (adjoint of P; Debye, Lorentz) and gcur (adjoint of J; Drude, Lorentz).
  float* const* gpol;
  float* const* gcur;
};

// Reverse step of step n: seeds of step n, then passes A, B, C.
int launch_adjoint_step(const StepParams& p, const AdjParams& q, const RegionFlush* regions, int n_regions,
                        const float2* w_e, const float2* w_h, int n_freq, int n, cudaStream_t stream);
// Record the current E of every design box into history slot `slot`.
int launch_design_record(const StepParams& p, const AdjParams& q, int slot, cudaStream_t stream);

}  // namespace fdtdb200
