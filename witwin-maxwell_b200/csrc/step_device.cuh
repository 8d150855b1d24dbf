// Device helpers shared by the fused step kernels (warp_kernel.cu,
// tma_kernel.cu): CPML slab addressing and recursion, injection-term and ADE
// pole application, E edge modes.  Arithmetic restated from
// witwin/maxwell/fdtd/cuda/kernels/magnetic.cu:62-212, electric.cu:242-311 and
// 462-941, dispersive.cu:18-83, sources.cu:135-154 and 485-545.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "engine.cuh"

namespace fdtdb200 {

namespace {

constexpr int kOut = 30;  // output z cells per warp
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float ldz(const float* base, int64_t off, bool ok) { return ok ? __ldg(base + off) : 0.0f; }

// Stored element types: FP32 (the exact path), FP16 and BF16 (reduced storage,
// FP32 arithmetic).
__device__ __forceinline__ float to_f32(float x) { return x; }
__device__ __forceinline__ float to_f32(__half x) { return __half2float(x); }
__device__ __forceinline__ float to_f32(__nv_bfloat16 x) { return __bfloat162float(x); }
template <typename T>
__device__ __forceinline__ T from_f32(float v);
template <>
__device__ __forceinline__ float from_f32<float>(float v) { return v; }
template <>
__device__ __forceinline__ __half from_f32<__half>(float v) { return __float2half_rn(v); }
template <>
__device__ __forceinline__ __nv_bfloat16 from_f32<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

// Field load of stored type TS (scaled by `scale` unless FP32), zero when !ok.
template <typename TS>
__device__ __forceinline__ float ldf(const float* base, int64_t off, bool ok, float scale) {
  if constexpr (sizeof(TS) == 4) {
    (void)scale;
    return ok ? __ldg(base + off) : 0.0f;
  } else {
    return ok ? to_f32(__ldg(reinterpret_cast<const TS*>(base) + off)) * scale : 0.0f;
  }
}

// Streaming field store of type TS (value multiplied by `inv` unless FP32).
template <typename TS>
__device__ __forceinline__ void stf(float* base, int64_t off, float v, float inv) {
  if constexpr (sizeof(TS) == 4) {
    (void)inv;
    __stcg(base + off, v);
  } else {
    TS* q = reinterpret_cast<TS*>(base) + off;
    *q = from_f32<TS>(v * inv);
  }
}

// L2 prefetch of the element at base + off of an array of stored type T (a
// hint: no register, no wait; callers pass in-bounds offsets only).
template <typename T>
__device__ __forceinline__ void pf_l2(const void* base, int64_t off) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const T*>(base) + off));
}

// ADE state element of type TA (FP32 or BF16, unscaled).
template <typename TA>
__device__ __forceinline__ float lda(const float* base, int64_t off) {
  return to_f32(reinterpret_cast<const TA*>(base)[off]);
}
template <typename TA>
__device__ __forceinline__ void sta(float* base, int64_t off, float v) {
  reinterpret_cast<TA*>(base)[off] = from_f32<TA>(v);
}

__device__ __forceinline__ int slab_coord(const StepParams& p, int axis, int coord, int extent) {
  const int lo = p.slab_lo[axis], hi = p.slab_hi[axis];
  if (coord < 0) return -1;
  if (coord < lo) return coord;
  const int hs = extent - hi;
  if (coord >= hs && coord < extent) return lo + coord - hs;
  return -1;
}

// psi = b psi + c d; returns d / kappa + psi (magnetic.cu:105-111)
__device__ __forceinline__ float psi_step(float d, float b, float c, float ik, const float* psi_in, float* psi_out,
                                          int off, bool write) {
  const float v = b * psi_in[off] + c * d;
  if (write) psi_out[off] = v;
  return d * ik + v;
}

// Same with the old psi value already loaded.
__device__ __forceinline__ float psi_apply(float d, float b, float c, float ik, float old, float* psi_out, int off,
                                           bool write) {
  const float v = b * old + c * d;
  if (write) psi_out[off] = v;
  return d * ik + v;
}

// Slab element offsets (32-bit: every engine array holds fewer than 2^31 elements).
__device__ __forceinline__ int xslab_off(const StepParams& p, int lx, int j, int k) { return (lx * p.NY + j) * p.P + k; }
__device__ __forceinline__ int yslab_off(const StepParams& p, int i, int ly, int k) {
  return (i * (p.slab_lo[1] + p.slab_hi[1]) + ly) * p.P + k;
}
// z slab: cell k (inside the low or high slab of its component) of row (i, j).
__device__ __forceinline__ int zslab_off(const StepParams& p, int i, int j, int k) {
  return (i * p.NY + j) * p.SZ + (k < p.zlo4 ? k : p.zlo4 + k - p.zhs4);
}

// True when the CSR list of `key` along `axis` holds at least one item.
__device__ __forceinline__ bool list_nonempty(const BoxIndex& ix, int axis, int key) {
  return __ldg(ix.ptr[axis] + key) < __ldg(ix.ptr[axis] + key + 1);
}

// Injection terms of one phase covering (i, j, k), scanning only the lists
// flagged non-empty; value added to component (comp - base).
__device__ __forceinline__ void add_terms(const StepParams& p, int phase, int base, int n, int i, int j, int k,
                                          bool sx, bool sy, bool sz, float& v0, float& v1, float& v2) {
  const BoxIndex& ix = p.term_index[phase];
  const int key[3] = {i, j, k};
  const bool scan[3] = {sx, sy, sz};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (!scan[a]) continue;
    const int b = __ldg(ix.ptr[a] + key[a]), e = __ldg(ix.ptr[a] + key[a] + 1);
    for (int x = b; x < e; ++x) {
      const InjectionTerm& t = p.terms[__ldg(ix.ids[a] + x)];
      if (i < t.i0 || i >= t.i1 || j < t.j0 || j >= t.j1 || k < t.k0 || k >= t.k1) continue;
      const int li = i - t.i0, lj = j - t.j0, lk = k - t.k0;
      float s;
      if (t.signal != nullptr) {
        s = __ldg(t.signal + n);
      } else {
        const int la = t.sample_axis == 0 ? li : (t.sample_axis == 1 ? lj : lk);
        s = __ldg(t.aux_hist + static_cast<int64_t>(n) * t.aux_len + __ldg(t.sample_index + la));
      }
      const float val = __ldg(t.coeff + (static_cast<int64_t>(li) * (t.j1 - t.j0) + lj) * (t.k1 - t.k0) + lk) * s * t.scale;
      const int c = t.comp - base;
      if (c == 0) v0 += val;
      else if (c == 1) v1 += val;
      else v2 += val;
    }
  }
}

// Advance the ADE poles covering (i, j, k) from E^n and subtract dt J / eps.
// `lane_poles` has bit b set when pole b (b < 32) covers this lane's (j, k);
// the plane list already restricts i.  Poles are taken three at a time with
// every state load issued before the first update, so the load latencies of a
// multi-component material overlap; the subtractions keep the list order.
#ifndef FDTD_ADE_BATCH
// Poles whose state loads are issued together.  1 in the 64-register kernel:
// a batch of three spills registers there and costs more than it hides.
#define FDTD_ADE_BATCH 1
#endif
// comp_mask: bit c set when component c is updated here (deferred wrap-face
// components are advanced by the wrap kernel instead).
template <typename TA = float>
__device__ __forceinline__ void ade(const StepParams& p, unsigned lane_poles, int i, int j, int k, float e0, float e1,
                                    float e2, float& v0, float& v1, float& v2, unsigned comp_mask = 7u) {
  constexpr int kB = FDTD_ADE_BATCH;
  const int b = __ldg(p.pole_plane_ptr + i), e = __ldg(p.pole_plane_ptr + i + 1);
  for (int x0 = b; x0 < e; x0 += kB) {
    const PoleTerm* pts[kB];
    int64_t offs[kB];
    bool act[kB];
    float drive[kB], ie[kB], pol[kB], cur[kB];
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      act[u] = false;
      pts[u] = p.poles;
      offs[u] = 0;
      drive[u] = ie[u] = pol[u] = cur[u] = 0.f;
      if (x0 + u < e) {
        const int id = __ldg(p.pole_plane_ids + x0 + u);
        const PoleTerm* pt = p.poles + id;
        act[u] = id < 32 ? ((lane_poles >> id) & 1u) != 0 : (j >= pt->j0 && j < pt->j1 && k >= pt->k0 && k < pt->k1);
        act[u] = act[u] && ((comp_mask >> pt->comp) & 1u);
        pts[u] = pt;
      }
      if (act[u]) {
        const PoleTerm& pt = *pts[u];
        const int64_t o =
            (static_cast<int64_t>(i - pt.i0) * (pt.j1 - pt.j0) + (j - pt.j0)) * pt.nkk + (k - pt.kk0);
        offs[u] = o;
        drive[u] = __ldg(pt.drive + o);
        ie[u] = __ldg(pt.inv_eps + o);
        if (pt.kind != 1) pol[u] = lda<TA>(pt.pol, o);
        if (pt.kind != 0) cur[u] = lda<TA>(pt.cur, o);
      }
    }
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      if (!act[u]) continue;
      const PoleTerm& pt = *pts[u];
      const int64_t o = offs[u];
      const int c = pt.comp;
      const float eo = c == 0 ? e0 : (c == 1 ? e1 : e2);
      float jn;
      if (pt.kind == 0) {
        const float prev = pol[u];
        const float next = pt.decay * prev + drive[u] * eo;
        sta<TA>(pt.pol, o, next);
        jn = (next - prev) * pt.inv_dt;
        sta<TA>(pt.cur, o, jn);
      } else if (pt.kind == 1) {
        jn = pt.decay * cur[u] + drive[u] * eo;
        sta<TA>(pt.cur, o, jn);
      } else {
        const float pl = pol[u];
        jn = pt.decay * cur[u] - pt.restoring * pl + drive[u] * eo;
        sta<TA>(pt.cur, o, jn);
        sta<TA>(pt.pol, o, pl + pt.dt * jn);
      }
      const float sub = pt.dt * jn * ie[u];
      if (c == 0) v0 -= sub;
      else if (c == 1) v1 -= sub;
      else v2 -= sub;
    }
  }
}

// E edge status (electric.cu:242-268): 0 update, 1 keep (NONE/PML edge),
// 2 PEC zero, 3 outside the Yee extent (stays zero), 4 deferred: a cell on a
// periodic or Bloch face, whose backward difference wraps to the far side of
// the grid; the step kernel leaves it (and its ADE state) alone and the wrap
// kernel (bloch.cu) updates it once the whole new H is in memory
// (electric.cu:133-168 bloch_backward_diff_axis, :23-40 boundary_diff_*).
constexpr int kModeDeferred = 4;
__host__ __device__ __forceinline__ bool wraps(int mode) { return mode == BND_PERIODIC || mode == BND_BLOCH; }
__device__ __forceinline__ int edge_mode(bool in_extent, bool alo, bool ahi, bool blo, bool bhi, int ma_lo, int ma_hi,
                                         int mb_lo, int mb_hi) {
  if (!in_extent) return 3;
  if ((alo && ma_lo == BND_PEC) || (ahi && ma_hi == BND_PEC) || (blo && mb_lo == BND_PEC) || (bhi && mb_hi == BND_PEC))
    return 2;
  if ((alo && wraps(ma_lo)) || (ahi && wraps(ma_hi)) || (blo && wraps(mb_lo)) || (bhi && wraps(mb_hi)))
    return kModeDeferred;
  return (alo || ahi || blo || bhi) ? 1 : 0;
}

__device__ __forceinline__ float pick(int mode, float updated, float old) {
  return mode == 0 ? updated : (mode == 1 ? old : 0.f);
}

// CPML profile values of one coordinate (b, c, 1/kappa).
struct Prof {
  float b, c, ik;
};
__device__ __forceinline__ Prof prof(const float* b, const float* c, const float* ik, int idx) {
  return {__ldg(b + idx), __ldg(c + idx), __ldg(ik + idx)};
}

// Lookup flags that do not change along the x march (bits of `lf`).
constexpr unsigned kLfHTermYm = 1u, kLfHTermYc = 2u, kLfHTermZ = 4u, kLfETermY = 8u, kLfETermZ = 16u;

}  // namespace

}  // namespace fdtdb200
