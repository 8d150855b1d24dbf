// z-vectorised fused leapfrog step: the warp-row decomposition of
// warp_kernel.cu with V (2 or 4) consecutive z cells per lane, so that every
// field, coefficient and x/y CPML access is one 8- or 16-byte load or store
// and the per-cell address, predicate and shuffle work is divided by V.
//
// Decomposition: a warp owns one y row j and 31 V consecutive z cells.  Lane l
// holds cells kb .. kb + V - 1 with kb = 31 V s - V + V l (s = blockIdx.y);
// lane 0 is the z halo group (its H feeds the first output cell's z-1
// neighbour, its E is not stored).  The warp marches +x over a chunk of planes
// exactly as the scalar kernel does: E^n(i+1) of rows j-1, j, j+1 is loaded
// once and reused as E^n(i) at the next plane, the halo row j-1 of Hx and Hz is
// recomputed, z+1 neighbours come from the next lane (and, for lane 31, from
// one extra scalar load), z-1 neighbours from the previous lane.
//
// Padded cells (z >= NZ inside the P-pitch row) are stored as zero; cells
// outside a component's Yee extent stay zero; CPML psi of masked cells keeps its
// old value.  ADE pole state is box-dense with its z range padded to multiples
// of four (kk0, nkk), so a lane group lies wholly inside or outside a pole box
// and the pole arrays are vector accesses too; padded pole cells have zero
// drive and zero 1/eps, so they stay zero and subtract exactly zero.
//
// Arithmetic restated from witwin/maxwell/fdtd/cuda/kernels/magnetic.cu:62-212,
// electric.cu:242-311 and 462-941, dispersive.cu:18-83, sources.cu:135-154 and
// 485-545; the per-cell expressions are those of warp_kernel.cu.
//
// Ring feed (D > 0): each warp streams its field rows through a private ring of
// D plane slots in shared memory with cp.async, D - 1 planes ahead of the math,
// so the DRAM latency of E(i+1) and H(i) is covered by the work of the planes
// in between without holding the prefetched values in registers.  A lane
// copies and reads only its own cells (and lane 31 its extra cells), so the
// per-thread cp.async groups order everything and no warp barrier is needed.
//
// This header is instantiated by the vec_*.cu files, one launch variant each.
#pragma once

#include "step_device.cuh"

namespace fdtdb200 {

namespace {

template <int V>
__device__ __forceinline__ void vld(float (&d)[V], const float* base, int off, bool ok) {
  if constexpr (V == 4) {
    float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ok) t = __ldg(reinterpret_cast<const float4*>(base + off));
    d[0] = t.x;
    d[1] = t.y;
    d[2] = t.z;
    d[3] = t.w;
  } else {
    float2 t = make_float2(0.f, 0.f);
    if (ok) t = __ldg(reinterpret_cast<const float2*>(base + off));
    d[0] = t.x;
    d[1] = t.y;
  }
}

// Coherent load for arrays this launch also writes (E psi, pole state).
template <int V>
__device__ __forceinline__ void vld_rw(float (&d)[V], const float* base, int off) {
  if constexpr (V == 4) {
    const float4 t = *reinterpret_cast<const float4*>(base + off);
    d[0] = t.x;
    d[1] = t.y;
    d[2] = t.z;
    d[3] = t.w;
  } else {
    const float2 t = *reinterpret_cast<const float2*>(base + off);
    d[0] = t.x;
    d[1] = t.y;
  }
}

// Streaming store of a field group (read again only by the next launch).
template <int V>
__device__ __forceinline__ void vst_cg(float* base, int off, const float (&s)[V]) {
  if constexpr (V == 4) __stcg(reinterpret_cast<float4*>(base + off), make_float4(s[0], s[1], s[2], s[3]));
  else __stcg(reinterpret_cast<float2*>(base + off), make_float2(s[0], s[1]));
}

template <int V>
__device__ __forceinline__ void vst(float* base, int off, const float (&s)[V]) {
  if constexpr (V == 4) *reinterpret_cast<float4*>(base + off) = make_float4(s[0], s[1], s[2], s[3]);
  else *reinterpret_cast<float2*>(base + off) = make_float2(s[0], s[1]);
}

template <int V>
__device__ __forceinline__ void vmask(float (&a)[V], unsigned bits) {
  if (bits != (1u << V) - 1u) {
#pragma unroll
    for (int t = 0; t < V; ++t)
      if (!((bits >> t) & 1u)) a[t] = 0.f;
  }
}

// Shared-memory ring slot of one warp: 13 rows of 32 V floats (E rows j-1
// x,y,z; j x,y,z; j+1 x,z; then H rows j-1 x,z; j x,y,z) and lane 31's three
// extra cells, padded to 16 bytes.
template <int V>
__host__ __device__ constexpr int ring_slot_floats() {
  return 13 * 32 * V + 4;
}

// cp.async of one lane group (V floats); zero-filled when !ok.
template <int V>
__device__ __forceinline__ void cpa(float* dst, const float* src, bool ok) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(src), "n"(V * 4), "r"(ok ? V * 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cpa1(float* dst, const float* src, bool ok) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int V>
__device__ __forceinline__ void sld(float (&d)[V], const float* s) {
  if constexpr (V == 4) {
    const float4 t = *reinterpret_cast<const float4*>(s);
    d[0] = t.x;
    d[1] = t.y;
    d[2] = t.z;
    d[3] = t.w;
  } else {
    const float2 t = *reinterpret_cast<const float2*>(s);
    d[0] = t.x;
    d[1] = t.y;
  }
}

// z+1 neighbours of a group: element t + 1, the next lane's first element,
// or (lane 31) the separately loaded cell after the warp's span.
template <int V>
__device__ __forceinline__ void zplus(const float (&a)[V], float extra, int lane, float (&out)[V]) {
  const float nx = __shfl_down_sync(kFull, a[0], 1);
#pragma unroll
  for (int t = 0; t + 1 < V; ++t) out[t] = a[t + 1];
  out[V - 1] = lane == 31 ? extra : nx;
}

// z-1 neighbours: element t - 1 or the previous lane's last element.
template <int V>
__device__ __forceinline__ void zminus(const float (&a)[V], float (&out)[V]) {
  out[0] = __shfl_up_sync(kFull, a[V - 1], 1);
#pragma unroll
  for (int t = 1; t < V; ++t) out[t] = a[t - 1];
}

// psi = b psi + c d; d <- d / kappa + psi on the cells of `bits`; psi of the
// other cells keeps its old value.  The old values come from `old`.
template <int V>
__device__ __forceinline__ void psi_apply_v(float (&d)[V], float b, float c, float ik, const float (&old)[V],
                                            float* out, int off, bool write, unsigned bits) {
  float st[V];
#pragma unroll
  for (int t = 0; t < V; ++t) {
    const float v = b * old[t] + c * d[t];
    const bool on = (bits >> t) & 1u;
    st[t] = on ? v : old[t];
    if (on) d[t] = d[t] * ik + v;
  }
  if (write) vst(out, off, st);
}

// Same with a per-cell profile (z slabs: b, c, 1/kappa vary along the group).
template <int V>
__device__ __forceinline__ void psi_apply_vz(float (&d)[V], const float (&b)[V], const float (&c)[V],
                                             const float (&ik)[V], const float (&old)[V], float* out, int off,
                                             bool write, unsigned bits) {
  float st[V];
#pragma unroll
  for (int t = 0; t < V; ++t) {
    const float v = b[t] * old[t] + c[t] * d[t];
    const bool on = (bits >> t) & 1u;
    st[t] = on ? v : old[t];
    if (on) d[t] = d[t] * ik[t] + v;
  }
  if (write) vst(out, off, st);
}

// In-place E psi recursion on the cells of `bits` (the cells being updated).
template <int V>
__device__ __forceinline__ void psi_step_v(float (&d)[V], float b, float c, float ik, float* psi, int off,
                                           unsigned bits) {
  float old[V];
  vld_rw(old, psi, off);
  psi_apply_v(d, b, c, ik, old, psi, off, true, bits);
}

// Injection terms of one phase covering the group (i, j, kb .. kb + V - 1);
// per cell the x-list, y-list and z-list contributions are added in the order
// of the scalar kernel's add_terms.
template <int V>
__device__ __forceinline__ void add_terms_v(const StepParams& p, int phase, int base, int n, int i, int j, int kb,
                                            bool sx, bool sy, unsigned zbits, float (&v0)[V], float (&v1)[V],
                                            float (&v2)[V]) {
  const BoxIndex& ix = p.term_index[phase];
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    if (!(a == 0 ? sx : sy)) continue;
    const int key = a == 0 ? i : j;
    const int b = __ldg(ix.ptr[a] + key), e = __ldg(ix.ptr[a] + key + 1);
    for (int x = b; x < e; ++x) {
      const InjectionTerm& t = p.terms[__ldg(ix.ids[a] + x)];
      if (i < t.i0 || i >= t.i1 || j < t.j0 || j >= t.j1 || kb + V <= t.k0 || kb >= t.k1) continue;
      const int li = i - t.i0, lj = j - t.j0;
      const int c = t.comp - base;
#pragma unroll
      for (int tt = 0; tt < V; ++tt) {
        const int k = kb + tt;
        if (k < t.k0 || k >= t.k1) continue;
        const int lk = k - t.k0;
        float s;
        if (t.signal != nullptr) {
          s = __ldg(t.signal + n);
        } else {
          const int la = t.sample_axis == 0 ? li : (t.sample_axis == 1 ? lj : lk);
          s = __ldg(t.aux_hist + static_cast<int64_t>(n) * t.aux_len + __ldg(t.sample_index + la));
        }
        const float val =
            __ldg(t.coeff + (static_cast<int64_t>(li) * (t.j1 - t.j0) + lj) * (t.k1 - t.k0) + lk) * s * t.scale;
        if (c == 0) v0[tt] += val;
        else if (c == 1) v1[tt] += val;
        else v2[tt] += val;
      }
    }
  }
  if (zbits) {
#pragma unroll
    for (int tt = 0; tt < V; ++tt) {
      if (!((zbits >> tt) & 1u)) continue;
      const int k = kb + tt;
      const int b = __ldg(ix.ptr[2] + k), e = __ldg(ix.ptr[2] + k + 1);
      for (int x = b; x < e; ++x) {
        const InjectionTerm& t = p.terms[__ldg(ix.ids[2] + x)];
        if (i < t.i0 || i >= t.i1 || j < t.j0 || j >= t.j1 || k < t.k0 || k >= t.k1) continue;
        const int li = i - t.i0, lj = j - t.j0, lk = k - t.k0;
        float s;
        if (t.signal != nullptr) {
          s = __ldg(t.signal + n);
        } else {
          const int la = t.sample_axis == 0 ? li : (t.sample_axis == 1 ? lj : lk);
          s = __ldg(t.aux_hist + static_cast<int64_t>(n) * t.aux_len + __ldg(t.sample_index + la));
        }
        const float val =
            __ldg(t.coeff + (static_cast<int64_t>(li) * (t.j1 - t.j0) + lj) * (t.k1 - t.k0) + lk) * s * t.scale;
        const int c = t.comp - base;
        if (c == 0) v0[tt] += val;
        else if (c == 1) v1[tt] += val;
        else v2[tt] += val;
      }
    }
  }
}

// ADE poles of plane i covering the group: advance from E^n and subtract
// dt J / eps (dispersive.cu:18-83).  `lane_poles` bit b: pole b (< 32) covers
// this lane's (j, group).  Poles are taken three at a time with every state
// load issued before the first update, so their latencies overlap; the
// subtractions keep the list order.
template <int V>
__device__ __forceinline__ void ade_v(const StepParams& p, unsigned lane_poles, int i, int j, int kb,
                                      const float (&e0)[V], const float (&e1)[V], const float (&e2)[V],
                                      float (&v0)[V], float (&v1)[V], float (&v2)[V]) {
  constexpr int kB = 3;
  const int b = __ldg(p.pole_plane_ptr + i), e = __ldg(p.pole_plane_ptr + i + 1);
  for (int x0 = b; x0 < e; x0 += kB) {
    const PoleTerm* pts[kB];
    int offs[kB];
    bool act[kB];
    float drive[kB][V], ie[kB][V], pol[kB][V], cur[kB][V];
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      act[u] = false;
      pts[u] = p.poles;
      offs[u] = 0;
      if (x0 + u < e) {
        const int id = __ldg(p.pole_plane_ids + x0 + u);
        const PoleTerm* pt = p.poles + id;
        act[u] = id < 32 ? ((lane_poles >> id) & 1u) != 0
                         : (j >= pt->j0 && j < pt->j1 && kb >= pt->kk0 && kb < pt->kk0 + pt->nkk);
        pts[u] = pt;
      }
      if (act[u]) {
        const PoleTerm& pt = *pts[u];
        const int o = ((i - pt.i0) * (pt.j1 - pt.j0) + (j - pt.j0)) * pt.nkk + (kb - pt.kk0);
        offs[u] = o;
        vld(drive[u], pt.drive, o, true);
        vld(ie[u], pt.inv_eps, o, true);
        if (pt.kind != 1) vld_rw(pol[u], pt.pol, o);
        if (pt.kind != 0) vld_rw(cur[u], pt.cur, o);
      }
    }
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      if (!act[u]) continue;
      const PoleTerm& pt = *pts[u];
      const int o = offs[u];
      const int c = pt.comp;
      float jn[V];
      if (pt.kind == 0) {
        float next[V];
#pragma unroll
        for (int t = 0; t < V; ++t) {
          const float eo = c == 0 ? e0[t] : (c == 1 ? e1[t] : e2[t]);
          next[t] = pt.decay * pol[u][t] + drive[u][t] * eo;
          jn[t] = (next[t] - pol[u][t]) * pt.inv_dt;
        }
        vst(pt.pol, o, next);
        vst(pt.cur, o, jn);
      } else if (pt.kind == 1) {
#pragma unroll
        for (int t = 0; t < V; ++t) {
          const float eo = c == 0 ? e0[t] : (c == 1 ? e1[t] : e2[t]);
          jn[t] = pt.decay * cur[u][t] + drive[u][t] * eo;
        }
        vst(pt.cur, o, jn);
      } else {
        float pn[V];
#pragma unroll
        for (int t = 0; t < V; ++t) {
          const float eo = c == 0 ? e0[t] : (c == 1 ? e1[t] : e2[t]);
          jn[t] = pt.decay * cur[u][t] - pt.restoring * pol[u][t] + drive[u][t] * eo;
          pn[t] = pol[u][t] + pt.dt * jn[t];
        }
        vst(pt.cur, o, jn);
        vst(pt.pol, o, pn);
      }
#pragma unroll
      for (int t = 0; t < V; ++t) {
        const float sub = pt.dt * jn[t] * ie[u][t];
        if (c == 0) v0[t] -= sub;
        else if (c == 1) v1[t] -= sub;
        else v2[t] -= sub;
      }
    }
  }
}

// The march of one warp task (row j, z block blockIdx.y, x chunk blockIdx.z).
template <int V, int D, bool kCpml, bool kCoef, bool kUniform>
__device__ __forceinline__ void vmarch(const StepParams& p, int n, int lane, int j) {
  constexpr unsigned kAll = (1u << V) - 1u;
  const int NX = p.NX, NY = p.NY, NZ = p.NZ, P = p.P;
  const int kb = blockIdx.y * (31 * V) - V + V * lane;
  const bool kin = kb >= 0 && kb < P;
  const bool out_lane = lane >= 1 && kin;
  const int i0 = blockIdx.z * p.CX;
  const int i1 = min(i0 + p.CX, NX);
  const int istart = max(i0 - 1, 0);
  const bool jm_ok = j >= 1, jp_ok = j + 1 < NY;
  const int jm = jm_ok ? j - 1 : 0, jp = jp_ok ? j + 1 : 0;
  const int kc = kin ? kb : 0;
  const int ps = NY * P;
  const int rm = jm * P + kc, rc = j * P + kc, rp = jp * P + kc;
  const bool xk = lane == 31 && kin && kb + V < P;  // lane 31 loads the cell after the span

  // per-cell z extents: bit t <-> cell kb + t inside NZ - 1 (Hx, Hy, Ez) / NZ (Ex, Ey, Hz)
  unsigned hzm = 0, ezm = 0;
#pragma unroll
  for (int t = 0; t < V; ++t) {
    const int k = kb + t;
    if (k >= 0 && k < NZ - 1) hzm |= 1u << t;
    if (k >= 0 && k < NZ) ezm |= 1u << t;
  }
  const bool yc_ok = j < NY - 1;
  float ihz[V], iez[V];
#pragma unroll
  for (int t = 0; t < V; ++t) {
    ihz[t] = kUniform ? p.inv_h_u[2] : __ldg(p.inv_h[2] + (((hzm >> t) & 1u) ? kb + t : 0));
    iez[t] = kUniform ? p.inv_e_u[2] : __ldg(p.inv_e[2] + (((ezm >> t) & 1u) ? kb + t : 0));
  }
  const float ihy_m = kUniform ? p.inv_h_u[1] : __ldg(p.inv_h[1] + jm);
  const float ihy_c = kUniform ? p.inv_h_u[1] : __ldg(p.inv_h[1] + (yc_ok ? j : 0));
  const float iey = kUniform ? p.inv_e_u[1] : __ldg(p.inv_e[1] + j);
  const bool ylo = j == 0, yhi = j == NY - 1;
  const bool lane_edge = ylo || yhi || hzm != kAll || kb == 0;
  int syh_m = -1, syh_c = -1, sye = -1;
  bool y_slab = false;
  // z slabs: bit t of zbh / zbe <-> cell kb + t lies in the z slab of the H
  // (extent NZ - 1) / E (extent NZ) components; the group's psi is one vector
  // at zslab_off(kb).  The group's z profile is re-read per plane (L1 hits).
  unsigned zbh = 0, zbe = 0;
  if (kCpml) {
    syh_m = jm_ok ? slab_coord(p, 1, jm, NY - 1) : -1;
    syh_c = slab_coord(p, 1, j, NY - 1);
    sye = slab_coord(p, 1, j, NY);
    y_slab = syh_m >= 0 || syh_c >= 0 || sye >= 0;
    if (kin && (kb < p.zlo4 || kb >= p.zhs4)) {
#pragma unroll
      for (int t = 0; t < V; ++t) {
        if (slab_coord(p, 2, kb + t, NZ - 1) >= 0) zbh |= 1u << t;
        if (slab_coord(p, 2, kb + t, NZ) >= 0) zbe |= 1u << t;
      }
    }
  }
  // first z cell of the group inside the padded slab segment (profile index base)
  const int kzb = (zbh | zbe) ? kb : 0;
  unsigned lf = 0, zh = 0, ze = 0;
  if (p.n_terms[1]) {
    if (jm_ok && list_nonempty(p.term_index[1], 1, jm)) lf |= kLfHTermYm;
    if (list_nonempty(p.term_index[1], 1, j)) lf |= kLfHTermYc;
    if (kin) {
#pragma unroll
      for (int t = 0; t < V; ++t)
        if (list_nonempty(p.term_index[1], 2, kb + t)) zh |= 1u << t;
    }
  }
  if (p.n_terms[0]) {
    if (list_nonempty(p.term_index[0], 1, j)) lf |= kLfETermY;
    if (kin) {
#pragma unroll
      for (int t = 0; t < V; ++t)
        if (list_nonempty(p.term_index[0], 2, kb + t)) ze |= 1u << t;
    }
  }
  unsigned lane_poles = 0;
  if (p.n_poles && out_lane) {
    const int np_ = min(p.n_poles, 32);
    for (int b = 0; b < np_; ++b) {
      const PoleTerm& pt = p.poles[b];
      if (j >= pt.j0 && j < pt.j1 && kb >= pt.kk0 && kb < pt.kk0 + pt.nkk) lane_poles |= 1u << b;
    }
  }

  // Ring feed: group q copies the E rows of plane q (q < NX) and the H rows of
  // plane q (q < i1) into slot q % D.
  constexpr int kSlot = ring_slot_floats<V>();
  constexpr int kRow = 32 * V;
  float* ring = nullptr;
  if constexpr (D > 0) {
    extern __shared__ __align__(16) float vec_smem[];
    ring = vec_smem + (threadIdx.x >> 5) * (D * kSlot);
  }
  const int lo = lane * V;
  auto issue = [&](int q) {
    if constexpr (D > 0) {
      if (q < NX && q <= i1) {
        float* s = ring + (q % D) * kSlot;
        const int oq = q * ps;
        cpa<V>(s + 0 * kRow + lo, p.Ein[0] + oq + rm, kin && jm_ok);
        cpa<V>(s + 1 * kRow + lo, p.Ein[1] + oq + rm, kin && jm_ok);
        cpa<V>(s + 2 * kRow + lo, p.Ein[2] + oq + rm, kin && jm_ok);
        cpa<V>(s + 3 * kRow + lo, p.Ein[0] + oq + rc, kin);
        cpa<V>(s + 4 * kRow + lo, p.Ein[1] + oq + rc, kin);
        cpa<V>(s + 5 * kRow + lo, p.Ein[2] + oq + rc, kin);
        cpa<V>(s + 6 * kRow + lo, p.Ein[0] + oq + rp, kin && jp_ok);
        cpa<V>(s + 7 * kRow + lo, p.Ein[2] + oq + rp, kin && jp_ok);
        if (q < i1) {
          cpa<V>(s + 8 * kRow + lo, p.Hin[0] + oq + rm, kin && jm_ok);
          cpa<V>(s + 9 * kRow + lo, p.Hin[2] + oq + rm, kin && jm_ok);
          cpa<V>(s + 10 * kRow + lo, p.Hin[0] + oq + rc, kin);
          cpa<V>(s + 11 * kRow + lo, p.Hin[1] + oq + rc, kin);
          cpa<V>(s + 12 * kRow + lo, p.Hin[2] + oq + rc, kin);
        }
        if (lane == 31) {
          cpa1(s + 13 * kRow + 0, p.Ein[1] + oq + (xk ? rm + V : 0), xk && jm_ok);
          cpa1(s + 13 * kRow + 1, p.Ein[0] + oq + (xk ? rc + V : 0), xk);
          cpa1(s + 13 * kRow + 2, p.Ein[1] + oq + (xk ? rc + V : 0), xk);
        }
      }
      cpa_commit();
    }
  };

  // E^n(i): row j-1 (x, y, z), row j (x, y, z), row j+1 (x, z); lane 31's extra z+1 cells
  float em0[V], em1[V], em2[V], ec0[V], ec1[V], ec2[V], ep0[V], ep2[V];
  float xem1 = 0.f, xec0 = 0.f, xec1 = 0.f;
  if constexpr (D > 0) {
#pragma unroll
    for (int q = 0; q < D; ++q) issue(istart + q);
    cpa_wait<D - 1>();
    const float* s = ring + (istart % D) * kSlot;
    sld(em0, s + 0 * kRow + lo);
    sld(em1, s + 1 * kRow + lo);
    sld(em2, s + 2 * kRow + lo);
    sld(ec0, s + 3 * kRow + lo);
    sld(ec1, s + 4 * kRow + lo);
    sld(ec2, s + 5 * kRow + lo);
    sld(ep0, s + 6 * kRow + lo);
    sld(ep2, s + 7 * kRow + lo);
    if (lane == 31) {
      xem1 = s[13 * kRow + 0];
      xec0 = s[13 * kRow + 1];
      xec1 = s[13 * kRow + 2];
    }
  } else {
    const int o = istart * ps;
    vld(em0, p.Ein[0], o + rm, kin && jm_ok);
    vld(em1, p.Ein[1], o + rm, kin && jm_ok);
    vld(em2, p.Ein[2], o + rm, kin && jm_ok);
    vld(ec0, p.Ein[0], o + rc, kin);
    vld(ec1, p.Ein[1], o + rc, kin);
    vld(ec2, p.Ein[2], o + rc, kin);
    vld(ep0, p.Ein[0], o + rp, kin && jp_ok);
    vld(ep2, p.Ein[2], o + rp, kin && jp_ok);
    if (xk) {
      xem1 = jm_ok ? __ldg(p.Ein[1] + o + rm + V) : 0.f;
      xec0 = __ldg(p.Ein[0] + o + rc + V);
      xec1 = __ldg(p.Ein[1] + o + rc + V);
    }
  }
  float hpz[V], hpy[V];  // Hz, Hy of row j at plane i-1
#pragma unroll
  for (int t = 0; t < V; ++t) hpz[t] = hpy[t] = 0.f;

  for (int i = istart; i < i1; ++i) {
    const bool own = i >= i0;
    const bool inext = i + 1 < NX;
    const int o = i * ps;
    const int on = o + ps;
    const unsigned pb = __ldg(p.plane_bits + i);
    float nm0[V], nm1[V], nm2[V], nc0[V], nc1[V], nc2[V], np0[V], np2[V];
    float xnm1 = 0.f, xnc0 = 0.f, xnc1 = 0.f;
    float hm0[V], hm2[V], hc0[V], hc1[V], hc2[V];
    if constexpr (D > 0) {
      cpa_wait<D - 2>();  // groups up to plane i + 1 have landed
      if (inext) {
        const float* s = ring + ((i + 1) % D) * kSlot;
        sld(nm0, s + 0 * kRow + lo);
        sld(nm1, s + 1 * kRow + lo);
        sld(nm2, s + 2 * kRow + lo);
        sld(nc0, s + 3 * kRow + lo);
        sld(nc1, s + 4 * kRow + lo);
        sld(nc2, s + 5 * kRow + lo);
        sld(np0, s + 6 * kRow + lo);
        sld(np2, s + 7 * kRow + lo);
        if (lane == 31) {
          xnm1 = s[13 * kRow + 0];
          xnc0 = s[13 * kRow + 1];
          xnc1 = s[13 * kRow + 2];
        }
      } else {
#pragma unroll
        for (int t = 0; t < V; ++t) nm0[t] = nm1[t] = nm2[t] = nc0[t] = nc1[t] = nc2[t] = np0[t] = np2[t] = 0.f;
      }
      const float* s = ring + (i % D) * kSlot;
      sld(hm0, s + 8 * kRow + lo);
      sld(hm2, s + 9 * kRow + lo);
      sld(hc0, s + 10 * kRow + lo);
      sld(hc1, s + 11 * kRow + lo);
      sld(hc2, s + 12 * kRow + lo);
    } else {
      vld(nm0, p.Ein[0], on + rm, kin && jm_ok && inext);
      vld(nm1, p.Ein[1], on + rm, kin && jm_ok && inext);
      vld(nm2, p.Ein[2], on + rm, kin && jm_ok && inext);
      vld(nc0, p.Ein[0], on + rc, kin && inext);
      vld(nc1, p.Ein[1], on + rc, kin && inext);
      vld(nc2, p.Ein[2], on + rc, kin && inext);
      vld(np0, p.Ein[0], on + rp, kin && jp_ok && inext);
      vld(np2, p.Ein[2], on + rp, kin && jp_ok && inext);
      if (xk && inext) {
        xnm1 = jm_ok ? __ldg(p.Ein[1] + on + rm + V) : 0.f;
        xnc0 = __ldg(p.Ein[0] + on + rc + V);
        xnc1 = __ldg(p.Ein[1] + on + rc + V);
      }
      vld(hm0, p.Hin[0], o + rm, kin && jm_ok);
      vld(hm2, p.Hin[2], o + rm, kin && jm_ok);
      vld(hc0, p.Hin[0], o + rc, kin);
      vld(hc1, p.Hin[1], o + rc, kin);
      vld(hc2, p.Hin[2], o + rc, kin);
    }
    const bool ix_ok = i < NX - 1;
    // cells whose H value exists: halo row Hx, Hz; row j Hx, Hy, Hz
    const unsigned mxb_ = jm_ok ? hzm : 0u, mzb_ = (jm_ok && ix_ok) ? ezm : 0u;
    const unsigned cxb_ = yc_ok ? hzm : 0u, cyb_ = ix_ok ? hzm : 0u, czb_ = (ix_ok && yc_ok) ? ezm : 0u;
    int sxh = -1, sxe = -1;
    float qx0[V], qx1[V], qx2[V], qy0[V], qy1[V], qy2[V], qy3[V], qz0[V], qz1[V], qz2[V];
    if (kCpml) {
      if (zbh) {
        vld(qz0, p.psiHin[0][1], zslab_off(p, i, jm, kb), jm_ok);
        vld(qz1, p.psiHin[0][1], zslab_off(p, i, j, kb), true);
        vld(qz2, p.psiHin[1][1], zslab_off(p, i, j, kb), true);
      }
      sxh = slab_coord(p, 0, i, NX - 1);
      sxe = slab_coord(p, 0, i, NX);
      if (sxh >= 0) {
        vld(qx0, p.psiHin[2][0], xslab_off(p, sxh, jm, kc), kin && jm_ok);
        vld(qx1, p.psiHin[1][0], xslab_off(p, sxh, j, kc), kin);
        vld(qx2, p.psiHin[2][0], xslab_off(p, sxh, j, kc), kin);
      }
      if (syh_m >= 0) {
        vld(qy0, p.psiHin[0][0], yslab_off(p, i, syh_m, kc), kin);
        vld(qy1, p.psiHin[2][1], yslab_off(p, i, syh_m, kc), kin);
      }
      if (syh_c >= 0) {
        vld(qy2, p.psiHin[0][0], yslab_off(p, i, syh_c, kc), kin);
        vld(qy3, p.psiHin[2][1], yslab_off(p, i, syh_c, kc), kin);
      }
    }
    float g0[V], g1[V], g2[V], c0[V], c1[V], c2[V];
#pragma unroll
    for (int t = 0; t < V; ++t) {
      g0[t] = p.edecay_u[0];
      g1[t] = p.edecay_u[1];
      g2[t] = p.edecay_u[2];
      c0[t] = p.ecurl_u[0];
      c1[t] = p.ecurl_u[1];
      c2[t] = p.ecurl_u[2];
    }
    if (kCoef) {
      const bool ld = own && out_lane;
      if (p.ecurl[0]) vld(c0, p.ecurl[0], o + rc, ld);
      if (p.ecurl[1]) vld(c1, p.ecurl[1], o + rc, ld);
      if (p.ecurl[2]) vld(c2, p.ecurl[2], o + rc, ld);
      if (p.edecay[0]) vld(g0, p.edecay[0], o + rc, ld);
      if (p.edecay[1]) vld(g1, p.edecay[1], o + rc, ld);
      if (p.edecay[2]) vld(g2, p.edecay[2], o + rc, ld);
    }
    const float ihx = kUniform ? p.inv_h_u[0] : __ldg(p.inv_h[0] + (ix_ok ? i : 0));
    float em1k[V], ec0k[V], ec1k[V];
    zplus(em1, xem1, lane, em1k);
    zplus(ec0, xec0, lane, ec0k);
    zplus(ec1, xec1, lane, ec1k);

    // ---------------- H^{n+1/2}(i): halo row j-1 (Hx, Hz), then row j ----------------
    float mxa[V], mxb[V], mza[V], mzb[V], cxa[V], cxb[V], cya[V], cyb[V], cza[V], czb[V];
#pragma unroll
    for (int t = 0; t < V; ++t) {
      mxa[t] = (ec2[t] - em2[t]) * ihy_m;
      mxb[t] = (em1k[t] - em1[t]) * ihz[t];
      mza[t] = (nm1[t] - em1[t]) * ihx;
      mzb[t] = (ec0[t] - em0[t]) * ihy_m;
      cxa[t] = (ep2[t] - ec2[t]) * ihy_c;
      cxb[t] = (ec1k[t] - ec1[t]) * ihz[t];
      cya[t] = (nc2[t] - ec2[t]) * ihx;
      cyb[t] = (ec0k[t] - ec0[t]) * ihz[t];
      cza[t] = (nc1[t] - ec1[t]) * ihx;
      czb[t] = (ep0[t] - ec0[t]) * ihy_c;
    }
    if (kCpml) {
      const bool wr = own && out_lane;
      if (sxh >= 0) {  // plane inside an x slab: uniform over the warp
        const Prof px = prof(p.hb[0], p.hc[0], p.hik[0], i);
        psi_apply_v(mza, px.b, px.c, px.ik, qx0, p.psiHout[2][0], 0, false, mzb_);
        psi_apply_v(cya, px.b, px.c, px.ik, qx1, p.psiHout[1][0], xslab_off(p, sxh, j, kc), wr, cyb_);
        psi_apply_v(cza, px.b, px.c, px.ik, qx2, p.psiHout[2][0], xslab_off(p, sxh, j, kc), wr, czb_);
      }
      if (y_slab) {
        if (syh_m >= 0) {
          const Prof py = prof(p.hb[1], p.hc[1], p.hik[1], jm);
          psi_apply_v(mxa, py.b, py.c, py.ik, qy0, p.psiHout[0][0], 0, false, mxb_);
          psi_apply_v(mzb, py.b, py.c, py.ik, qy1, p.psiHout[2][1], 0, false, mzb_);
        }
        if (syh_c >= 0) {
          const Prof py = prof(p.hb[1], p.hc[1], p.hik[1], j);
          psi_apply_v(cxa, py.b, py.c, py.ik, qy2, p.psiHout[0][0], yslab_off(p, i, syh_c, kc), wr, cxb_);
          psi_apply_v(czb, py.b, py.c, py.ik, qy3, p.psiHout[2][1], yslab_off(p, i, syh_c, kc), wr, czb_);
        }
      }
      if (zbh) {
        const int zo = zslab_off(p, i, j, kb);
        float bzh[V], czh[V], ikzh[V];
#pragma unroll
        for (int t = 0; t < V; ++t) {
          const int kz = ((zbh >> t) & 1u) ? kzb + t : 0;
          bzh[t] = __ldg(p.hb[2] + kz);
          czh[t] = __ldg(p.hc[2] + kz);
          ikzh[t] = __ldg(p.hik[2] + kz);
        }
        psi_apply_vz(mxb, bzh, czh, ikzh, qz0, p.psiHout[0][1], 0, false, mxb_ & zbh);
        psi_apply_vz(cxb, bzh, czh, ikzh, qz1, p.psiHout[0][1], zo, wr, cxb_ & zbh);
        psi_apply_vz(cyb, bzh, czh, ikzh, qz2, p.psiHout[1][1], zo, wr, cyb_ & zbh);
      }
    }
    float dHx[V], cHx[V], dHy[V], cHy[V], dHz[V], cHz[V], dHxm[V], cHxm[V], dHzm[V], cHzm[V];
#pragma unroll
    for (int t = 0; t < V; ++t) {
      dHx[t] = dHxm[t] = p.hdecay_u[0];
      cHx[t] = cHxm[t] = p.hcurl_u[0];
      dHy[t] = p.hdecay_u[1];
      cHy[t] = p.hcurl_u[1];
      dHz[t] = dHzm[t] = p.hdecay_u[2];
      cHz[t] = cHzm[t] = p.hcurl_u[2];
    }
    if (kCoef) {
      if (p.hdecay[0]) { vld(dHx, p.hdecay[0], o + rc, kin); vld(dHxm, p.hdecay[0], o + rm, kin && jm_ok); }
      if (p.hcurl[0]) { vld(cHx, p.hcurl[0], o + rc, kin); vld(cHxm, p.hcurl[0], o + rm, kin && jm_ok); }
      if (p.hdecay[1]) vld(dHy, p.hdecay[1], o + rc, kin);
      if (p.hcurl[1]) vld(cHy, p.hcurl[1], o + rc, kin);
      if (p.hdecay[2]) { vld(dHz, p.hdecay[2], o + rc, kin); vld(dHzm, p.hdecay[2], o + rm, kin && jm_ok); }
      if (p.hcurl[2]) { vld(cHz, p.hcurl[2], o + rc, kin); vld(cHzm, p.hcurl[2], o + rm, kin && jm_ok); }
    }
    float hmx[V], hmy[V], hmz[V], hcx[V], hcy[V], hcz[V];
#pragma unroll
    for (int t = 0; t < V; ++t) {
      hmx[t] = hm0[t] * dHxm[t] - cHxm[t] * (mxa[t] - mxb[t]);
      hmy[t] = 0.f;
      hmz[t] = hm2[t] * dHzm[t] - cHzm[t] * (mza[t] - mzb[t]);
      hcx[t] = hc0[t] * dHx[t] - cHx[t] * (cxa[t] - cxb[t]);
      hcy[t] = hc1[t] * dHy[t] - cHy[t] * (cyb[t] - cya[t]);
      hcz[t] = hc2[t] * dHz[t] - cHz[t] * (cza[t] - czb[t]);
    }
    vmask(hmx, mxb_);
    vmask(hmz, mzb_);
    vmask(hcx, cxb_);
    vmask(hcy, cyb_);
    vmask(hcz, czb_);
    // TFSF magnetic corrections, also on the halo row so it equals the owner's value
    if (kin && ((pb & kPlaneHTerms) || (lf & (kLfHTermYm | kLfHTermYc)) || zh)) {
      if (jm_ok) add_terms_v(p, 1, 3, n, i, jm, kb, pb & kPlaneHTerms, lf & kLfHTermYm, zh, hmx, hmy, hmz);
      add_terms_v(p, 1, 3, n, i, j, kb, pb & kPlaneHTerms, lf & kLfHTermYc, zh, hcx, hcy, hcz);
    }
    if (own && out_lane) {
      vst_cg(p.Hout[0], o + rc, hcx);
      vst_cg(p.Hout[1], o + rc, hcy);
      vst_cg(p.Hout[2], o + rc, hcz);
    }

    // ---------------- E^{n+1}(i), row j ----------------
    float hxk[V], hyk[V];
    zminus(hcx, hxk);
    zminus(hcy, hyk);
    if (own && out_lane) {
      const float iex = kUniform ? p.inv_e_u[0] : __ldg(p.inv_e[0] + i);
      float d0a[V], d0b[V], d1a[V], d1b[V], d2a[V], d2b[V];
#pragma unroll
      for (int t = 0; t < V; ++t) {
        d0a[t] = (hcz[t] - hmz[t]) * iey;
        d0b[t] = (hcy[t] - hyk[t]) * iez[t];
        d1a[t] = (hcz[t] - hpz[t]) * iex;
        d1b[t] = (hcx[t] - hxk[t]) * iez[t];
        d2a[t] = (hcy[t] - hpy[t]) * iex;
        d2b[t] = (hcx[t] - hmx[t]) * iey;
      }
      // per-cell edge status (electric.cu:242-268): u* = updated, k* = kept
      unsigned u0 = kAll, u1 = kAll, u2 = kAll, k0 = 0, k1 = 0, k2 = 0;
      if (lane_edge || i == 0 || i == NX - 1) {
        const bool xlo = i == 0, xhi = i == NX - 1;
        u0 = u1 = u2 = 0;
#pragma unroll
        for (int t = 0; t < V; ++t) {
          const int k = kb + t;
          const bool zlo = k == 0, zhi = k == NZ - 1;
          const bool ezk = (ezm >> t) & 1u, hzk = (hzm >> t) & 1u;
          const int m0 = edge_mode(ix_ok && ezk, ylo, yhi, zlo, zhi, p.bnd[2], p.bnd[3], p.bnd[4], p.bnd[5]);
          const int m1 = edge_mode(yc_ok && ezk, xlo, xhi, zlo, zhi, p.bnd[0], p.bnd[1], p.bnd[4], p.bnd[5]);
          const int m2 = edge_mode(hzk, xlo, xhi, ylo, yhi, p.bnd[0], p.bnd[1], p.bnd[2], p.bnd[3]);
          u0 |= (m0 == 0 ? 1u : 0u) << t;
          u1 |= (m1 == 0 ? 1u : 0u) << t;
          u2 |= (m2 == 0 ? 1u : 0u) << t;
          k0 |= (m0 == 1 ? 1u : 0u) << t;
          k1 |= (m1 == 1 ? 1u : 0u) << t;
          k2 |= (m2 == 1 ? 1u : 0u) << t;
        }
      }
      if (kCpml) {
        if (sxe >= 0) {
          const Prof px = prof(p.eb[0], p.ec[0], p.eik[0], i);
          psi_step_v(d1a, px.b, px.c, px.ik, p.psiE[1][0], xslab_off(p, sxe, j, kc), u1);
          psi_step_v(d2a, px.b, px.c, px.ik, p.psiE[2][0], xslab_off(p, sxe, j, kc), u2);
        }
        if (sye >= 0) {
          const Prof py = prof(p.eb[1], p.ec[1], p.eik[1], j);
          psi_step_v(d0a, py.b, py.c, py.ik, p.psiE[0][0], yslab_off(p, i, sye, kc), u0);
          psi_step_v(d2b, py.b, py.c, py.ik, p.psiE[2][1], yslab_off(p, i, sye, kc), u2);
        }
        if (zbe) {
          const int zo = zslab_off(p, i, j, kb);
          float bze[V], cze[V], ikze[V];
#pragma unroll
          for (int t = 0; t < V; ++t) {
            const int kz = ((zbe >> t) & 1u) ? kzb + t : 0;
            bze[t] = __ldg(p.eb[2] + kz);
            cze[t] = __ldg(p.ec[2] + kz);
            ikze[t] = __ldg(p.eik[2] + kz);
          }
          float o0[V], o1[V];
          vld_rw(o0, p.psiE[0][1], zo);
          vld_rw(o1, p.psiE[1][1], zo);
          psi_apply_vz(d0b, bze, cze, ikze, o0, p.psiE[0][1], zo, true, u0 & zbe);
          psi_apply_vz(d1b, bze, cze, ikze, o1, p.psiE[1][1], zo, true, u1 & zbe);
        }
      }
      float v0[V], v1[V], v2[V];
#pragma unroll
      for (int t = 0; t < V; ++t) {
        v0[t] = ec0[t] * g0[t] + c0[t] * (d0a[t] - d0b[t]);
        v1[t] = ec1[t] * g1[t] + c1[t] * (d1b[t] - d1a[t]);
        v2[t] = ec2[t] * g2[t] + c2[t] * (d2a[t] - d2b[t]);
      }
      if ((u0 & u1 & u2) != kAll) {
#pragma unroll
        for (int t = 0; t < V; ++t) {
          v0[t] = ((u0 >> t) & 1u) ? v0[t] : (((k0 >> t) & 1u) ? ec0[t] : 0.f);
          v1[t] = ((u1 >> t) & 1u) ? v1[t] : (((k1 >> t) & 1u) ? ec1[t] : 0.f);
          v2[t] = ((u2 >> t) & 1u) ? v2[t] : (((k2 >> t) & 1u) ? ec2[t] : 0.f);
        }
      }
      // ADE subtraction, TFSF electric corrections and soft sources: the
      // additive terms of witwin/maxwell/fdtd/runtime/stepping.py:2295-2320.
      if ((pb & kPlanePoles) && lane_poles) ade_v(p, lane_poles, i, j, kb, ec0, ec1, ec2, v0, v1, v2);
      if ((pb & kPlaneETerms) || (lf & kLfETermY) || ze)
        add_terms_v(p, 0, 0, n, i, j, kb, pb & kPlaneETerms, lf & kLfETermY, ze, v0, v1, v2);
      // scenes without TFSF end the E update on PEC faces (stepping.py:2316-2318):
      // cells neither updated nor kept are PEC (or outside the extent, zero anyway)
      if (p.pec_clamp && (u0 & u1 & u2) != kAll) {
#pragma unroll
        for (int t = 0; t < V; ++t) {
          if (!((u0 | k0) >> t & 1u)) v0[t] = 0.f;
          if (!((u1 | k1) >> t & 1u)) v1[t] = 0.f;
          if (!((u2 | k2) >> t & 1u)) v2[t] = 0.f;
        }
      }
      vst_cg(p.Eout[0], o + rc, v0);
      vst_cg(p.Eout[1], o + rc, v1);
      vst_cg(p.Eout[2], o + rc, v2);
    }
#pragma unroll
    for (int t = 0; t < V; ++t) {
      hpz[t] = hcz[t];
      hpy[t] = hcy[t];
      em0[t] = nm0[t];
      em1[t] = nm1[t];
      em2[t] = nm2[t];
      ec0[t] = nc0[t];
      ec1[t] = nc1[t];
      ec2[t] = nc2[t];
      ep0[t] = np0[t];
      ep2[t] = np2[t];
    }
    xem1 = xnm1;
    xec0 = xnc0;
    xec1 = xnc1;
    issue(i + D);  // slot i % D is consumed: refill it with plane i + D
  }
}

// Footprint class of each warp task of the vectorised kernel (see
// classify_kernel in warp_kernel.cu): planes [istart, i1), rows j-1 and j,
// cells kb .. kb + V - 1 of every lane.
template <int V>
__global__ void classify_vec_kernel(const StepParams p, int n_kblocks, int n_chunks, unsigned char* out) {
  const int lane = threadIdx.x & 31;
  const int64_t task = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int NX = p.NX, NY = p.NY, NZ = p.NZ, P = p.P;
  if (task >= static_cast<int64_t>(n_chunks) * n_kblocks * NY) return;
  const int j = static_cast<int>(task % NY);
  const int s = static_cast<int>((task / NY) % n_kblocks);
  const int c = static_cast<int>(task / (static_cast<int64_t>(NY) * n_kblocks));
  const int kb = s * (31 * V) - V + V * lane;
  const int i0 = c * p.CX, i1 = min(i0 + p.CX, NX), istart = max(i0 - 1, 0);
  const int jm = j >= 1 ? j - 1 : j;
  bool cpml = false, coef = false;
  if (p.cpml) {
    cpml = slab_coord(p, 1, jm, NY - 1) >= 0 || slab_coord(p, 1, j, NY - 1) >= 0 || slab_coord(p, 1, j, NY) >= 0;
    for (int t = 0; t < V; ++t) {
      const int k = kb + t;
      if (k >= 0 && k < P && (slab_coord(p, 2, k, NZ - 1) >= 0 || slab_coord(p, 2, k, NZ) >= 0)) cpml = true;
    }
    for (int i = istart; i < i1 && !cpml; ++i) cpml = slab_coord(p, 0, i, NX - 1) >= 0 || slab_coord(p, 0, i, NX) >= 0;
  }
  for (int comp = 0; comp < 6 && !coef; ++comp) {
    const float* dec = comp < 3 ? p.edecay[comp] : p.hdecay[comp - 3];
    const float* cur = comp < 3 ? p.ecurl[comp] : p.hcurl[comp - 3];
    if (!dec && !cur) continue;
    const float dbg = comp < 3 ? p.edecay_u[comp] : p.hdecay_u[comp - 3];
    const float cbg = comp < 3 ? p.ecurl_u[comp] : p.hcurl_u[comp - 3];
    const int e0 = (comp == 0 || comp == 4 || comp == 5) ? NX - 1 : NX;
    const int e1 = (comp == 1 || comp == 3 || comp == 5) ? NY - 1 : NY;
    const int e2 = (comp == 2 || comp == 3 || comp == 4) ? NZ - 1 : NZ;
    for (int i = istart; i < i1 && !coef; ++i) {
      for (int r = 0; r < 2; ++r) {
        const int jj = r ? j : jm;
        for (int t = 0; t < V; ++t) {
          const int k = kb + t;
          if (k < 0 || k >= P || i >= e0 || jj >= e1 || k >= e2) continue;
          const int64_t o = (static_cast<int64_t>(i) * NY + jj) * P + k;
          if (dec && __ldg(dec + o) != dbg) coef = true;
          if (cur && __ldg(cur + o) != cbg) coef = true;
        }
      }
    }
  }
  // cells whose coefficients an instantaneous nonlinearity rewrites every step
  if (p.nl_lo[0] < p.nl_hi[0] && istart < p.nl_hi[0] && i1 > p.nl_lo[0] && kb < p.nl_hi[2] &&
      kb + V > p.nl_lo[2] && ((jm >= p.nl_lo[1] && jm < p.nl_hi[1]) || (j >= p.nl_lo[1] && j < p.nl_hi[1])))
    coef = true;
  const unsigned any_cpml = __any_sync(kFull, cpml), any_coef = __any_sync(kFull, coef);
  if (lane == 0) out[task] = static_cast<unsigned char>((any_cpml ? kClassCpml : 0u) | (any_coef ? kClassCoef : 0u));
}

}  // namespace

// kAnyCpml / kAnyCoef: the scene has CPML slabs / some coefficient array; each
// warp runs the cheapest march that is exact for its footprint class.
template <int V, int D, bool kAnyCpml, bool kAnyCoef, bool kUniform, int kMinBlocks>
__global__ void __launch_bounds__(256, kMinBlocks) vec_step_kernel(const StepParams p, int n) {
  if (p.step_base) n += __ldg(p.step_base);
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (j >= p.NY) return;  // whole warp; this kernel has no block-level barrier
  unsigned cls = 0;
  if (kAnyCpml || kAnyCoef)
    cls = __ldg(p.warp_class + (static_cast<int64_t>(blockIdx.z) * gridDim.y + blockIdx.y) * p.NY + j);
  if (kAnyCpml && (cls & kClassCpml)) {
    if (kAnyCoef && (cls & kClassCoef)) vmarch<V, D, true, true, kUniform>(p, n, lane, j);
    else vmarch<V, D, true, false, kUniform>(p, n, lane, j);
  } else {
    if (kAnyCoef && (cls & kClassCoef)) vmarch<V, D, false, true, kUniform>(p, n, lane, j);
    else vmarch<V, D, false, false, kUniform>(p, n, lane, j);
  }
}

// Defines `int NAME(const StepParams&, int n, dim3 grid, bool cpml, bool coef,
// bool uniform, cudaStream_t)`: launches vec_step_kernel<V, D, ...> with 256
// threads (eight rows) per CTA and the ring's dynamic shared memory.
#define FDTD_VEC_LAUNCHER(NAME, V, D, MB)                                                                     \
  int NAME(const StepParams& p, int n, dim3 grid, bool cpml, bool coef, bool uni, cudaStream_t stream) {    \
    constexpr int kSmem = (D) > 0 ? 8 * (D) * ring_slot_floats<V>() * 4 : 0;                                 \
    static bool attr_done[64] = {};                                                                          \
    int dev = 0;                                                                                             \
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return static_cast<int>(cudaErrorInvalidDevice); \
    void (*k)(const StepParams, int);                                                                        \
    if (uni) {                                                                                               \
      if (cpml) k = coef ? vec_step_kernel<V, D, true, true, true, MB> : vec_step_kernel<V, D, true, false, true, MB>; \
      else k = coef ? vec_step_kernel<V, D, false, true, true, MB> : vec_step_kernel<V, D, false, false, true, MB>;    \
    } else {                                                                                                 \
      if (cpml) k = coef ? vec_step_kernel<V, D, true, true, false, MB> : vec_step_kernel<V, D, true, false, false, MB>; \
      else k = coef ? vec_step_kernel<V, D, false, true, false, MB> : vec_step_kernel<V, D, false, false, false, MB>;    \
    }                                                                                                        \
    if (kSmem > 48 * 1024 && !attr_done[dev]) {                                                              \
      const void* ks[8] = {(const void*)vec_step_kernel<V, D, true, true, true, MB>,                          \
                           (const void*)vec_step_kernel<V, D, true, false, true, MB>,                         \
                           (const void*)vec_step_kernel<V, D, false, true, true, MB>,                         \
                           (const void*)vec_step_kernel<V, D, false, false, true, MB>,                        \
                           (const void*)vec_step_kernel<V, D, true, true, false, MB>,                         \
                           (const void*)vec_step_kernel<V, D, true, false, false, MB>,                        \
                           (const void*)vec_step_kernel<V, D, false, true, false, MB>,                        \
                           (const void*)vec_step_kernel<V, D, false, false, false, MB>};                      \
      for (const void* f : ks) {                                                                             \
        const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem);   \
        if (e != cudaSuccess) return static_cast<int>(e);                                                    \
      }                                                                                                      \
      attr_done[dev] = true;                                                                                 \
    }                                                                                                        \
    k<<<grid, 256, kSmem, stream>>>(p, n);                                                                   \
    return static_cast<int>(cudaGetLastError());                                                             \
  }

}  // namespace fdtdb200
