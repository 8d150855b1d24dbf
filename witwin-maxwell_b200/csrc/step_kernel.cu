// Fused leapfrog step kernel: one launch advances H^{n-1/2} -> H^{n+1/2} and
// E^n -> E^{n+1} over the whole grid.
//
// Work decomposition (2.5-D blocking): a CTA owns TY consecutive y rows of the
// node grid, every z cell of those rows (a thread holds four consecutive z cells
// as one float4), and a chunk of CX x planes that it marches through in +x.
// For each plane i it
//   A. loads E^n(i+1) and H^{n-1/2}(i) for its rows (plus one halo row on each
//      side) with 128-bit loads,
//   B. computes H^{n+1/2}(i) for its rows and the -y halo row (the halo value
//      is recomputed, never stored) and stages it in shared memory,
//   C. computes E^{n+1}(i) for its rows from the staged H plane, the H plane of
//      the previous iteration (held in registers), CPML psi slabs, ADE poles,
//      soft/TFSF injection terms, and writes monitor samples.
// E and H are double-buffered across steps (read buffer -> write buffer), so
// the halo recomputation never observes a neighbour's already-advanced values.
// The CPML psi of H is double-buffered for the same reason; psi of E and the
// ADE state are only touched by their owner and are updated in place.
//
// The arithmetic restates witwin/maxwell/fdtd/cuda/kernels/magnetic.cu:62-212
// (H with CPML), electric.cu:242-311 and 462-941 (E with boundary modes and
// CPML), dispersive.cu:18-83 (ADE), sources.cu:135-154 and 485-545 (patch and
// TFSF line injection), observers.cu:7-78 (monitor sampling).
#include "engine.cuh"

namespace fdtdb200 {

namespace {

__device__ __forceinline__ float4 ldg4(const float* base, int64_t off) {
  return __ldg(reinterpret_cast<const float4*>(base + off));
}

__device__ __forceinline__ void st4(float* base, int64_t off, const float (&v)[4]) {
  *reinterpret_cast<float4*>(base + off) = make_float4(v[0], v[1], v[2], v[3]);
}

__device__ __forceinline__ void unpack4(float4 v, float (&o)[4]) {
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
  o[3] = v.w;
}

// Advance one CPML psi value held in slab storage and return the corrected
// derivative d * (1/kappa) + psi.  `axis_off` is the slab-local element offset
// (or -1 outside the slab).
__device__ __forceinline__ float cpml_corrected(float d, int coord, int64_t slab_off, const float* psi_in,
                                                float* psi_out, bool write, const float* b, const float* c,
                                                const float* ik) {
  if (slab_off < 0) return d * __ldg(ik + coord);
  const float v = __ldg(b + coord) * psi_in[slab_off] + __ldg(c + coord) * d;
  if (write) psi_out[slab_off] = v;
  return d * __ldg(ik + coord) + v;
}

// Slab element offset of the psi array of a given axis for cell (i, j, k).
// Layouts: x slab [Lx][NY][P], y slab [NX][Ly][P], z slab [NX][NY][SZ].
__device__ __forceinline__ int64_t slab_offset(const StepParams& p, int axis, int i, int j, int k, int extent) {
  const int lo = p.slab_lo[axis], hi = p.slab_hi[axis];
  if (lo + hi == 0) return -1;
  const int coord = axis == 0 ? i : (axis == 1 ? j : k);
  const int local = slab_local(coord, lo, extent - hi, hi);
  if (local < 0) return -1;
  if (axis == 0) return (static_cast<int64_t>(local) * p.NY + j) * p.P + k;
  if (axis == 1) return (static_cast<int64_t>(i) * (lo + hi) + local) * p.P + k;
  return (static_cast<int64_t>(i) * p.NY + j) * p.SZ + local;
}

__device__ __forceinline__ float term_value(const InjectionTerm& t, int n, int li, int lj, int lk, int i, int j,
                                            int k) {
  const int nj = t.j1 - t.j0, nk = t.k1 - t.k0;
  const float cval = __ldg(t.coeff + (static_cast<int64_t>(li) * nj + lj) * nk + lk);
  float s;
  if (t.signal != nullptr) {
    s = __ldg(t.signal + n);
  } else {
    const int coord = t.sample_axis == 0 ? i : (t.sample_axis == 1 ? j : k);
    const int li_axis = t.sample_axis == 0 ? li : (t.sample_axis == 1 ? lj : lk);
    (void)coord;
    s = __ldg(t.aux_hist + static_cast<int64_t>(n) * t.aux_len + __ldg(t.sample_index + li_axis));
  }
  return cval * s * t.scale;
}

// Add every injection term of component `comp` that covers lanes of (i, j, k0..k0+3).
__device__ __forceinline__ void apply_terms(const StepParams& p, int comp, int n, int i, int j, int k0,
                                            float (&v)[4]) {
  if (p.n_terms == 0) return;
  const int beg = __ldg(p.term_plane_ptr + i), end = __ldg(p.term_plane_ptr + i + 1);
  for (int x = beg; x < end; ++x) {
    const InjectionTerm& t = p.terms[__ldg(p.term_plane_ids + x)];
    if (t.comp != comp || j < t.j0 || j >= t.j1 || k0 + 4 <= t.k0 || k0 >= t.k1) continue;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k = k0 + e;
      if (k >= t.k0 && k < t.k1) v[e] += term_value(t, n, i - t.i0, j - t.j0, k - t.k0, i, j, k);
    }
  }
}

__device__ __forceinline__ void write_samples(const StepParams& p, int comp, int slot, int i, int j, int k0,
                                              const float (&v)[4]) {
  if (p.n_regions == 0) return;
  const int beg = __ldg(p.region_plane_ptr + i), end = __ldg(p.region_plane_ptr + i + 1);
  float* out = p.samples + static_cast<int64_t>(slot) * p.n_samples;
  for (int x = beg; x < end; ++x) {
    const SampleRegion& r = p.regions[__ldg(p.region_plane_ids + x)];
    if (r.comp != comp || j < r.j0 || j >= r.j1 || k0 + 4 <= r.k0 || k0 >= r.k1) continue;
    const int nj = r.j1 - r.j0, nk = r.k1 - r.k0;
    const int64_t row = r.base + (static_cast<int64_t>(i - r.i0) * nj + (j - r.j0)) * nk;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k = k0 + e;
      if (k >= r.k0 && k < r.k1) out[row + (k - r.k0)] = v[e];
    }
  }
}

}  // namespace

__global__ void __launch_bounds__(512) fused_step_kernel(const StepParams p, int n, int slot) {
  extern __shared__ float smem[];
  const int SPR = p.P + 8;
  const int plane_floats = p.ROWS * SPR;
  float* sE = smem;                     // [3][ROWS][SPR], element k of a row at index k + 4
  float* sH = smem + 3 * plane_floats;  // [3][ROWS][SPR]
  const int t = threadIdx.x;
  const int r = t / p.Q;
  const int q = t - r * p.Q;
  const bool thread_active = r < p.ROWS;
  const int j0 = blockIdx.x * p.TY;
  const int gj = j0 - 1 + r;
  const bool row_ok = thread_active && gj >= 0 && gj < p.NY;
  const int i0 = blockIdx.y * p.CX;
  const int i1 = min(i0 + p.CX, p.NX);
  const int k0 = 4 * q;
  const bool h_row = row_ok && r <= p.TY;
  const bool e_row = row_ok && r >= 1 && r <= p.TY;
  const int NX = p.NX, NY = p.NY, NZ = p.NZ;

  for (int x = t; x < 6 * plane_floats; x += blockDim.x) smem[x] = 0.0f;
  __syncthreads();

  const int istart = max(i0 - 1, 0);
  float ec[3][4], en[3][4], hp[3][4], hc[3][4];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      ec[c][e] = 0.0f;
      en[c][e] = 0.0f;
      hp[c][e] = 0.0f;
      hc[c][e] = 0.0f;
    }

  if (row_ok) {
    const int64_t o = (static_cast<int64_t>(istart) * NY + gj) * p.P + k0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      unpack4(ldg4(p.Ein[c], o), ec[c]);
      float* row = sE + c * plane_floats + r * SPR + 4 + k0;
      *reinterpret_cast<float4*>(row) = make_float4(ec[c][0], ec[c][1], ec[c][2], ec[c][3]);
    }
  }

  for (int i = istart; i < i1; ++i) {
    const bool own_plane = i >= i0;
    const int64_t o = (static_cast<int64_t>(i) * NY + gj) * p.P + k0;
    float hold[3][4];
    // ---------------- A: loads ----------------
    if (row_ok) {
      if (i + 1 < NX) {
        const int64_t on = o + static_cast<int64_t>(NY) * p.P;
#pragma unroll
        for (int c = 0; c < 3; ++c) unpack4(ldg4(p.Ein[c], on), en[c]);
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int e = 0; e < 4; ++e) en[c][e] = 0.0f;
      }
    }
    if (h_row) {
#pragma unroll
      for (int c = 0; c < 3; ++c) unpack4(ldg4(p.Hin[c], o), hold[c]);
    }
    __syncthreads();
    // ---------------- B: H^{n+1/2}(i) ----------------
    if (h_row) {
      const float* sEx = sE + 0 * plane_floats + r * SPR + 4;
      const float* sEy = sE + 1 * plane_floats + r * SPR + 4;
      const float* sEz = sE + 2 * plane_floats + r * SPR + 4;
      const bool write_state = own_plane && r >= 1;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int k = k0 + e;
        // Hx: a-axis y (dEz/dy), b-axis z (dEy/dz), curl = a - b
        {
          float h = 0.0f;
          if (i < NX && gj < NY - 1 && k < NZ - 1) {
            const float da = (sEz[SPR + k] - ec[2][e]) * __ldg(p.inv_h[1] + gj);
            const float db = (sEy[k + 1] - ec[1][e]) * __ldg(p.inv_h[2] + k);
            float ea = da, eb = db;
            if (p.cpml) {
              const int64_t sa = slab_offset(p, 1, i, gj, k, NY - 1);
              const int64_t sb = slab_offset(p, 2, i, gj, k, NZ - 1);
              ea = cpml_corrected(da, gj, sa, p.psiHin[0][0], p.psiHout[0][0], write_state, p.hb[1], p.hc[1], p.hik[1]);
              eb = cpml_corrected(db, k, sb, p.psiHin[0][1], p.psiHout[0][1], write_state, p.hb[2], p.hc[2], p.hik[2]);
            }
            const float dec = p.hdecay[0] ? __ldg(p.hdecay[0] + o + e) : p.hdecay_u[0];
            const float cc = p.hcurl[0] ? __ldg(p.hcurl[0] + o + e) : p.hcurl_u[0];
            h = hold[0][e] * dec - cc * (ea - eb);
          }
          hc[0][e] = h;
        }
        // Hy: a-axis x (dEz/dx), b-axis z (dEx/dz), curl = b - a
        {
          float h = 0.0f;
          if (i < NX - 1 && k < NZ - 1) {
            const float da = (en[2][e] - ec[2][e]) * __ldg(p.inv_h[0] + i);
            const float db = (sEx[k + 1] - ec[0][e]) * __ldg(p.inv_h[2] + k);
            float ea = da, eb = db;
            if (p.cpml) {
              const int64_t sa = slab_offset(p, 0, i, gj, k, NX - 1);
              const int64_t sb = slab_offset(p, 2, i, gj, k, NZ - 1);
              ea = cpml_corrected(da, i, sa, p.psiHin[1][0], p.psiHout[1][0], write_state, p.hb[0], p.hc[0], p.hik[0]);
              eb = cpml_corrected(db, k, sb, p.psiHin[1][1], p.psiHout[1][1], write_state, p.hb[2], p.hc[2], p.hik[2]);
            }
            const float dec = p.hdecay[1] ? __ldg(p.hdecay[1] + o + e) : p.hdecay_u[1];
            const float cc = p.hcurl[1] ? __ldg(p.hcurl[1] + o + e) : p.hcurl_u[1];
            h = hold[1][e] * dec - cc * (eb - ea);
          }
          hc[1][e] = h;
        }
        // Hz: a-axis x (dEy/dx), b-axis y (dEx/dy), curl = a - b
        {
          float h = 0.0f;
          if (i < NX - 1 && gj < NY - 1 && k < NZ) {
            const float da = (en[1][e] - ec[1][e]) * __ldg(p.inv_h[0] + i);
            const float db = (sEx[SPR + k] - ec[0][e]) * __ldg(p.inv_h[1] + gj);
            float ea = da, eb = db;
            if (p.cpml) {
              const int64_t sa = slab_offset(p, 0, i, gj, k, NX - 1);
              const int64_t sb = slab_offset(p, 1, i, gj, k, NY - 1);
              ea = cpml_corrected(da, i, sa, p.psiHin[2][0], p.psiHout[2][0], write_state, p.hb[0], p.hc[0], p.hik[0]);
              eb = cpml_corrected(db, gj, sb, p.psiHin[2][1], p.psiHout[2][1], write_state, p.hb[1], p.hc[1], p.hik[1]);
            }
            const float dec = p.hdecay[2] ? __ldg(p.hdecay[2] + o + e) : p.hdecay_u[2];
            const float cc = p.hcurl[2] ? __ldg(p.hcurl[2] + o + e) : p.hcurl_u[2];
            h = hold[2][e] * dec - cc * (ea - eb);
          }
          hc[2][e] = h;
        }
      }
      // TFSF magnetic corrections apply to halo rows too so that the staged
      // halo equals the owner's value.
#pragma unroll
      for (int c = 0; c < 3; ++c) apply_terms(p, 3 + c, n, i, gj, k0, hc[c]);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float* row = sH + c * plane_floats + r * SPR + 4 + k0;
        *reinterpret_cast<float4*>(row) = make_float4(hc[c][0], hc[c][1], hc[c][2], hc[c][3]);
      }
      if (write_state) {
#pragma unroll
        for (int c = 0; c < 3; ++c) st4(p.Hout[c], o, hc[c]);
#pragma unroll
        for (int c = 0; c < 3; ++c) write_samples(p, 3 + c, slot, i, gj, k0, hc[c]);
      }
    }
    __syncthreads();
    // ---------------- C: E^{n+1}(i) ----------------
    if (e_row && own_plane) {
      const float* sHx = sH + 0 * plane_floats + r * SPR + 4;
      const float* sHy = sH + 1 * plane_floats + r * SPR + 4;
      const float* sHz = sH + 2 * plane_floats + r * SPR + 4;
      float enew[3][4];
      float jsub[3][4];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int e = 0; e < 4; ++e) jsub[c][e] = 0.0f;
      // ADE: advance the pole state from E^n and collect dt * J / eps.
      for (int x = 0; x < p.n_poles; ++x) {
        const PoleTerm& pt = p.poles[x];
        if (i < pt.i0 || i >= pt.i1 || gj < pt.j0 || gj >= pt.j1 || k0 + 4 <= pt.k0 || k0 >= pt.k1) continue;
        const int64_t rowb =
            (static_cast<int64_t>(i - pt.i0) * (pt.j1 - pt.j0) + (gj - pt.j0)) * (pt.k1 - pt.k0) - pt.k0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (pt.comp != c) continue;
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int k = k0 + e;
            if (k < pt.k0 || k >= pt.k1) continue;
            const int64_t b = rowb + k;
            const float eold = ec[c][e];
            const float drive = __ldg(pt.drive + b);
            float jn;
            if (pt.kind == 0) {
              const float prev = pt.pol[b];
              const float next = pt.decay * prev + drive * eold;
              pt.pol[b] = next;
              jn = (next - prev) * pt.inv_dt;
              pt.cur[b] = jn;
            } else if (pt.kind == 1) {
              jn = pt.decay * pt.cur[b] + drive * eold;
              pt.cur[b] = jn;
            } else {
              const float pol = pt.pol[b];
              jn = pt.decay * pt.cur[b] - pt.restoring * pol + drive * eold;
              pt.cur[b] = jn;
              pt.pol[b] = pol + pt.dt * jn;
            }
            jsub[c][e] += pt.dt * jn * __ldg(pt.inv_eps + b);
          }
        }
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int k = k0 + e;
        // Ex: a-axis y (dHz/dy), b-axis z (dHy/dz), curl = a - b
        {
          float v = ec[0][e];
          if (i < NX - 1 && k < NZ) {
            const bool ylo = gj == 0, yhi = gj == NY - 1, zlo = k == 0, zhi = k == NZ - 1;
            const bool pec = (ylo && p.bnd[2] == BND_PEC) || (yhi && p.bnd[3] == BND_PEC) ||
                             (zlo && p.bnd[4] == BND_PEC) || (zhi && p.bnd[5] == BND_PEC);
            if (pec) {
              v = 0.0f;
            } else if (!(ylo || yhi || zlo || zhi)) {
              const float da = (hc[2][e] - sHz[-SPR + k]) * __ldg(p.inv_e[1] + gj);
              const float db = (hc[1][e] - sHy[k - 1]) * __ldg(p.inv_e[2] + k);
              float ea = da, eb = db;
              if (p.cpml) {
                const int64_t sa = slab_offset(p, 1, i, gj, k, NY);
                const int64_t sb = slab_offset(p, 2, i, gj, k, NZ);
                ea = cpml_corrected(da, gj, sa, p.psiE[0][0], p.psiE[0][0], true, p.eb[1], p.ec[1], p.eik[1]);
                eb = cpml_corrected(db, k, sb, p.psiE[0][1], p.psiE[0][1], true, p.eb[2], p.ec[2], p.eik[2]);
              }
              const float dec = p.edecay[0] ? __ldg(p.edecay[0] + o + e) : p.edecay_u[0];
              const float cc = p.ecurl[0] ? __ldg(p.ecurl[0] + o + e) : p.ecurl_u[0];
              v = v * dec + cc * (ea - eb);
            }
          } else {
            v = 0.0f;
          }
          enew[0][e] = v;
        }
        // Ey: a-axis x (dHz/dx), b-axis z (dHx/dz), curl = b - a
        {
          float v = ec[1][e];
          if (gj < NY - 1 && k < NZ) {
            const bool xlo = i == 0, xhi = i == NX - 1, zlo = k == 0, zhi = k == NZ - 1;
            const bool pec = (xlo && p.bnd[0] == BND_PEC) || (xhi && p.bnd[1] == BND_PEC) ||
                             (zlo && p.bnd[4] == BND_PEC) || (zhi && p.bnd[5] == BND_PEC);
            if (pec) {
              v = 0.0f;
            } else if (!(xlo || xhi || zlo || zhi)) {
              const float da = (hc[2][e] - hp[2][e]) * __ldg(p.inv_e[0] + i);
              const float db = (hc[0][e] - sHx[k - 1]) * __ldg(p.inv_e[2] + k);
              float ea = da, eb = db;
              if (p.cpml) {
                const int64_t sa = slab_offset(p, 0, i, gj, k, NX);
                const int64_t sb = slab_offset(p, 2, i, gj, k, NZ);
                ea = cpml_corrected(da, i, sa, p.psiE[1][0], p.psiE[1][0], true, p.eb[0], p.ec[0], p.eik[0]);
                eb = cpml_corrected(db, k, sb, p.psiE[1][1], p.psiE[1][1], true, p.eb[2], p.ec[2], p.eik[2]);
              }
              const float dec = p.edecay[1] ? __ldg(p.edecay[1] + o + e) : p.edecay_u[1];
              const float cc = p.ecurl[1] ? __ldg(p.ecurl[1] + o + e) : p.ecurl_u[1];
              v = v * dec + cc * (eb - ea);
            }
          } else {
            v = 0.0f;
          }
          enew[1][e] = v;
        }
        // Ez: a-axis x (dHy/dx), b-axis y (dHx/dy), curl = a - b
        {
          float v = ec[2][e];
          if (k < NZ - 1) {
            const bool xlo = i == 0, xhi = i == NX - 1, ylo = gj == 0, yhi = gj == NY - 1;
            const bool pec = (xlo && p.bnd[0] == BND_PEC) || (xhi && p.bnd[1] == BND_PEC) ||
                             (ylo && p.bnd[2] == BND_PEC) || (yhi && p.bnd[3] == BND_PEC);
            if (pec) {
              v = 0.0f;
            } else if (!(xlo || xhi || ylo || yhi)) {
              const float da = (hc[1][e] - hp[1][e]) * __ldg(p.inv_e[0] + i);
              const float db = (hc[0][e] - sHx[-SPR + k]) * __ldg(p.inv_e[1] + gj);
              float ea = da, eb = db;
              if (p.cpml) {
                const int64_t sa = slab_offset(p, 0, i, gj, k, NX);
                const int64_t sb = slab_offset(p, 1, i, gj, k, NY);
                ea = cpml_corrected(da, i, sa, p.psiE[2][0], p.psiE[2][0], true, p.eb[0], p.ec[0], p.eik[0]);
                eb = cpml_corrected(db, gj, sb, p.psiE[2][1], p.psiE[2][1], true, p.eb[1], p.ec[1], p.eik[1]);
              }
              const float dec = p.edecay[2] ? __ldg(p.edecay[2] + o + e) : p.edecay_u[2];
              const float cc = p.ecurl[2] ? __ldg(p.ecurl[2] + o + e) : p.ecurl_u[2];
              v = v * dec + cc * (ea - eb);
            }
          } else {
            v = 0.0f;
          }
          enew[2][e] = v;
        }
      }
      // TFSF electric corrections and soft sources, then the ADE subtraction
      // (the order of witwin/maxwell/fdtd/runtime/stepping.py:2295-2320).
#pragma unroll
      for (int c = 0; c < 3; ++c) apply_terms(p, c, n, i, gj, k0, enew[c]);
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int e = 0; e < 4; ++e) enew[c][e] -= jsub[c][e];
#pragma unroll
      for (int c = 0; c < 3; ++c) st4(p.Eout[c], o, enew[c]);
#pragma unroll
      for (int c = 0; c < 3; ++c) write_samples(p, c, slot, i, gj, k0, enew[c]);
    }
    // Stage E^n(i+1) for the next plane and rotate the x-march registers.
    if (row_ok) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float* row = sE + c * plane_floats + r * SPR + 4 + k0;
        *reinterpret_cast<float4*>(row) = make_float4(en[c][0], en[c][1], en[c][2], en[c][3]);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          ec[c][e] = en[c][e];
          hp[c][e] = hc[c][e];
        }
      }
    }
  }
}

}  // namespace fdtdb200
