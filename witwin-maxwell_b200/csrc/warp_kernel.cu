// Warp-granular fused leapfrog step: one launch advances H^{n-1/2} ->
// H^{n+1/2} and E^n -> E^{n+1} over the whole grid with no shared memory and
// no block barriers.
//
// Decomposition: a warp owns one y row j and 30 consecutive z cells
// (lane l <-> k = 30 s - 1 + l; lane 0 and lane 31 are halo lanes) and marches
// in +x over a chunk of planes.  Per plane i it
//   - loads E^n(i+1) for rows j-1, j, j+1 (the values become E^n(i) of the
//     next plane, so every E value is loaded once per warp),
//   - computes H^{n+1/2}(i) for rows j-1 (a halo row, recomputed and never
//     stored) and j; z+1 neighbours come from the next lane (__shfl_down),
//   - computes E^{n+1}(i) for row j from the H of rows j, j-1, the H of the
//     previous plane (registers) and the z-1 neighbour (__shfl_up).
// Monitor samples are gathered by a separate kernel after the step.
// Neighbour-row reads are L1/L2 hits (the warps of a block own consecutive
// rows), so DRAM sees each field once per step.  E, H and the H CPML psi are
// double-buffered across steps, so halo recomputation reads unmodified old
// values; E psi and ADE state are touched only by their owning lane.
//
// Arithmetic restated from witwin/maxwell/fdtd/cuda/kernels/magnetic.cu:62-212,
// electric.cu:242-311 and 462-941, dispersive.cu:18-83, sources.cu:135-154 and
// 485-545, observers.cu:7-78.
#include "engine.cuh"

namespace fdtdb200 {

namespace {

constexpr int kOut = 30;  // output z cells per warp
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float ldz(const float* base, int64_t off, bool ok) { return ok ? __ldg(base + off) : 0.0f; }

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

// Slab element offsets (32-bit: every engine array holds fewer than 2^31 elements).
__device__ __forceinline__ int xslab_off(const StepParams& p, int lx, int j, int k) { return (lx * p.NY + j) * p.P + k; }
__device__ __forceinline__ int yslab_off(const StepParams& p, int i, int ly, int k) {
  return (i * (p.slab_lo[1] + p.slab_hi[1]) + ly) * p.P + k;
}
__device__ __forceinline__ int zslab_off(const StepParams& p, int i, int j, int lz) { return (i * p.NY + j) * p.SZ + lz; }

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
// the plane list already restricts i.
__device__ __forceinline__ void ade(const StepParams& p, unsigned lane_poles, int i, int j, int k, float e0, float e1,
                                    float e2, float& v0, float& v1, float& v2) {
  const int b = __ldg(p.pole_plane_ptr + i), e = __ldg(p.pole_plane_ptr + i + 1);
  for (int x = b; x < e; ++x) {
    const int id = __ldg(p.pole_plane_ids + x);
    if (id < 32 && !((lane_poles >> id) & 1u)) continue;
    const PoleTerm& pt = p.poles[id];
    if (id >= 32 && (j < pt.j0 || j >= pt.j1 || k < pt.k0 || k >= pt.k1)) continue;
    const int64_t o = (static_cast<int64_t>(i - pt.i0) * (pt.j1 - pt.j0) + (j - pt.j0)) * (pt.k1 - pt.k0) + (k - pt.k0);
    const int c = pt.comp;
    const float eo = c == 0 ? e0 : (c == 1 ? e1 : e2);
    const float drive = __ldg(pt.drive + o);
    float jn;
    if (pt.kind == 0) {
      const float prev = pt.pol[o];
      const float next = pt.decay * prev + drive * eo;
      pt.pol[o] = next;
      jn = (next - prev) * pt.inv_dt;
      pt.cur[o] = jn;
    } else if (pt.kind == 1) {
      jn = pt.decay * pt.cur[o] + drive * eo;
      pt.cur[o] = jn;
    } else {
      const float pol = pt.pol[o];
      jn = pt.decay * pt.cur[o] - pt.restoring * pol + drive * eo;
      pt.cur[o] = jn;
      pt.pol[o] = pol + pt.dt * jn;
    }
    const float sub = pt.dt * jn * __ldg(pt.inv_eps + o);
    if (c == 0) v0 -= sub;
    else if (c == 1) v1 -= sub;
    else v2 -= sub;
  }
}

// E edge status (electric.cu:242-268): 0 update, 1 keep (NONE/PML edge),
// 2 PEC zero, 3 outside the Yee extent (stays zero).
__device__ __forceinline__ int edge_mode(bool in_extent, bool alo, bool ahi, bool blo, bool bhi, int ma_lo, int ma_hi,
                                         int mb_lo, int mb_hi) {
  if (!in_extent) return 3;
  if ((alo && ma_lo == BND_PEC) || (ahi && ma_hi == BND_PEC) || (blo && mb_lo == BND_PEC) || (bhi && mb_hi == BND_PEC))
    return 2;
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

// kCpml: the scene has CPML slabs.  kCoef: some decay/curl coefficient is a
// per-cell array.  kMinBlocks trades registers for occupancy.
// kUniform: every axis has constant spacing, so the inverse spacings are the
// scalars p.inv_e_u / p.inv_h_u.
template <bool kCpml, bool kCoef, bool kUniform, int kMinBlocks>
__global__ void __launch_bounds__(256, kMinBlocks) warp_step_kernel(const StepParams p, int n, int slot) {
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int NX = p.NX, NY = p.NY, NZ = p.NZ, P = p.P;
  if (j >= NY) return;  // whole warp; this kernel has no block-level barrier
  const int k = blockIdx.y * kOut - 1 + lane;
  const bool kok = k >= 0 && k < P;
  const bool out_lane = lane >= 1 && lane <= kOut && k < P;
  const int i0 = blockIdx.z * p.CX;
  const int i1 = min(i0 + p.CX, NX);
  const int istart = max(i0 - 1, 0);
  const bool jm_ok = j >= 1, jp_ok = j + 1 < NY;
  const int jm = jm_ok ? j - 1 : 0, jp = jp_ok ? j + 1 : 0;
  const int kc = kok ? k : 0;
  const int ps = NY * P;
  const int rm = jm * P + kc, rc = j * P + kc, rp = jp * P + kc;

  // ---- loop-invariant per-lane / per-row data ----
  const bool hz_kok = k >= 0 && k < NZ - 1;  // Hx, Hy extent along z
  const bool ez_kok = k >= 0 && k < NZ;      // Ex, Ey (and Hz) extent along z
  const bool yc_ok = j < NY - 1;             // Hx, Hz extent along y (row j)
  const float ihz = kUniform ? p.inv_h_u[2] : __ldg(p.inv_h[2] + (hz_kok ? k : 0));
  const float iez = kUniform ? p.inv_e_u[2] : __ldg(p.inv_e[2] + (ez_kok ? k : 0));
  const float ihy_m = kUniform ? p.inv_h_u[1] : __ldg(p.inv_h[1] + jm);
  const float ihy_c = kUniform ? p.inv_h_u[1] : __ldg(p.inv_h[1] + (yc_ok ? j : 0));
  const float iey = kUniform ? p.inv_e_u[1] : __ldg(p.inv_e[1] + j);
  const bool ylo = j == 0, yhi = j == NY - 1, zlo = k == 0, zhi = k == NZ - 1;
  const bool lane_edge = ylo || yhi || k <= 0 || k >= NZ - 1;
  int szh = -1, sze = -1, syh_m = -1, syh_c = -1, sye = -1;
  Prof pzh{0.f, 0.f, 1.f}, pze{0.f, 0.f, 1.f}, pym{0.f, 0.f, 1.f}, pyc{0.f, 0.f, 1.f}, pye{0.f, 0.f, 1.f};
  if (kCpml) {
    szh = slab_coord(p, 2, k, NZ - 1);
    sze = slab_coord(p, 2, k, NZ);
    syh_m = jm_ok ? slab_coord(p, 1, jm, NY - 1) : -1;
    syh_c = slab_coord(p, 1, j, NY - 1);
    sye = slab_coord(p, 1, j, NY);
    if (szh >= 0) pzh = prof(p.hb[2], p.hc[2], p.hik[2], k);
    if (sze >= 0) pze = prof(p.eb[2], p.ec[2], p.eik[2], k);
    if (syh_m >= 0) pym = prof(p.hb[1], p.hc[1], p.hik[1], jm);
    if (syh_c >= 0) pyc = prof(p.hb[1], p.hc[1], p.hik[1], j);
    if (sye >= 0) pye = prof(p.eb[1], p.ec[1], p.eik[1], j);
  }
  unsigned lf = 0;
  if (p.n_terms[1]) {
    if (jm_ok && list_nonempty(p.term_index[1], 1, jm)) lf |= kLfHTermYm;
    if (list_nonempty(p.term_index[1], 1, j)) lf |= kLfHTermYc;
    if (kok && list_nonempty(p.term_index[1], 2, k)) lf |= kLfHTermZ;
  }
  if (p.n_terms[0]) {
    if (list_nonempty(p.term_index[0], 1, j)) lf |= kLfETermY;
    if (kok && list_nonempty(p.term_index[0], 2, k)) lf |= kLfETermZ;
  }

  unsigned lane_poles = 0;
  if (p.n_poles && out_lane) {
    const int np_ = min(p.n_poles, 32);
    for (int b = 0; b < np_; ++b) {
      const PoleTerm& pt = p.poles[b];
      if (j >= pt.j0 && j < pt.j1 && k >= pt.k0 && k < pt.k1) lane_poles |= 1u << b;
    }
  }

  // E^n(i) registers: row j-1 (x, y, z), row j (x, y, z), row j+1 (x, z)
  float em0, em1, em2, ec0, ec1, ec2, ep0, ep2;
  {
    const int o = istart * ps;
    em0 = ldz(p.Ein[0], o + rm, kok && jm_ok);
    em1 = ldz(p.Ein[1], o + rm, kok && jm_ok);
    em2 = ldz(p.Ein[2], o + rm, kok && jm_ok);
    ec0 = ldz(p.Ein[0], o + rc, kok);
    ec1 = ldz(p.Ein[1], o + rc, kok);
    ec2 = ldz(p.Ein[2], o + rc, kok);
    ep0 = ldz(p.Ein[0], o + rp, kok && jp_ok);
    ep2 = ldz(p.Ein[2], o + rp, kok && jp_ok);
  }
  float hpz = 0.f, hpy = 0.f;  // Hz, Hy of row j at plane i-1

  for (int i = istart; i < i1; ++i) {
    const bool own = i >= i0;
    const bool inext = i + 1 < NX;
    const int o = i * ps;
    const int on = o + ps;
    const unsigned pb = __ldg(p.plane_bits + i);
    // E^n(i+1) of rows j-1, j, j+1 (the next plane's E^n(i))
    const float nm0 = ldz(p.Ein[0], on + rm, kok && jm_ok && inext);
    const float nm1 = ldz(p.Ein[1], on + rm, kok && jm_ok && inext);
    const float nm2 = ldz(p.Ein[2], on + rm, kok && jm_ok && inext);
    const float nc0 = ldz(p.Ein[0], on + rc, kok && inext);
    const float nc1 = ldz(p.Ein[1], on + rc, kok && inext);
    const float nc2 = ldz(p.Ein[2], on + rc, kok && inext);
    const float np0 = ldz(p.Ein[0], on + rp, kok && jp_ok && inext);
    const float np2 = ldz(p.Ein[2], on + rp, kok && jp_ok && inext);
    // H^{n-1/2}(i) of rows j-1 and j
    const float hm0 = ldz(p.Hin[0], o + rm, kok && jm_ok);
    const float hm2 = ldz(p.Hin[2], o + rm, kok && jm_ok);
    const float hc0 = ldz(p.Hin[0], o + rc, kok);
    const float hc1 = ldz(p.Hin[1], o + rc, kok);
    const float hc2 = ldz(p.Hin[2], o + rc, kok);
    // E coefficient arrays of this plane, issued early so their latency hides
    // behind the H update
    float g0 = p.edecay_u[0], g1 = p.edecay_u[1], g2 = p.edecay_u[2];
    float c0 = p.ecurl_u[0], c1 = p.ecurl_u[1], c2 = p.ecurl_u[2];
    if (kCoef) {
      const bool ld = own && out_lane;
      if (p.ecurl[0]) c0 = ldz(p.ecurl[0], o + rc, ld);
      if (p.ecurl[1]) c1 = ldz(p.ecurl[1], o + rc, ld);
      if (p.ecurl[2]) c2 = ldz(p.ecurl[2], o + rc, ld);
      if (p.edecay[0]) g0 = ldz(p.edecay[0], o + rc, ld);
      if (p.edecay[1]) g1 = ldz(p.edecay[1], o + rc, ld);
      if (p.edecay[2]) g2 = ldz(p.edecay[2], o + rc, ld);
    }
    const bool ix_ok = i < NX - 1;
    const float ihx = kUniform ? p.inv_h_u[0] : __ldg(p.inv_h[0] + (ix_ok ? i : 0));
    // z+1 neighbours of rows j-1 and j (the halo row needs Ey only: its Hy is unused)
    const float em1k = __shfl_down_sync(kFull, em1, 1);
    const float ec0k = __shfl_down_sync(kFull, ec0, 1);
    const float ec1k = __shfl_down_sync(kFull, ec1, 1);

    // ---------------- H^{n+1/2}(i): halo row j-1 (Hx, Hz), then row j ----------------
    // Hx: dEz/dy - dEy/dz; Hy: dEx/dz - dEz/dx; Hz: dEy/dx - dEx/dy
    float mxa = (ec2 - em2) * ihy_m, mxb = (em1k - em1) * ihz;
    float mza = (nm1 - em1) * ihx, mzb = (ec0 - em0) * ihy_m;
    float cxa = (ep2 - ec2) * ihy_c, cxb = (ec1k - ec1) * ihz;
    float cya = (nc2 - ec2) * ihx, cyb = (ec0k - ec0) * ihz;
    float cza = (nc1 - ec1) * ihx, czb = (ep0 - ec0) * ihy_c;
    const bool mx_ok = jm_ok && hz_kok, mz_ok = jm_ok && ix_ok && ez_kok;
    const bool cx_ok = yc_ok && hz_kok, cy_ok = ix_ok && hz_kok, cz_ok = ix_ok && yc_ok && ez_kok;
    int sxh = -1, sxe = -1;
    if (kCpml) {
      sxh = slab_coord(p, 0, i, NX - 1);
      sxe = slab_coord(p, 0, i, NX);
      if (sxh >= 0 || szh >= 0 || syh_m >= 0 || syh_c >= 0) {
        const bool wr = own && out_lane;
        Prof pxh{0.f, 0.f, 1.f};
        if (sxh >= 0) pxh = prof(p.hb[0], p.hc[0], p.hik[0], i);
        if (syh_m >= 0 && mx_ok) mxa = psi_step(mxa, pym.b, pym.c, pym.ik, p.psiHin[0][0], p.psiHout[0][0], yslab_off(p, i, syh_m, k), false);
        if (szh >= 0 && mx_ok) mxb = psi_step(mxb, pzh.b, pzh.c, pzh.ik, p.psiHin[0][1], p.psiHout[0][1], zslab_off(p, i, jm, szh), false);
        if (sxh >= 0 && mz_ok) mza = psi_step(mza, pxh.b, pxh.c, pxh.ik, p.psiHin[2][0], p.psiHout[2][0], xslab_off(p, sxh, jm, k), false);
        if (syh_m >= 0 && mz_ok) mzb = psi_step(mzb, pym.b, pym.c, pym.ik, p.psiHin[2][1], p.psiHout[2][1], yslab_off(p, i, syh_m, k), false);
        if (syh_c >= 0 && cx_ok) cxa = psi_step(cxa, pyc.b, pyc.c, pyc.ik, p.psiHin[0][0], p.psiHout[0][0], yslab_off(p, i, syh_c, k), wr);
        if (szh >= 0 && cx_ok) cxb = psi_step(cxb, pzh.b, pzh.c, pzh.ik, p.psiHin[0][1], p.psiHout[0][1], zslab_off(p, i, j, szh), wr);
        if (sxh >= 0 && cy_ok) cya = psi_step(cya, pxh.b, pxh.c, pxh.ik, p.psiHin[1][0], p.psiHout[1][0], xslab_off(p, sxh, j, k), wr);
        if (szh >= 0 && cy_ok) cyb = psi_step(cyb, pzh.b, pzh.c, pzh.ik, p.psiHin[1][1], p.psiHout[1][1], zslab_off(p, i, j, szh), wr);
        if (sxh >= 0 && cz_ok) cza = psi_step(cza, pxh.b, pxh.c, pxh.ik, p.psiHin[2][0], p.psiHout[2][0], xslab_off(p, sxh, j, k), wr);
        if (syh_c >= 0 && cz_ok) czb = psi_step(czb, pyc.b, pyc.c, pyc.ik, p.psiHin[2][1], p.psiHout[2][1], yslab_off(p, i, syh_c, k), wr);
      }
    }
    float dHx = p.hdecay_u[0], cHx = p.hcurl_u[0], dHy = p.hdecay_u[1], cHy = p.hcurl_u[1], dHz = p.hdecay_u[2],
          cHz = p.hcurl_u[2];
    float dHxm = dHx, cHxm = cHx, dHzm = dHz, cHzm = cHz;
    if (kCoef) {
      if (p.hdecay[0]) { dHx = ldz(p.hdecay[0], o + rc, kok); dHxm = ldz(p.hdecay[0], o + rm, kok && jm_ok); }
      if (p.hcurl[0]) { cHx = ldz(p.hcurl[0], o + rc, kok); cHxm = ldz(p.hcurl[0], o + rm, kok && jm_ok); }
      if (p.hdecay[1]) dHy = ldz(p.hdecay[1], o + rc, kok);
      if (p.hcurl[1]) cHy = ldz(p.hcurl[1], o + rc, kok);
      if (p.hdecay[2]) { dHz = ldz(p.hdecay[2], o + rc, kok); dHzm = ldz(p.hdecay[2], o + rm, kok && jm_ok); }
      if (p.hcurl[2]) { cHz = ldz(p.hcurl[2], o + rc, kok); cHzm = ldz(p.hcurl[2], o + rm, kok && jm_ok); }
    }
    float hmx = mx_ok ? hm0 * dHxm - cHxm * (mxa - mxb) : 0.f;
    float hmy = 0.f;
    float hmz = mz_ok ? hm2 * dHzm - cHzm * (mza - mzb) : 0.f;
    float hcx = cx_ok ? hc0 * dHx - cHx * (cxa - cxb) : 0.f;
    float hcy = cy_ok ? hc1 * dHy - cHy * (cyb - cya) : 0.f;
    float hcz = cz_ok ? hc2 * dHz - cHz * (cza - czb) : 0.f;
    // TFSF magnetic corrections, also on the halo row so it equals the owner's value
    if (kok && ((pb & kPlaneHTerms) || (lf & (kLfHTermYm | kLfHTermYc | kLfHTermZ)))) {
      if (jm_ok)
        add_terms(p, 1, 3, n, i, jm, k, pb & kPlaneHTerms, lf & kLfHTermYm, lf & kLfHTermZ, hmx, hmy, hmz);
      add_terms(p, 1, 3, n, i, j, k, pb & kPlaneHTerms, lf & kLfHTermYc, lf & kLfHTermZ, hcx, hcy, hcz);
    }
    if (own && out_lane) {
      __stcg(p.Hout[0] + o + rc, hcx);
      __stcg(p.Hout[1] + o + rc, hcy);
      __stcg(p.Hout[2] + o + rc, hcz);
    }

    // ---------------- E^{n+1}(i), row j ----------------
    const float hxk = __shfl_up_sync(kFull, hcx, 1);
    const float hyk = __shfl_up_sync(kFull, hcy, 1);
    if (own && out_lane) {
      const float iex = kUniform ? p.inv_e_u[0] : __ldg(p.inv_e[0] + i);
      // Ex: dHz/dy - dHy/dz; Ey: dHx/dz - dHz/dx; Ez: dHy/dx - dHx/dy
      float d0a = (hcz - hmz) * iey, d0b = (hcy - hyk) * iez;
      float d1a = (hcz - hpz) * iex, d1b = (hcx - hxk) * iez;
      float d2a = (hcy - hpy) * iex, d2b = (hcx - hmx) * iey;
      int m0 = 0, m1 = 0, m2 = 0;
      if (lane_edge || i == 0 || i == NX - 1) {
        const bool xlo = i == 0, xhi = i == NX - 1;
        m0 = edge_mode(i < NX - 1 && ez_kok, ylo, yhi, zlo, zhi, p.bnd[2], p.bnd[3], p.bnd[4], p.bnd[5]);
        m1 = edge_mode(yc_ok && ez_kok, xlo, xhi, zlo, zhi, p.bnd[0], p.bnd[1], p.bnd[4], p.bnd[5]);
        m2 = edge_mode(hz_kok, xlo, xhi, ylo, yhi, p.bnd[0], p.bnd[1], p.bnd[2], p.bnd[3]);
      }
      if (kCpml && (sxe >= 0 || sye >= 0 || sze >= 0)) {
        Prof pxe{0.f, 0.f, 1.f};
        if (sxe >= 0) pxe = prof(p.eb[0], p.ec[0], p.eik[0], i);
        if (sye >= 0 && m0 == 0) d0a = psi_step(d0a, pye.b, pye.c, pye.ik, p.psiE[0][0], p.psiE[0][0], yslab_off(p, i, sye, k), true);
        if (sze >= 0 && m0 == 0) d0b = psi_step(d0b, pze.b, pze.c, pze.ik, p.psiE[0][1], p.psiE[0][1], zslab_off(p, i, j, sze), true);
        if (sxe >= 0 && m1 == 0) d1a = psi_step(d1a, pxe.b, pxe.c, pxe.ik, p.psiE[1][0], p.psiE[1][0], xslab_off(p, sxe, j, k), true);
        if (sze >= 0 && m1 == 0) d1b = psi_step(d1b, pze.b, pze.c, pze.ik, p.psiE[1][1], p.psiE[1][1], zslab_off(p, i, j, sze), true);
        if (sxe >= 0 && m2 == 0) d2a = psi_step(d2a, pxe.b, pxe.c, pxe.ik, p.psiE[2][0], p.psiE[2][0], xslab_off(p, sxe, j, k), true);
        if (sye >= 0 && m2 == 0) d2b = psi_step(d2b, pye.b, pye.c, pye.ik, p.psiE[2][1], p.psiE[2][1], yslab_off(p, i, sye, k), true);
      }
      float v0 = pick(m0, ec0 * g0 + c0 * (d0a - d0b), ec0);
      float v1 = pick(m1, ec1 * g1 + c1 * (d1b - d1a), ec1);
      float v2 = pick(m2, ec2 * g2 + c2 * (d2a - d2b), ec2);
      // ADE subtraction, TFSF electric corrections and soft sources: the
      // additive terms of witwin/maxwell/fdtd/runtime/stepping.py:2295-2320.
      if (pb & kPlanePoles) ade(p, lane_poles, i, j, k, ec0, ec1, ec2, v0, v1, v2);
      if ((pb & kPlaneETerms) || (lf & (kLfETermY | kLfETermZ)))
        add_terms(p, 0, 0, n, i, j, k, pb & kPlaneETerms, lf & kLfETermY, lf & kLfETermZ, v0, v1, v2);
      __stcg(p.Eout[0] + o + rc, v0);
      __stcg(p.Eout[1] + o + rc, v1);
      __stcg(p.Eout[2] + o + rc, v2);
    }
    hpz = hcz;
    hpy = hcy;
    em0 = nm0;
    em1 = nm1;
    em2 = nm2;
    ec0 = nc0;
    ec1 = nc1;
    ec2 = nc2;
    ep0 = np0;
    ep2 = np2;
  }
}

#define FDTD_INSTANTIATE(CPML, COEF, UNI)                                                  \
  template __global__ void warp_step_kernel<CPML, COEF, UNI, 1>(const StepParams, int, int); \
  template __global__ void warp_step_kernel<CPML, COEF, UNI, 3>(const StepParams, int, int); \
  template __global__ void warp_step_kernel<CPML, COEF, UNI, 4>(const StepParams, int, int);
FDTD_INSTANTIATE(false, false, false)
FDTD_INSTANTIATE(false, true, false)
FDTD_INSTANTIATE(true, false, false)
FDTD_INSTANTIATE(true, true, false)
FDTD_INSTANTIATE(false, false, true)
FDTD_INSTANTIATE(false, true, true)
FDTD_INSTANTIATE(true, false, true)
FDTD_INSTANTIATE(true, true, true)
#undef FDTD_INSTANTIATE

}  // namespace fdtdb200
