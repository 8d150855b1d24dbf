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
#include <type_traits>

#include "step_device.cuh"

namespace fdtdb200 {

// L2 prefetch of row j's fields for the plane ip of an x march: H^{n-1/2} of
// plane ip and E^n of plane ip + 1 (row offset rc, plane stride ps; nothing
// past the chunk end i1).  The neighbour rows j +- 1 are prefetched by the
// warps that own them.
template <typename TS>
__device__ __forceinline__ void prefetch_row(const StepParams& p, int ip, int i1, int ps, int rc, bool kok) {
  if (!kok || ip >= i1) return;
  const int64_t q = static_cast<int64_t>(ip) * ps + rc;
  pf_l2<TS>(p.Hin[0], q);
  pf_l2<TS>(p.Hin[1], q);
  pf_l2<TS>(p.Hin[2], q);
  if (ip + 1 < p.NX) {
    pf_l2<TS>(p.Ein[0], q + ps);
    pf_l2<TS>(p.Ein[1], q + ps);
    pf_l2<TS>(p.Ein[2], q + ps);
  }
}

// The march of one warp task (row j, z block kb, x chunk ch).
// kCpml: run the CPML psi code (the task's footprint touches a slab).  kCoef:
// read the per-cell decay/curl arrays (some coefficient of the footprint
// differs from the background scalars p.*_u).  kUniform: every axis has
// constant spacing, so the inverse spacings are the scalars p.inv_e_u/inv_h_u.
// TS: stored field type (float = the exact FP32 path; __half / __nv_bfloat16 =
// reduced storage with per-component scales).  ADE pole state is BF16 with
// BF16 fields and FP32 otherwise (FP16 would need per-pole scales that the
// source tables do not bound).  kPf: L2 prefetch of the fields p.pf_dist planes
// ahead of the march.  kAde: the ADE poles run here (false when the ADE pass
// after the step kernel advances them; the pole code is then not compiled).
template <typename TS, bool kCpml, bool kCoef, bool kUniform, bool kPf = false, bool kAde = true>
__device__ __forceinline__ void march(const StepParams& p, int n, int lane, int j, int kb, int ch) {
  using TA = typename std::conditional<std::is_same<TS, __nv_bfloat16>::value, __nv_bfloat16, float>::type;
  const int NX = p.NX, NY = p.NY, NZ = p.NZ, P = p.P;
  const int k = kb * kOut - 1 + lane;
  const bool kok = k >= 0 && k < P;
  const bool out_lane = lane >= 1 && lane <= kOut && k < P;
  const int i0 = ch * p.CX;
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
  // CPML slab coordinates; the profile values are re-read (L1 hits) inside the
  // slab branches rather than held in registers across the march.  y_slab is
  // uniform over the warp; z_slab is made uniform with a vote, so a warp
  // outside every z slab skips the z psi code entirely.
  int szh = -1, sze = -1, syh_m = -1, syh_c = -1, sye = -1;
  bool y_slab = false, z_slab = false;
  if (kCpml) {
    szh = slab_coord(p, 2, k, NZ - 1);
    sze = slab_coord(p, 2, k, NZ);
    syh_m = jm_ok ? slab_coord(p, 1, jm, NY - 1) : -1;
    syh_c = slab_coord(p, 1, j, NY - 1);
    sye = slab_coord(p, 1, j, NY);
    y_slab = syh_m >= 0 || syh_c >= 0 || sye >= 0;
    z_slab = __any_sync(kFull, szh >= 0 || sze >= 0);
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
  if (kAde && p.n_poles && out_lane) {
    const int np_ = min(p.n_poles, 32);
    for (int b = 0; b < np_; ++b) {
      const PoleTerm& pt = p.poles[b];
      if (j >= pt.j0 && j < pt.j1 && k >= pt.k0 && k < pt.k1) lane_poles |= 1u << b;
    }
  }
  // warp-uniform: some pole box covers one of this warp's (row, z) cells
  // (poles beyond the 32 of the lane mask are checked inside ade)
  bool warp_poles = false;
  if constexpr (kAde) warp_poles = __any_sync(kFull, lane_poles != 0) || p.n_poles > 32;

  // E^n(i) registers: row j-1 (x, y, z), row j (x, y, z), row j+1 (x, z)
  float em0, em1, em2, ec0, ec1, ec2, ep0, ep2;
  {
    const int o = istart * ps;
    em0 = ldf<TS>(p.Ein[0], o + rm, kok && jm_ok, p.fscale[0]);
    em1 = ldf<TS>(p.Ein[1], o + rm, kok && jm_ok, p.fscale[1]);
    em2 = ldf<TS>(p.Ein[2], o + rm, kok && jm_ok, p.fscale[2]);
    ec0 = ldf<TS>(p.Ein[0], o + rc, kok, p.fscale[0]);
    ec1 = ldf<TS>(p.Ein[1], o + rc, kok, p.fscale[1]);
    ec2 = ldf<TS>(p.Ein[2], o + rc, kok, p.fscale[2]);
    ep0 = ldf<TS>(p.Ein[0], o + rp, kok && jp_ok, p.fscale[0]);
    ep2 = ldf<TS>(p.Ein[2], o + rp, kok && jp_ok, p.fscale[2]);
  }
  float hpz = 0.f, hpy = 0.f;  // Hz, Hy of row j at plane i-1
  if constexpr (kPf) {
    for (int d = 1; d < p.pf_dist; ++d) prefetch_row<TS>(p, istart + d, i1, ps, rc, kok);
  }

  for (int i = istart; i < i1; ++i) {
    const bool own = i >= i0;
    const bool inext = i + 1 < NX;
    const int o = i * ps;
    const int on = o + ps;
    if constexpr (kPf) {
      if (p.pf_dist) prefetch_row<TS>(p, i + p.pf_dist, i1, ps, rc, kok);
    }
    const unsigned pb = __ldg(p.plane_bits + i);
    // E^n(i+1) of rows j-1, j, j+1 (the next plane's E^n(i))
    const float nm0 = ldf<TS>(p.Ein[0], on + rm, kok && jm_ok && inext, p.fscale[0]);
    const float nm1 = ldf<TS>(p.Ein[1], on + rm, kok && jm_ok && inext, p.fscale[1]);
    const float nm2 = ldf<TS>(p.Ein[2], on + rm, kok && jm_ok && inext, p.fscale[2]);
    const float nc0 = ldf<TS>(p.Ein[0], on + rc, kok && inext, p.fscale[0]);
    const float nc1 = ldf<TS>(p.Ein[1], on + rc, kok && inext, p.fscale[1]);
    const float nc2 = ldf<TS>(p.Ein[2], on + rc, kok && inext, p.fscale[2]);
    const float np0 = ldf<TS>(p.Ein[0], on + rp, kok && jp_ok && inext, p.fscale[0]);
    const float np2 = ldf<TS>(p.Ein[2], on + rp, kok && jp_ok && inext, p.fscale[2]);
    // H^{n-1/2}(i) of rows j-1 and j
    const float hm0 = ldf<TS>(p.Hin[0], o + rm, kok && jm_ok, p.fscale[3]);
    const float hm2 = ldf<TS>(p.Hin[2], o + rm, kok && jm_ok, p.fscale[5]);
    const float hc0 = ldf<TS>(p.Hin[0], o + rc, kok, p.fscale[3]);
    const float hc1 = ldf<TS>(p.Hin[1], o + rc, kok, p.fscale[4]);
    const float hc2 = ldf<TS>(p.Hin[2], o + rc, kok, p.fscale[5]);
    const bool ix_ok = i < NX - 1;
    const bool mx_ok = jm_ok && hz_kok, mz_ok = jm_ok && ix_ok && ez_kok;
    const bool cx_ok = yc_ok && hz_kok, cy_ok = ix_ok && hz_kok, cz_ok = ix_ok && yc_ok && ez_kok;
    // Old H psi values of this plane, loaded before the curl math so their
    // latency overlaps it: x slab (Hz row j-1, Hy, Hz), y slab (Hx, Hz of rows
    // j-1 and j), z slab (Hx row j-1, Hx, Hy).
    int sxh = -1, sxe = -1;
    float qx0 = 0.f, qx1 = 0.f, qx2 = 0.f, qy0 = 0.f, qy1 = 0.f, qy2 = 0.f, qy3 = 0.f, qz0 = 0.f, qz1 = 0.f, qz2 = 0.f;
    if (kCpml) {
      sxh = slab_coord(p, 0, i, NX - 1);
      sxe = slab_coord(p, 0, i, NX);
      if (sxh >= 0) {
        qx0 = ldz(p.psiHin[2][0], xslab_off(p, sxh, jm, k), mz_ok);
        qx1 = ldz(p.psiHin[1][0], xslab_off(p, sxh, j, k), cy_ok);
        qx2 = ldz(p.psiHin[2][0], xslab_off(p, sxh, j, k), cz_ok);
      }
      if (y_slab) {
        if (syh_m >= 0) {
          qy0 = ldz(p.psiHin[0][0], yslab_off(p, i, syh_m, k), mx_ok);
          qy1 = ldz(p.psiHin[2][1], yslab_off(p, i, syh_m, k), mz_ok);
        }
        if (syh_c >= 0) {
          qy2 = ldz(p.psiHin[0][0], yslab_off(p, i, syh_c, k), cx_ok);
          qy3 = ldz(p.psiHin[2][1], yslab_off(p, i, syh_c, k), cz_ok);
        }
      }
      if (z_slab && szh >= 0) {
        qz0 = ldz(p.psiHin[0][1], zslab_off(p, i, jm, k), mx_ok);
        qz1 = ldz(p.psiHin[0][1], zslab_off(p, i, j, k), cx_ok);
        qz2 = ldz(p.psiHin[1][1], zslab_off(p, i, j, k), cy_ok);
      }
    }
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
    if (kCpml) {
      const bool wr = own && out_lane;
      if (sxh >= 0) {  // plane inside an x slab: uniform over the warp
        const Prof px = prof(p.hb[0], p.hc[0], p.hik[0], i);
        if (mz_ok) mza = psi_apply(mza, px.b, px.c, px.ik, qx0, p.psiHout[2][0], xslab_off(p, sxh, jm, k), false);
        if (cy_ok) cya = psi_apply(cya, px.b, px.c, px.ik, qx1, p.psiHout[1][0], xslab_off(p, sxh, j, k), wr);
        if (cz_ok) cza = psi_apply(cza, px.b, px.c, px.ik, qx2, p.psiHout[2][0], xslab_off(p, sxh, j, k), wr);
      }
      if (y_slab) {
        if (syh_m >= 0) {
          const Prof py = prof(p.hb[1], p.hc[1], p.hik[1], jm);
          if (mx_ok) mxa = psi_apply(mxa, py.b, py.c, py.ik, qy0, p.psiHout[0][0], yslab_off(p, i, syh_m, k), false);
          if (mz_ok) mzb = psi_apply(mzb, py.b, py.c, py.ik, qy1, p.psiHout[2][1], yslab_off(p, i, syh_m, k), false);
        }
        if (syh_c >= 0) {
          const Prof py = prof(p.hb[1], p.hc[1], p.hik[1], j);
          if (cx_ok) cxa = psi_apply(cxa, py.b, py.c, py.ik, qy2, p.psiHout[0][0], yslab_off(p, i, syh_c, k), wr);
          if (cz_ok) czb = psi_apply(czb, py.b, py.c, py.ik, qy3, p.psiHout[2][1], yslab_off(p, i, syh_c, k), wr);
        }
      }
      if (z_slab && szh >= 0) {
        const Prof pz = prof(p.hb[2], p.hc[2], p.hik[2], k);
        if (mx_ok) mxb = psi_apply(mxb, pz.b, pz.c, pz.ik, qz0, p.psiHout[0][1], zslab_off(p, i, jm, k), false);
        if (cx_ok) cxb = psi_apply(cxb, pz.b, pz.c, pz.ik, qz1, p.psiHout[0][1], zslab_off(p, i, j, k), wr);
        if (cy_ok) cyb = psi_apply(cyb, pz.b, pz.c, pz.ik, qz2, p.psiHout[1][1], zslab_off(p, i, j, k), wr);
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
      stf<TS>(p.Hout[0], o + rc, hcx, p.finv[3]);
      stf<TS>(p.Hout[1], o + rc, hcy, p.finv[4]);
      stf<TS>(p.Hout[2], o + rc, hcz, p.finv[5]);
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
        // a PMC face keeps its tangential E updated: it counts as no face here
        const int pm = p.pmc;
        const bool xlo = i == 0 && !(pm & 1), xhi = i == NX - 1 && !(pm & 2);
        const bool ylo_ = ylo && !(pm & 4), yhi_ = yhi && !(pm & 8);
        const bool zlo_ = zlo && !(pm & 16), zhi_ = zhi && !(pm & 32);
        m0 = edge_mode(i < NX - 1 && ez_kok, ylo_, yhi_, zlo_, zhi_, p.bnd[2], p.bnd[3], p.bnd[4], p.bnd[5]);
        m1 = edge_mode(yc_ok && ez_kok, xlo, xhi, zlo_, zhi_, p.bnd[0], p.bnd[1], p.bnd[4], p.bnd[5]);
        m2 = edge_mode(hz_kok, xlo, xhi, ylo_, yhi_, p.bnd[0], p.bnd[1], p.bnd[2], p.bnd[3]);
        if (pm) {
          // the H outside a PMC face mirrors the H inside with the opposite
          // sign, so the difference across the face doubles (the missing
          // neighbour reads as zero here)
          if ((i == 0 && (pm & 1)) || (i == NX - 1 && (pm & 2))) {
            d1a *= 2.0f;
            d2a *= 2.0f;
          }
          if ((ylo && (pm & 4)) || (yhi && (pm & 8))) {
            d0a *= 2.0f;
            d2b *= 2.0f;
          }
          if ((zlo && (pm & 16)) || (zhi && (pm & 32))) {
            d0b *= 2.0f;
            d1b *= 2.0f;
          }
        }
      }
      if (kCpml) {
        if (sxe >= 0) {
          const Prof px = prof(p.eb[0], p.ec[0], p.eik[0], i);
          if (m1 == 0) d1a = psi_step(d1a, px.b, px.c, px.ik, p.psiE[1][0], p.psiE[1][0], xslab_off(p, sxe, j, k), true);
          if (m2 == 0) d2a = psi_step(d2a, px.b, px.c, px.ik, p.psiE[2][0], p.psiE[2][0], xslab_off(p, sxe, j, k), true);
        }
        if (sye >= 0) {
          const Prof py = prof(p.eb[1], p.ec[1], p.eik[1], j);
          if (m0 == 0) d0a = psi_step(d0a, py.b, py.c, py.ik, p.psiE[0][0], p.psiE[0][0], yslab_off(p, i, sye, k), true);
          if (m2 == 0) d2b = psi_step(d2b, py.b, py.c, py.ik, p.psiE[2][1], p.psiE[2][1], yslab_off(p, i, sye, k), true);
        }
        if (z_slab && sze >= 0) {
          const Prof pz = prof(p.eb[2], p.ec[2], p.eik[2], k);
          if (m0 == 0) d0b = psi_step(d0b, pz.b, pz.c, pz.ik, p.psiE[0][1], p.psiE[0][1], zslab_off(p, i, j, k), true);
          if (m1 == 0) d1b = psi_step(d1b, pz.b, pz.c, pz.ik, p.psiE[1][1], p.psiE[1][1], zslab_off(p, i, j, k), true);
        }
      }
      float v0 = pick(m0, ec0 * g0 + c0 * (d0a - d0b), ec0);
      float v1 = pick(m1, ec1 * g1 + c1 * (d1b - d1a), ec1);
      float v2 = pick(m2, ec2 * g2 + c2 * (d2a - d2b), ec2);
      // ADE subtraction, TFSF electric corrections and soft sources: the
      // additive terms of witwin/maxwell/fdtd/runtime/stepping.py:2295-2320.
      if (kAde && (pb & kPlanePoles) && warp_poles) {
        const unsigned upd = (m0 != kModeDeferred ? 1u : 0u) | (m1 != kModeDeferred ? 2u : 0u) |
                             (m2 != kModeDeferred ? 4u : 0u);
        ade<TA>(p, lane_poles, i, j, k, ec0, ec1, ec2, v0, v1, v2, upd);
      }
      if ((pb & kPlaneETerms) || (lf & (kLfETermY | kLfETermZ)))
        add_terms(p, 0, 0, n, i, j, k, pb & kPlaneETerms, lf & kLfETermY, lf & kLfETermZ, v0, v1, v2);
      // scenes without TFSF end the E update on PEC faces (stepping.py:2316-2318)
      if (p.pec_clamp) {
        if (m0 == 2) v0 = 0.f;
        if (m1 == 2) v1 = 0.f;
        if (m2 == 2) v2 = 0.f;
      }
      // deferred (wrap-face) cells are written by the wrap kernel
      if (m0 != kModeDeferred) stf<TS>(p.Eout[0], o + rc, v0, p.finv[0]);
      if (m1 != kModeDeferred) stf<TS>(p.Eout[1], o + rc, v1, p.finv[1]);
      if (m2 != kModeDeferred) stf<TS>(p.Eout[2], o + rc, v2, p.finv[2]);
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

// kAnyCpml / kAnyCoef: the scene has CPML slabs / some coefficient array.
// Each warp reads its class and runs the cheapest march that is exact for its
// footprint, so the CPML and coefficient code runs only where it changes the
// result.  kMinBlocks trades registers for occupancy.  The plain body (no
// CPML, no coefficient arrays) prefetches its fields into L2 ahead of the
// march, except in the kernel that also holds the CPML + coefficient body and
// the pole code: there the extra code shifts the register allocation of the
// heavy bodies and costs more than the prefetch gains (measured on the
// dispersive workload; without the pole code the prefetch gains 3 %).
template <bool kAnyCpml, bool kAnyCoef, bool kUniform, int kMinBlocks, bool kAde>
__global__ void __launch_bounds__(256, kMinBlocks) warp_step_kernel(const StepParams p, int n, int slot) {
  (void)slot;
  constexpr bool kPlainPrefetch = !(kAnyCpml && kAnyCoef) || !kAde;
  if (p.step_base) n += __ldg(p.step_base);
  const int lane = threadIdx.x & 31;
  // task of this warp in the full grid (a region launch covers a sub-grid)
  const int j = (blockIdx.x + p.rb0) * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int kb = blockIdx.y + p.kb0, ch = blockIdx.z + p.ch0;
  unsigned cls = 0;
  if ((kAnyCpml || kAnyCoef) && j < p.NY)
    cls = __ldg(p.warp_class + (static_cast<int64_t>(ch) * p.n_kb + kb) * p.NY + j);
  // shell_only: the CTAs without a CPML warp belong to the row-tile kernel
  // (its CTAs cover the same rows, z block and chunk)
  if (kAnyCpml && p.shell_only && !__syncthreads_or(cls & kClassCpml)) return;
  if (j >= p.NY) return;  // whole warp; no block-level barrier follows
  if (kAnyCpml && (cls & kClassCpml)) {
    if (kAnyCoef && (cls & kClassCoef)) march<float, true, true, kUniform, false, kAde>(p, n, lane, j, kb, ch);
    else march<float, true, false, kUniform, false, kAde>(p, n, lane, j, kb, ch);
  } else {
    if (kAnyCoef && (cls & kClassCoef)) march<float, false, true, kUniform, false, kAde>(p, n, lane, j, kb, ch);
    else march<float, false, false, kUniform, kPlainPrefetch, kAde>(p, n, lane, j, kb, ch);
  }
}

// Reduced-storage step kernel (TS = __half or __nv_bfloat16): the 64-register
// launch of warp_step_kernel with fields in TS and ADE state in BF16.
template <typename TS, bool kAnyCpml, bool kAnyCoef, bool kUniform>
__global__ void __launch_bounds__(256, 4) warp_step_kernel_rs(const StepParams p, int n) {
  if (p.step_base) n += __ldg(p.step_base);
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (j >= p.NY) return;
  unsigned cls = 0;
  if (kAnyCpml || kAnyCoef)
    cls = __ldg(p.warp_class + (static_cast<int64_t>(blockIdx.z) * gridDim.y + blockIdx.y) * p.NY + j);
  if (kAnyCpml && (cls & kClassCpml)) {
    if (kAnyCoef && (cls & kClassCoef)) march<TS, true, true, kUniform>(p, n, lane, j, blockIdx.y, blockIdx.z);
    else march<TS, true, false, kUniform>(p, n, lane, j, blockIdx.y, blockIdx.z);
  } else {
    if (kAnyCoef && (cls & kClassCoef)) march<TS, false, true, kUniform>(p, n, lane, j, blockIdx.y, blockIdx.z);
    else march<TS, false, false, kUniform>(p, n, lane, j, blockIdx.y, blockIdx.z);
  }
}

int launch_step_reduced(const StepParams& p, int n, dim3 grid, bool cpml, bool coef, bool uni, cudaStream_t stream) {
#define FDTD_RS_PICK(TS)                                                                   \
  do {                                                                                     \
    if (uni) {                                                                             \
      if (cpml) {                                                                          \
        if (coef) warp_step_kernel_rs<TS, true, true, true><<<grid, 256, 0, stream>>>(p, n);   \
        else warp_step_kernel_rs<TS, true, false, true><<<grid, 256, 0, stream>>>(p, n);       \
      } else {                                                                             \
        if (coef) warp_step_kernel_rs<TS, false, true, true><<<grid, 256, 0, stream>>>(p, n);  \
        else warp_step_kernel_rs<TS, false, false, true><<<grid, 256, 0, stream>>>(p, n);      \
      }                                                                                    \
    } else {                                                                               \
      if (cpml) {                                                                          \
        if (coef) warp_step_kernel_rs<TS, true, true, false><<<grid, 256, 0, stream>>>(p, n);  \
        else warp_step_kernel_rs<TS, true, false, false><<<grid, 256, 0, stream>>>(p, n);      \
      } else {                                                                             \
        if (coef) warp_step_kernel_rs<TS, false, true, false><<<grid, 256, 0, stream>>>(p, n); \
        else warp_step_kernel_rs<TS, false, false, false><<<grid, 256, 0, stream>>>(p, n);     \
      }                                                                                    \
    }                                                                                      \
  } while (0)
  if (p.storage == kStoreF16) FDTD_RS_PICK(__half);
  else FDTD_RS_PICK(__nv_bfloat16);
#undef FDTD_RS_PICK
  return static_cast<int>(cudaGetLastError());
}

namespace {

// Yee extent of component c (0..2 Ex..Ez, 3..5 Hx..Hz) along each axis.
__device__ __forceinline__ void comp_ext(int c, int NX, int NY, int NZ, int& e0, int& e1, int& e2) {
  e0 = (c == 0 || c == 4 || c == 5) ? NX - 1 : NX;
  e1 = (c == 1 || c == 3 || c == 5) ? NY - 1 : NY;
  e2 = (c == 2 || c == 3 || c == 4) ? NZ - 1 : NZ;
}

// One warp per task; the footprint is every (plane, row, lane) the march
// touches: planes [istart, i1), rows j-1 and j, lanes k = 30 s - 1 .. 30 s + 30.
__global__ void classify_kernel(const StepParams p, int n_kblocks, int n_chunks, unsigned char* out) {
  const int lane = threadIdx.x & 31;
  const int64_t task = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int NX = p.NX, NY = p.NY, NZ = p.NZ, P = p.P;
  if (task >= static_cast<int64_t>(n_chunks) * n_kblocks * NY) return;
  const int j = static_cast<int>(task % NY);
  const int s = static_cast<int>((task / NY) % n_kblocks);
  const int c = static_cast<int>(task / (static_cast<int64_t>(NY) * n_kblocks));
  const int k = s * kOut - 1 + lane;
  const bool kok = k >= 0 && k < P;
  const int i0 = c * p.CX, i1 = min(i0 + p.CX, NX), istart = max(i0 - 1, 0);
  const int jm = j >= 1 ? j - 1 : j;
  bool cpml = false;
  if (p.cpml) {
    cpml = (kok && (slab_coord(p, 2, k, NZ - 1) >= 0 || slab_coord(p, 2, k, NZ) >= 0)) ||
           slab_coord(p, 1, jm, NY - 1) >= 0 || slab_coord(p, 1, j, NY - 1) >= 0 || slab_coord(p, 1, j, NY) >= 0;
    for (int i = istart; i < i1 && !cpml; ++i) cpml = slab_coord(p, 0, i, NX - 1) >= 0 || slab_coord(p, 0, i, NX) >= 0;
  }
  bool coef = false;
  for (int comp = 0; comp < 6; ++comp) {
    const float* dec = comp < 3 ? p.edecay[comp] : p.hdecay[comp - 3];
    const float* cur = comp < 3 ? p.ecurl[comp] : p.hcurl[comp - 3];
    if (!dec && !cur) continue;
    const float dbg = comp < 3 ? p.edecay_u[comp] : p.hdecay_u[comp - 3];
    const float cbg = comp < 3 ? p.ecurl_u[comp] : p.hcurl_u[comp - 3];
    int e0, e1, e2;
    comp_ext(comp, NX, NY, NZ, e0, e1, e2);
    for (int i = istart; i < i1 && !coef; ++i) {
      for (int r = 0; r < 2; ++r) {
        const int jj = r ? j : jm;
        if (!kok || i >= e0 || jj >= e1 || k >= e2) continue;
        const int64_t o = (static_cast<int64_t>(i) * NY + jj) * P + k;
        if (dec && __ldg(dec + o) != dbg) coef = true;
        if (cur && __ldg(cur + o) != cbg) coef = true;
      }
    }
  }
  // cells whose coefficients an instantaneous nonlinearity rewrites every step
  if (p.nl_lo[0] < p.nl_hi[0] && istart < p.nl_hi[0] && i1 > p.nl_lo[0] && kok && k >= p.nl_lo[2] &&
      k < p.nl_hi[2] && ((jm >= p.nl_lo[1] && jm < p.nl_hi[1]) || (j >= p.nl_lo[1] && j < p.nl_hi[1])))
    coef = true;
  const unsigned any_cpml = __any_sync(kFull, cpml), any_coef = __any_sync(kFull, coef);
  if (lane == 0) out[task] = static_cast<unsigned char>((any_cpml ? kClassCpml : 0u) | (any_coef ? kClassCoef : 0u));
}

}  // namespace

int launch_classify(const StepParams& p, int n_kblocks, int n_chunks, unsigned char* out, cudaStream_t stream) {
  const int64_t tasks = static_cast<int64_t>(n_chunks) * n_kblocks * p.NY;
  const int64_t blocks = (tasks + 7) / 8;
  classify_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(p, n_kblocks, n_chunks, out);
  return static_cast<int>(cudaGetLastError());
}

#define FDTD_INSTANTIATE(CPML, COEF, UNI)                                                         \
  template __global__ void warp_step_kernel<CPML, COEF, UNI, 1, true>(const StepParams, int, int);  \
  template __global__ void warp_step_kernel<CPML, COEF, UNI, 3, true>(const StepParams, int, int);  \
  template __global__ void warp_step_kernel<CPML, COEF, UNI, 4, true>(const StepParams, int, int);  \
  template __global__ void warp_step_kernel<CPML, COEF, UNI, 3, false>(const StepParams, int, int); \
  template __global__ void warp_step_kernel<CPML, COEF, UNI, 4, false>(const StepParams, int, int);
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
