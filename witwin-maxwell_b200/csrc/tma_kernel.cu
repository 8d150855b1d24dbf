// TMA-fed fused leapfrog step.  Same per-warp march as warp_kernel.cu (a warp
// owns y row j and 30 z cells, lane l <-> k = 30 s - 1 + l, and marches +x
// over a chunk of planes), but the E^n and H^{n-1/2} values of each plane come
// from shared memory: a producer warp streams whole plane tiles with
// cp.async.bulk.tensor (TMA) into a ring of kStages stages, several planes
// ahead of the eight consumer warps, so the loads' latency no longer stalls
// the march and no registers hold prefetched values.
//
// Tile of one stage (one x plane, the CTA's 8 rows and 30-cell z block):
//   E components: rows j0-1 .. j0+8 (10) x 36 z cells, box start a = the
//   multiple of 4 at or below 30 s - 1 (TMA wants 16-byte aligned x
//   coordinates), so lane l reads column l + (30 s - 1 - a);
//   H components: rows j0-1 .. j0+7 (9) x 36.
// Out-of-range rows, columns and the plane x = NX arrive as zeros (TMA fill),
// which is the value the warp kernel substitutes for them.
//
// Pipeline: full[s] completes when the stage's bytes have landed (producer
// arrive.expect_tx + complete_tx); empty[s] completes when all 8 consumer
// warps have finished the plane (one arrival per warp).  Iteration i reads
// the stages of planes i and i + 1 and releases plane i's stage.  Every wait
// is bounded; on timeout the warp records FDTD_ERR_TIMEOUT in p.status and
// stops, and the producer waits (bounded) for its issued copies before
// leaving.
//
// Arithmetic restated from witwin/maxwell/fdtd/cuda/kernels/magnetic.cu:62-212,
// electric.cu:242-311 and 462-941, dispersive.cu:18-83, sources.cu:135-154 and
// 485-545.
#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/fdtd_b200.h"
#include "step_device.cuh"
#include "tma_step.cuh"

namespace fdtdb200 {

namespace {

constexpr int kCols = 36;              // z cells per tile row
constexpr int kERows = kTmaRows + 2;   // E rows j0-1 .. j0+8
constexpr int kHRows = kTmaRows + 1;   // H rows j0-1 .. j0+7
constexpr int kEPad = 384;             // floats per E component tile (>= 10 x 36, 128-byte multiple)
constexpr int kHPad = 352;             // floats per H component tile (>= 9 x 36, 128-byte multiple)
constexpr int kStageFloats = 3 * kEPad + 3 * kHPad;
constexpr uint32_t kEBytes = kCols * kERows * 4;  // one E component box
constexpr uint32_t kHBytes = kCols * kHRows * 4;  // one H component box
// try_wait rounds of the final drain (the producer waiting for its own issued
// copies before the block exits); the pipeline waits use p.wait_limit.
constexpr uint32_t kSpinLimit = 1u << 20;

static_assert(kERows * kCols <= kEPad && kHRows * kCols <= kHPad, "tile pads too small");
static_assert((kEPad * 4) % 128 == 0 && (kHPad * 4) % 128 == 0, "tiles must stay 128-byte aligned");

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Bounded wait for the phase of parity `parity` to complete.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint32_t limit) {
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 3-D tiled TMA load (no multicast) of box {36, rows, 1} at (x, y, z).
__device__ __forceinline__ void tma_load(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void report_timeout(int* status) {
  if (status) atomicExch(status, FDTD_ERR_TIMEOUT);
}

struct Ring {
  float* stages;      // kStages x kStageFloats
  uint32_t full0;     // shared address of full[0] (8 bytes apart)
  uint32_t empty0;    // shared address of empty[0]
  int istart, i1;     // planes consumed: istart .. i1 (i1 read as the last "next" plane)
  uint32_t limit;     // try_wait rounds of a pipeline wait (StepParams::wait_limit)
};

// Consumer side: wait until the stage of plane q has landed.
__device__ __forceinline__ bool ring_wait_full(const Ring& r, int q) {
  const int u = q - r.istart;
  return mbar_wait(r.full0 + 8u * (u % kStages), (u / kStages) & 1, r.limit);
}

}  // namespace

// A consumer warp whose row lies beyond the grid computes nothing but still
// waits for and releases every stage, so the empty barriers keep their count.
__device__ __forceinline__ void idle_march(const Ring& ring, int lane, int* status) {
  if (!ring_wait_full(ring, ring.istart)) {
    report_timeout(status);
    return;
  }
  for (int i = ring.istart; i < ring.i1; ++i) {
    if (!ring_wait_full(ring, i + 1)) {
      report_timeout(status);
      return;
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(ring.empty0 + 8u * ((i - ring.istart) % kStages));
  }
}

// March of one consumer warp (tile row w, grid row j < NY) with the warp
// kernel's arithmetic; see warp_kernel.cu for kCpml / kCoef / kUniform.
template <bool kCpml, bool kCoef, bool kUniform>
__device__ __forceinline__ void tma_march(const StepParams& p, const Ring& ring, int n, int lane, int w, int j,
                                          int col) {
  const int NX = p.NX, NY = p.NY, NZ = p.NZ, P = p.P;
  const int k = blockIdx.y * kOut - 1 + lane;
  const bool kok = k >= 0 && k < P;
  const bool out_lane = lane >= 1 && lane <= kOut && k < P;
  const int i0 = blockIdx.z * p.CX;
  const int i1 = ring.i1;
  const int istart = ring.istart;
  const bool jm_ok = j >= 1, jp_ok = j + 1 < NY;
  const int jm = jm_ok ? j - 1 : 0;
  const int kc = kok ? k : 0;
  const int ps = NY * P;
  const int rm = jm * P + kc, rc = j * P + kc;
  const int rw = w * kCols, rw1 = (w + 1) * kCols, rw2 = (w + 2) * kCols;
  (void)jp_ok;

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
  if (p.n_poles && out_lane) {
    const int np_ = min(p.n_poles, 32);
    for (int b = 0; b < np_; ++b) {
      const PoleTerm& pt = p.poles[b];
      if (j >= pt.j0 && j < pt.j1 && k >= pt.k0 && k < pt.k1) lane_poles |= 1u << b;
    }
  }

  float hpz = 0.f, hpy = 0.f;  // Hz, Hy of row j at plane i-1

  if (!ring_wait_full(ring, istart)) {
    report_timeout(p.status);
    return;
  }
  for (int i = istart; i < i1; ++i) {
    const bool own = i >= i0;
    const int o = i * ps;
    if (!ring_wait_full(ring, i + 1)) {
      report_timeout(p.status);
      return;
    }
    const int su = (i - istart) % kStages, sn = (i + 1 - istart) % kStages;
    const float* sE = ring.stages + su * kStageFloats;
    const float* sH = sE + 3 * kEPad;
    const float* sN = ring.stages + sn * kStageFloats;
    const unsigned pb = __ldg(p.plane_bits + i);
    // E^n(i) rows j-1, j, j+1; E^n(i+1) values the H update needs; H^{n-1/2}(i)
    const float em0 = sE[rw + col], em1 = sE[kEPad + rw + col], em2 = sE[2 * kEPad + rw + col];
    const float ec0 = sE[rw1 + col], ec1 = sE[kEPad + rw1 + col], ec2 = sE[2 * kEPad + rw1 + col];
    const float ep0 = sE[rw2 + col], ep2 = sE[2 * kEPad + rw2 + col];
    const float nm1 = sN[kEPad + rw + col], nc1 = sN[kEPad + rw1 + col], nc2 = sN[2 * kEPad + rw1 + col];
    const float hm0 = sH[rw + col], hm2 = sH[2 * kHPad + rw + col];
    const float hc0 = sH[rw1 + col], hc1 = sH[kHPad + rw1 + col], hc2 = sH[2 * kHPad + rw1 + col];
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
      const float em1k = sE[kEPad + rw + col + 1];
    const float ec0k = sE[rw1 + col + 1];
    const float ec1k = sE[kEPad + rw1 + col + 1];

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
      if (pb & kPlanePoles) ade(p, lane_poles, i, j, k, ec0, ec1, ec2, v0, v1, v2);
      if ((pb & kPlaneETerms) || (lf & (kLfETermY | kLfETermZ)))
        add_terms(p, 0, 0, n, i, j, k, pb & kPlaneETerms, lf & kLfETermY, lf & kLfETermZ, v0, v1, v2);
      // scenes without TFSF end the E update on PEC faces (stepping.py:2316-2318)
      if (p.pec_clamp) {
        if (m0 == 2) v0 = 0.f;
        if (m1 == 2) v1 = 0.f;
        if (m2 == 2) v2 = 0.f;
      }
      __stcg(p.Eout[0] + o + rc, v0);
      __stcg(p.Eout[1] + o + rc, v1);
      __stcg(p.Eout[2] + o + rc, v2);
    }
    hpz = hcz;
    hpy = hcy;
    // release plane i's stage
    __syncwarp();
    if (lane == 0) mbar_arrive(ring.empty0 + 8u * su);
  }
}

// Grid as the warp kernel ((NY+7)/8, z blocks, x chunks); block = 8 consumer
// warps + 1 producer warp; dynamic shared memory = tma_smem_bytes().
template <bool kAnyCpml, bool kAnyCoef, bool kUniform>
__global__ void __launch_bounds__(kTmaThreads, 3) tma_step_kernel(const StepParams p, const __grid_constant__ TmaMaps maps, int n) {
  if (p.step_base) n += __ldg(p.step_base);
  extern __shared__ unsigned char smem_raw[];
  float* stages = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  uint64_t* bars = reinterpret_cast<uint64_t*>(stages + kStages * kStageFloats);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i0 = blockIdx.z * p.CX;
  Ring ring;
  ring.stages = stages;
  ring.full0 = smem_addr(bars);
  ring.empty0 = smem_addr(bars + kStages);
  ring.istart = max(i0 - 1, 0);
  ring.i1 = min(i0 + p.CX, p.NX);
  ring.limit = static_cast<uint32_t>(p.wait_limit);
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(ring.full0 + 8u * s, 1);
      mbar_init(ring.empty0 + 8u * s, kTmaRows);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int j0 = blockIdx.x * kTmaRows;
  const int kb = static_cast<int>(blockIdx.y) * kOut - 1;
  const int a = (kb >> 2) << 2;  // 16-byte aligned box start (arithmetic shift floors)

  if (warp == kTmaRows) {
    // ---------------- producer ----------------
    if (lane != 0) return;
    const int planes = ring.i1 - ring.istart + 1;  // istart .. i1
    int issued = 0;
    bool ok = true;
    for (int u = 0; u < planes && ok; ++u) {
      const int s = u % kStages, q = ring.istart + u;
      if (u >= kStages && !mbar_wait(ring.empty0 + 8u * s, ((u / kStages) - 1) & 1, ring.limit)) {
        report_timeout(p.status);
        ok = false;
        break;
      }
      const bool with_h = q < ring.i1;
      const uint32_t bar = ring.full0 + 8u * s;
      mbar_expect_tx(bar, 3 * kEBytes + (with_h ? 3 * kHBytes : 0));
      float* st = stages + s * kStageFloats;
      for (int c = 0; c < 3; ++c) tma_load(smem_addr(st + c * kEPad), &maps.e[c], a, j0 - 1, q, bar);
      if (with_h)
        for (int c = 0; c < 3; ++c) tma_load(smem_addr(st + 3 * kEPad + c * kHPad), &maps.h[c], a, j0 - 1, q, bar);
      issued = u + 1;
    }
    // Every issued copy has landed before the block can exit.
    for (int u = max(0, issued - kStages); u < issued; ++u) {
      if (!mbar_wait(ring.full0 + 8u * (u % kStages), (u / kStages) & 1, kSpinLimit)) {
        report_timeout(p.status);
        break;
      }
    }
    return;
  }

  // ---------------- consumers ----------------
  const int j = j0 + warp;
  if (j >= p.NY) {
    idle_march(ring, lane, p.status);
    return;
  }
  const int col = lane + (kb - a);
  unsigned cls = 0;
  if (kAnyCpml || kAnyCoef)
    cls = __ldg(p.warp_class + (static_cast<int64_t>(blockIdx.z) * gridDim.y + blockIdx.y) * p.NY + j);
  if (kAnyCpml && (cls & kClassCpml)) {
    if (kAnyCoef && (cls & kClassCoef)) tma_march<true, true, kUniform>(p, ring, n, lane, warp, j, col);
    else tma_march<true, false, kUniform>(p, ring, n, lane, warp, j, col);
  } else {
    if (kAnyCoef && (cls & kClassCoef)) tma_march<false, true, kUniform>(p, ring, n, lane, warp, j, col);
    else tma_march<false, false, kUniform>(p, ring, n, lane, warp, j, col);
  }
}

size_t tma_smem_bytes() { return sizeof(float) * kStages * kStageFloats + 2 * kStages * sizeof(uint64_t) + 128; }

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(ptr);
  }
  return fn;
}

}  // namespace

int encode_field_map(CUtensorMap* map, const float* base, int NX, int NY, int P, int rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return -1;
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(P), static_cast<cuuint64_t>(NY), static_cast<cuuint64_t>(NX)};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(P) * 4, static_cast<cuuint64_t>(P) * NY * 4};
  const cuuint32_t box[3] = {static_cast<cuuint32_t>(kCols), static_cast<cuuint32_t>(rows), 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : static_cast<int>(r);
}

int tma_rows_e() { return kERows; }
int tma_rows_h() { return kHRows; }

#define FDTD_TMA_INSTANTIATE(CPML, COEF, UNI) \
  template __global__ void tma_step_kernel<CPML, COEF, UNI>(const StepParams, const __grid_constant__ TmaMaps, int);
FDTD_TMA_INSTANTIATE(false, false, false)
FDTD_TMA_INSTANTIATE(false, true, false)
FDTD_TMA_INSTANTIATE(true, false, false)
FDTD_TMA_INSTANTIATE(true, true, false)
FDTD_TMA_INSTANTIATE(false, false, true)
FDTD_TMA_INSTANTIATE(false, true, true)
FDTD_TMA_INSTANTIATE(true, false, true)
FDTD_TMA_INSTANTIATE(true, true, true)
#undef FDTD_TMA_INSTANTIATE

}  // namespace fdtdb200
