// Row-tile fused leapfrog step, TMA-fed (launch variant 10): one launch
// advances H^{n-1/2} -> H^{n+1/2} and E^n -> E^{n+1} over the whole grid.
//
// A CTA covers rows j0 .. j0+7 and one z block of 30 output cells (lane l <->
// k = 30 s - 1 + l; lanes 0 and 31 are the z halo) and marches +x over a chunk
// of planes.  Its ten warps:
//   - a producer warp whose elected lane streams each plane's tiles with
//     cp.async.bulk.tensor (TMA, no multicast) into a ring of stages, several
//     planes ahead: E^n rows j0-1 .. j0+8 and H^{n-1/2} rows j0-1 .. j0+7, 36 z
//     cells from a 16-byte aligned start (the tensor maps of tma_kernel.cu);
//   - eight row warps (row j = j0 + w) that read every operand of their row
//     from shared memory (own row, row j+1, z+1 column, next plane), so the
//     march issues no global loads and no per-lane address arithmetic for them;
//   - one halo warp that computes H^{n+1/2} Hz, Hx of row j0-1 (the E update
//     of row j0 needs them) from the same tiles.
// Per plane i: every consumer waits for the stage of plane i+1, computes
// H(i), publishes Hz, Hx in a small exchange buffer, meets the other consumers
// at a named barrier, computes E^{n+1}(i) from H of row j-1 (exchange
// buffer), its own H(i) and H(i-1) (registers) and the z-1 neighbours
// (__shfl_up), stores H(i) and E(i), and releases the stage of plane i.  The
// exchange buffer alternates between two planes: a buffer written before the
// barrier of plane i is read after it and next written before the barrier of
// plane i+2.
//
// Every wait is bounded (StepParams::wait_limit polling rounds).  A wait that
// runs out records FDTD_ERR_TIMEOUT in p.status; the warp then carries on
// without waiting (its values are garbage, which the status makes the host
// discard) so that every consumer still meets every named barrier, and the
// producer stops issuing and waits, with its own fixed bound, for the copies
// it issued before the block exits.
//
// Per-warp bodies (template switches): kCoef (per-cell coefficient arrays),
// kEdge (the row or z block touches a domain face or lanes leave a
// component's extent; interior bodies carry no masks and only planes 0 and
// NX - 1 take the edge path), kTerms (an injection term reaches the warp's
// chunk).  CPML slabs are not handled here: with CPML in the scene, the CTAs
// that meet a slab return at once and the warp kernel (warp_kernel.cu), whose
// independent warps hide the psi loads better than a CTA held together by a
// per-plane barrier, runs exactly those CTAs after this kernel.  Poles are not
// compiled in: the ADE pass (ade_pass.cu) runs them after both.  Periodic /
// Bloch faces are not handled here; those engines use the warp kernel.
//
// Arithmetic restated from witwin/maxwell/fdtd/cuda/kernels/magnetic.cu:62-212,
// electric.cu:242-311 and 462-941, sources.cu:135-154 and 485-545.
#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/fdtd_b200.h"
#include "step_device.cuh"
#include "tma_step.cuh"

namespace fdtdb200 {

namespace {

constexpr int kRows = 8;                      // row warps per CTA
constexpr int kConsumers = (kRows + 1) * 32;  // row warps + halo warp (named barrier 1)
constexpr int kThreads = kConsumers + 32;     // + producer warp
constexpr int kCols = 36;                     // z cells per tile row
constexpr int kEPad = 384;                    // floats per E component tile (10 x 36, 128-byte multiple)
constexpr int kHPad = 352;                    // floats per H component tile (9 x 36)
constexpr int kStage = 3 * kEPad + 3 * kHPad;
constexpr uint32_t kEBytes = kCols * (kRows + 2) * 4;
constexpr uint32_t kHBytes = kCols * (kRows + 1) * 4;
constexpr uint32_t kDrainLimit = 1u << 20;  // polling rounds of the producer's final drain

static_assert((kEPad * 4) % 128 == 0 && (kHPad * 4) % 128 == 0, "tiles must stay 128-byte aligned");
static_assert(kCols * (kRows + 2) <= kEPad && kCols * (kRows + 1) <= kHPad, "tile pads too small");

__device__ __forceinline__ uint32_t saddr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// Bounded wait for the phase of parity `parity`; false when `limit` polls ran out.
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
// Named barrier of the nine consumer warps (the producer never joins it).
__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kConsumers) : "memory"); }

template <int R>
struct Ring {
  float* stages;   // R x kStage floats
  float* xbuf;     // H^{n+1/2} exchange: [2][kRows + 1][2][32] (rows j0-1 .. j0+7; Hz, Hx)
  uint32_t full0;  // shared address of full[0] (8 bytes apart)
  uint32_t empty0; // shared address of empty[0]
  int istart, i1;  // planes istart .. i1 - 1 are computed; istart .. i1 are loaded
  uint32_t limit;  // polling rounds of a consumer wait
  int* status;
};

// Wait for the stage of plane q; on timeout record it and go on without waiting.
template <int R>
__device__ __forceinline__ void wait_plane(const Ring<R>& r, int q, bool& ok) {
  const int u = q - r.istart;
  if (ok && !mbar_wait(r.full0 + 8u * (u % R), (u / R) & 1, r.limit)) {
    ok = false;
    if ((threadIdx.x & 31) == 0) atomicExch(r.status, FDTD_ERR_TIMEOUT);
  }
}

// One elected lane of the (converged) warp arrives on the stage's empty barrier.
template <int R>
__device__ __forceinline__ void release_plane(const Ring<R>& r, int q, int lane) {
  (void)lane;
  const uint32_t bar = r.empty0 + 8u * ((q - r.istart) % R);
  asm volatile(
      "{\n\t.reg .pred P;\n\t"
      "elect.sync _|P, 0xffffffff;\n\t"
      "@P mbarrier.arrive.shared::cta.b64 _, [%0];\n\t}" ::"r"(bar)
      : "memory");
}

__device__ __forceinline__ float sel(bool ok, float v) { return ok ? v : 0.0f; }

// Loop-invariant data of a row warp.
struct RowCtx {
  int k, rc, ps, i0, w, j, col;
  bool kok, out_lane, hz_kok, ez_kok, yc_ok, lane_edge, ylo, yhi, zlo, zhi;
  float ihz, iez, ihy_c, iey;
  unsigned lf;
};

// One plane of a row warp.  hpz, hpy: Hz, Hy of plane i-1 (updated to plane i).
// Planes before i0 (the halo plane i0 - 1) compute H only, for the next plane;
// planes 0 and NX - 1 take the edge path.  pb: the plane's kPlane* bits;
// kTerms: the warp meets an injection term in its chunk.
template <int R, bool kCoef, bool kUniform, bool kEdge, bool kTerms>
__device__ __forceinline__ void row_plane(const StepParams& p, const Ring<R>& ring, const RowCtx& c, int n, int lane,
                                          int i, unsigned pb, float& hpz, float& hpy, bool& ok) {
  const int NX = p.NX;
  const int u = i - ring.istart;
  const int o = i * c.ps + c.rc;
  const bool own = i >= c.i0;
  const bool plane_edge = i == 0 || i == NX - 1;
  const bool ix_ok = i < NX - 1;
  const bool cy_ok = ix_ok && c.hz_kok, cz_ok = ix_ok && c.yc_ok && c.ez_kok, cx_ok = c.yc_ok && c.hz_kok;
  // Coefficient arrays are loaded before the stage wait, so their latency
  // overlaps it: a warp that waits on them holds up the whole CTA at the named
  // barrier.
  float g0 = p.edecay_u[0], g1 = p.edecay_u[1], g2 = p.edecay_u[2];
  float c0 = p.ecurl_u[0], c1 = p.ecurl_u[1], c2 = p.ecurl_u[2];
  float dHx = p.hdecay_u[0], cHx = p.hcurl_u[0], dHy = p.hdecay_u[1], cHy = p.hcurl_u[1], dHz = p.hdecay_u[2],
        cHz = p.hcurl_u[2];
  if (kCoef) {
    const bool ld = own && c.out_lane;
    if (p.ecurl[0]) c0 = ldz(p.ecurl[0], o, ld);
    if (p.ecurl[1]) c1 = ldz(p.ecurl[1], o, ld);
    if (p.ecurl[2]) c2 = ldz(p.ecurl[2], o, ld);
    if (p.edecay[0]) g0 = ldz(p.edecay[0], o, ld);
    if (p.edecay[1]) g1 = ldz(p.edecay[1], o, ld);
    if (p.edecay[2]) g2 = ldz(p.edecay[2], o, ld);
    if (p.hdecay[0]) dHx = ldz(p.hdecay[0], o, c.kok);
    if (p.hcurl[0]) cHx = ldz(p.hcurl[0], o, c.kok);
    if (p.hdecay[1]) dHy = ldz(p.hdecay[1], o, c.kok);
    if (p.hcurl[1]) cHy = ldz(p.hcurl[1], o, c.kok);
    if (p.hdecay[2]) dHz = ldz(p.hdecay[2], o, c.kok);
    if (p.hcurl[2]) cHz = ldz(p.hcurl[2], o, c.kok);
  }
  wait_plane(ring, i + 1, ok);
  const float* st = ring.stages + (u % R) * kStage;
  const float* sn = ring.stages + ((u + 1) % R) * kStage;
  const int rw = (c.w + 1) * kCols + c.col;  // row j inside the E and H tiles
  const int rp = rw + kCols;                 // row j + 1 (E tile)
  const float e0 = st[rw], e1 = st[kEPad + rw], e2 = st[2 * kEPad + rw];
  const float e0k = st[rw + 1], e1k = st[kEPad + rw + 1];
  const float exp_ = st[rp], ezp = st[2 * kEPad + rp];
  const float n1 = sn[kEPad + rw], n2 = sn[2 * kEPad + rw];
  const float* sh = st + 3 * kEPad;
  const float h0 = sh[rw], h1 = sh[kHPad + rw], h2 = sh[2 * kHPad + rw];
  const float ihx = kUniform ? p.inv_h_u[0] : __ldg(p.inv_h[0] + (i < NX - 1 ? i : 0));

  // ---------------- H^{n+1/2}(i), row j ----------------
  // Hx: dEz/dy - dEy/dz; Hy: dEx/dz - dEz/dx; Hz: dEy/dx - dEx/dy
  float cxa = (ezp - e2) * c.ihy_c, cxb = (e1k - e1) * c.ihz;
  float cya = (n2 - e2) * ihx, cyb = (e0k - e0) * c.ihz;
  float cza = (n1 - e1) * ihx, czb = (exp_ - e0) * c.ihy_c;
  float hx = h0 * dHx - cHx * (cxa - cxb);
  float hy = h1 * dHy - cHy * (cyb - cya);
  float hz = h2 * dHz - cHz * (cza - czb);
  if (kEdge) {
    hx = sel(cx_ok, hx);
    hy = sel(cy_ok, hy);
    hz = sel(cz_ok, hz);
  } else if (plane_edge) {  // plane NX - 1 lies outside the Hy, Hz extents
    hy = sel(i < NX - 1, hy);
    hz = sel(i < NX - 1, hz);
  }
  if (kTerms && c.kok && ((pb & kPlaneHTerms) || (c.lf & (kLfHTermYc | kLfHTermZ))))
    add_terms(p, 1, 3, n, i, c.j, c.k, pb & kPlaneHTerms, c.lf & kLfHTermYc, c.lf & kLfHTermZ, hx, hy, hz);
  float* xb = ring.xbuf + (u & 1) * (kRows + 1) * 64;
  xb[(c.w + 1) * 64 + lane] = hz;
  xb[(c.w + 1) * 64 + 32 + lane] = hx;
  consumer_sync();

  // ---------------- E^{n+1}(i), row j ----------------
  const float hzm = xb[c.w * 64 + lane], hxm = xb[c.w * 64 + 32 + lane];  // row j-1
  const float hxk = __shfl_up_sync(kFull, hx, 1);
  const float hyk = __shfl_up_sync(kFull, hy, 1);
  if (own && c.out_lane) {
    const float iex = kUniform ? p.inv_e_u[0] : __ldg(p.inv_e[0] + i);
    // Ex: dHz/dy - dHy/dz; Ey: dHx/dz - dHz/dx; Ez: dHy/dx - dHx/dy
    float d0a = (hz - hzm) * c.iey, d0b = (hy - hyk) * c.iez;
    float d1a = (hz - hpz) * iex, d1b = (hx - hxk) * c.iez;
    float d2a = (hy - hpy) * iex, d2b = (hx - hxm) * c.iey;
    int m0 = 0, m1 = 0, m2 = 0;
    if (kEdge ? (c.lane_edge || plane_edge) : plane_edge) {
      const bool xlo = i == 0, xhi = i == NX - 1;
      m0 = edge_mode(i < NX - 1 && c.ez_kok, c.ylo, c.yhi, c.zlo, c.zhi, p.bnd[2], p.bnd[3], p.bnd[4], p.bnd[5]);
      m1 = edge_mode(c.yc_ok && c.ez_kok, xlo, xhi, c.zlo, c.zhi, p.bnd[0], p.bnd[1], p.bnd[4], p.bnd[5]);
      m2 = edge_mode(c.hz_kok, xlo, xhi, c.ylo, c.yhi, p.bnd[0], p.bnd[1], p.bnd[2], p.bnd[3]);
    }
    float v0 = pick(m0, e0 * g0 + c0 * (d0a - d0b), e0);
    float v1 = pick(m1, e1 * g1 + c1 * (d1b - d1a), e1);
    float v2 = pick(m2, e2 * g2 + c2 * (d2a - d2b), e2);
    if (kTerms && ((pb & kPlaneETerms) || (c.lf & (kLfETermY | kLfETermZ))))
      add_terms(p, 0, 0, n, i, c.j, c.k, pb & kPlaneETerms, c.lf & kLfETermY, c.lf & kLfETermZ, v0, v1, v2);
    // scenes without TFSF end the E update on PEC faces (stepping.py:2316-2318)
    if (p.pec_clamp) {
      if (m0 == 2) v0 = 0.f;
      if (m1 == 2) v1 = 0.f;
      if (m2 == 2) v2 = 0.f;
    }
    __stcg(p.Hout[0] + o, hx);
    __stcg(p.Hout[1] + o, hy);
    __stcg(p.Hout[2] + o, hz);
    __stcg(p.Eout[0] + o, v0);
    __stcg(p.Eout[1] + o, v1);
    __stcg(p.Eout[2] + o, v2);
  }
  hpz = hz;
  hpy = hy;
  release_plane(ring, i, lane);
}

// The planes istart .. i1 - 1 of a chunk with the body of one warp class.
template <int R, bool kCoef, bool kUniform, bool kEdge, bool kTerms, class PBits>
__device__ __forceinline__ void planes(const StepParams& p, const Ring<R>& ring, const RowCtx& c, int n, int lane,
                                       PBits pbits) {
  bool ok = true;
  wait_plane(ring, ring.istart, ok);
  float hpz = 0.f, hpy = 0.f;  // H of plane istart - 1: read only for owned planes (i >= i0 > istart)
  for (int i = ring.istart; i < ring.i1; ++i)
    row_plane<R, kCoef, kUniform, kEdge, kTerms>(p, ring, c, n, lane, i, pbits(i), hpz, hpy, ok);
}

template <int R, bool kCoef, bool kUniform, bool kEdge>
__device__ __forceinline__ void row_march(const StepParams& p, const Ring<R>& ring, int n, int lane, int w, int j,
                                          int col) {
  const int NY = p.NY, NZ = p.NZ, P = p.P;
  RowCtx c;
  c.w = w;
  c.j = j;
  c.col = col;
  c.k = blockIdx.y * kOut - 1 + lane;
  c.kok = kEdge ? (c.k >= 0 && c.k < P) : true;
  c.out_lane = lane >= 1 && lane <= kOut && (kEdge ? c.k < P : true);
  c.i0 = blockIdx.z * p.CX;
  c.ps = NY * P;
  c.rc = j * P + (c.kok ? c.k : 0);
  c.hz_kok = kEdge ? (c.k >= 0 && c.k < NZ - 1) : true;
  c.ez_kok = kEdge ? (c.k >= 0 && c.k < NZ) : true;
  c.yc_ok = kEdge ? j < NY - 1 : true;
  c.ihz = kUniform ? p.inv_h_u[2] : __ldg(p.inv_h[2] + (c.hz_kok ? c.k : 0));
  c.iez = kUniform ? p.inv_e_u[2] : __ldg(p.inv_e[2] + (c.ez_kok ? c.k : 0));
  c.ihy_c = kUniform ? p.inv_h_u[1] : __ldg(p.inv_h[1] + (c.yc_ok ? j : 0));
  c.iey = kUniform ? p.inv_e_u[1] : __ldg(p.inv_e[1] + j);
  c.ylo = j == 0;
  c.yhi = j == NY - 1;
  c.zlo = c.k == 0;
  c.zhi = c.k == NZ - 1;
  c.lane_edge = c.ylo || c.yhi || c.k <= 0 || c.k >= NZ - 1;
  c.lf = 0;
  if (p.n_terms[1]) {
    if (list_nonempty(p.term_index[1], 1, j)) c.lf |= kLfHTermYc;
    if (c.kok && list_nonempty(p.term_index[1], 2, c.k)) c.lf |= kLfHTermZ;
  }
  if (p.n_terms[0]) {
    if (list_nonempty(p.term_index[0], 1, j)) c.lf |= kLfETermY;
    if (c.kok && list_nonempty(p.term_index[0], 2, c.k)) c.lf |= kLfETermZ;
  }
  // kPlane* bits of the chunk's planes istart .. istart + 63, gathered once
  // (lane l reads planes istart + l and istart + 32 + l); chunks are at most
  // 63 planes long
  uint64_t bits_h = 0, bits_e = 0;
  if (p.n_terms[0] | p.n_terms[1]) {
    for (int half = 0; half < 2; ++half) {
      const int q = ring.istart + 32 * half + lane;
      const unsigned pb = q < ring.i1 ? __ldg(p.plane_bits + q) : 0u;
      bits_h |= static_cast<uint64_t>(__ballot_sync(kFull, pb & kPlaneHTerms)) << (32 * half);
      bits_e |= static_cast<uint64_t>(__ballot_sync(kFull, pb & kPlaneETerms)) << (32 * half);
    }
  }
  auto pbits = [&](int i) -> unsigned {
    const int u = i - ring.istart;
    return (static_cast<unsigned>(bits_h >> u) & 1u) * kPlaneHTerms | (static_cast<unsigned>(bits_e >> u) & 1u) * kPlaneETerms;
  };
  // warps that no injection term reaches in this chunk run a body without the
  // term code (a warp-uniform choice: both bodies meet the named barrier)
  const bool terms = (bits_h | bits_e) != 0 || __any_sync(kFull, c.lf != 0);
  if (terms) planes<R, kCoef, kUniform, kEdge, true>(p, ring, c, n, lane, pbits);
  else planes<R, kCoef, kUniform, kEdge, false>(p, ring, c, n, lane, [](int) { return 0u; });
}

// A row warp whose row lies beyond the grid: publishes zeros, keeps the named
// barrier count and releases every stage.
template <int R>
__device__ __forceinline__ void idle_march(const Ring<R>& ring, int lane, int w) {
  for (int i = ring.istart; i < ring.i1; ++i) {
    const int u = i - ring.istart;
    float* xb = ring.xbuf + (u & 1) * (kRows + 1) * 64;
    xb[(w + 1) * 64 + lane] = 0.0f;
    xb[(w + 1) * 64 + 32 + lane] = 0.0f;
    consumer_sync();
    release_plane(ring, i, lane);
  }
}

// Halo warp: H^{n+1/2} Hz, Hx of row a = j0 - 1 from tile rows 0 (row a) and 1
// (row j0).
template <int R, bool kCoef, bool kUniform>
__device__ __forceinline__ void halo_march(const StepParams& p, const Ring<R>& ring, int n, int lane, int j0, int col) {
  const int NX = p.NX, NY = p.NY, NZ = p.NZ, P = p.P;
  const int k = blockIdx.y * kOut - 1 + lane;
  const bool kok = k >= 0 && k < P;
  const int ja = j0 - 1;
  const bool a_ok = ja >= 0;
  const bool hz_kok = k >= 0 && k < NZ - 1, ez_kok = k >= 0 && k < NZ;
  const int ps = NY * P;
  unsigned lfa = 0;
  if (a_ok && p.n_terms[1]) {
    if (list_nonempty(p.term_index[1], 1, ja)) lfa |= kLfHTermYm;
    if (kok && list_nonempty(p.term_index[1], 2, k)) lfa |= kLfHTermZ;
  }
  const float ihz = kUniform ? p.inv_h_u[2] : __ldg(p.inv_h[2] + (hz_kok ? k : 0));
  const float ihy = kUniform ? p.inv_h_u[1] : __ldg(p.inv_h[1] + (a_ok ? ja : 0));
  bool ok = true;
  wait_plane(ring, ring.istart, ok);
  for (int i = ring.istart; i < ring.i1; ++i) {
    const int u = i - ring.istart;
    wait_plane(ring, i + 1, ok);
    const float* st = ring.stages + (u % R) * kStage;
    const float* sn = ring.stages + ((u + 1) % R) * kStage;
    float hx = 0.f, hz = 0.f;
    if (a_ok) {
      const bool ix_ok = i < NX - 1;
      const bool mx_ok = hz_kok, mz_ok = ix_ok && ez_kok;  // row a < NY - 1 always
      const float ihx = kUniform ? p.inv_h_u[0] : __ldg(p.inv_h[0] + (ix_ok ? i : 0));
      const int r0 = col, r1 = kCols + col;  // rows a and j0
      const float e0 = st[r0], e1 = st[kEPad + r0], e2 = st[2 * kEPad + r0];
      const float e1k = st[kEPad + r0 + 1];
      const float ezj = st[2 * kEPad + r1], exj = st[r1];
      const float n1 = sn[kEPad + r0];
      float mxa = (ezj - e2) * ihy, mxb = (e1k - e1) * ihz;
      float mza = (n1 - e1) * ihx, mzb = (exj - e0) * ihy;
      const int oa = i * ps + ja * P + (kok ? k : 0);
      float dHx = p.hdecay_u[0], cHx = p.hcurl_u[0], dHz = p.hdecay_u[2], cHz = p.hcurl_u[2];
      if (kCoef) {
        if (p.hdecay[0]) dHx = ldz(p.hdecay[0], oa, kok);
        if (p.hcurl[0]) cHx = ldz(p.hcurl[0], oa, kok);
        if (p.hdecay[2]) dHz = ldz(p.hdecay[2], oa, kok);
        if (p.hcurl[2]) cHz = ldz(p.hcurl[2], oa, kok);
      }
      const float* sh = st + 3 * kEPad;
      hx = mx_ok ? sh[r0] * dHx - cHx * (mxa - mxb) : 0.f;
      hz = mz_ok ? sh[2 * kHPad + r0] * dHz - cHz * (mza - mzb) : 0.f;
      if (p.n_terms[1] && kok) {
        const unsigned pb = __ldg(p.plane_bits + i);
        if ((pb & kPlaneHTerms) || (lfa & (kLfHTermYm | kLfHTermZ))) {
          float hy = 0.f;
          add_terms(p, 1, 3, n, i, ja, k, pb & kPlaneHTerms, lfa & kLfHTermYm, lfa & kLfHTermZ, hx, hy, hz);
        }
      }
    }
    float* xb = ring.xbuf + (u & 1) * (kRows + 1) * 64;
    xb[lane] = hz;
    xb[32 + lane] = hx;
    consumer_sync();
    release_plane(ring, i, lane);
  }
}

// Grid: ((NY + 7) / 8, z blocks of 30 cells, x chunks of p.CX planes) -- the
// warp kernel's grid; block: 8 row warps, the halo warp, the producer warp;
// dynamic shared memory: smem_bytes<R>().
template <int R>
constexpr size_t smem_bytes() {
  return sizeof(float) * (R * kStage + 2 * (kRows + 1) * 64) + 2 * R * sizeof(uint64_t);
}

template <int R, bool kAnyCpml, bool kAnyCoef, bool kUniform>
__global__ void __launch_bounds__(kThreads, 3) tile_step_kernel(const StepParams p, const __grid_constant__ TmaMaps maps,
                                                                int n) {
  // dynamic shared memory starts the CTA's shared window (no static shared
  // data here), so it is aligned far beyond the 128 bytes the tiles need; it
  // is indexed directly so that every access stays a shared-memory access
  extern __shared__ __align__(1024) float smem_f[];
  if (p.step_base) n += __ldg(p.step_base);
  float* stages = smem_f;
  Ring<R> ring;
  ring.stages = stages;
  ring.xbuf = stages + R * kStage;
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring.xbuf + 2 * (kRows + 1) * 64);
  ring.full0 = saddr(bars);
  ring.empty0 = saddr(bars + R);
  const int i0 = blockIdx.z * p.CX;
  ring.istart = max(i0 - 1, 0);
  ring.i1 = min(i0 + p.CX, p.NX);
  ring.limit = static_cast<uint32_t>(p.wait_limit);
  ring.status = p.status;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < R; ++s) {
      mbar_init(ring.full0 + 8u * s, 1);
      mbar_init(ring.empty0 + 8u * s, kRows + 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  const int j0 = blockIdx.x * kRows;
  // Warp classes (kClass* bits of the warp-task table, whose footprint covers
  // rows j - 1 and j): a row warp takes its row's, the halo warp row j0's.
  // With CPML in the scene this kernel leaves every CTA that meets a slab to
  // the warp kernel, which runs those CTAs alone (the same rows j0 - 1 .. j0 + 7
  // decide there); the row-tile bodies carry no psi code.
  unsigned cls = 0;
  if ((kAnyCpml || kAnyCoef) && warp <= kRows) {
    const int jr = warp == kRows ? min(j0, p.NY - 1) : j0 + warp;
    if (jr < p.NY)
      cls = __ldg(p.warp_class + (static_cast<int64_t>(blockIdx.z) * gridDim.y + blockIdx.y) * p.NY + jr);
  }
  const int cta_cpml = __syncthreads_or(kAnyCpml ? (cls & kClassCpml) : 0u);
  if (cta_cpml) return;
  const int kb = static_cast<int>(blockIdx.y) * kOut - 1;
  const int a = (kb >> 2) << 2;  // 16-byte aligned box start (arithmetic shift floors)
  const int col = lane + (kb - a);

  if (warp == kRows + 1) {
    // ---------------- producer ----------------
    if (lane != 0) return;
    const int planes = ring.i1 - ring.istart + 1;  // istart .. i1
    int issued = 0;
    for (int u = 0; u < planes; ++u) {
      const int s = u % R, q = ring.istart + u;
      if (u >= R && !mbar_wait(ring.empty0 + 8u * s, ((u / R) - 1) & 1, ring.limit)) {
        atomicExch(p.status, FDTD_ERR_TIMEOUT);
        break;
      }
      const bool with_h = q < ring.i1;
      const uint32_t bar = ring.full0 + 8u * s;
      mbar_expect_tx(bar, 3 * kEBytes + (with_h ? 3 * kHBytes : 0));
      float* st = stages + s * kStage;
      for (int c = 0; c < 3; ++c) tma_load(saddr(st + c * kEPad), &maps.e[c], a, j0 - 1, q, bar);
      if (with_h)
        for (int c = 0; c < 3; ++c) tma_load(saddr(st + 3 * kEPad + c * kHPad), &maps.h[c], a, j0 - 1, q, bar);
      issued = u + 1;
    }
    // every issued copy lands before the block can exit
    for (int u = max(0, issued - R); u < issued; ++u) {
      if (!mbar_wait(ring.full0 + 8u * (u % R), (u / R) & 1, kDrainLimit)) {
        atomicExch(p.status, FDTD_ERR_TIMEOUT);
        break;
      }
    }
    return;
  }
  if (warp == kRows) {
    if (kAnyCoef && (cls & kClassCoef)) halo_march<R, true, kUniform>(p, ring, n, lane, j0, col);
    else halo_march<R, false, kUniform>(p, ring, n, lane, j0, col);
    return;
  }
  const int j = j0 + warp;
  if (j >= p.NY) {
    idle_march(ring, lane, warp);
    return;
  }
  const bool edge = j == 0 || j >= p.NY - 1 || kb < 1 || kb + 31 > p.NZ - 2;
  if (kAnyCoef && (cls & kClassCoef)) {
    if (edge) row_march<R, true, kUniform, true>(p, ring, n, lane, warp, j, col);
    else row_march<R, true, kUniform, false>(p, ring, n, lane, warp, j, col);
  } else {
    if (edge) row_march<R, false, kUniform, true>(p, ring, n, lane, warp, j, col);
    else row_march<R, false, kUniform, false>(p, ring, n, lane, warp, j, col);
  }
}

// R: stages of the TMA ring.
template <int R>
int launch_ring(const StepParams& p, const TmaMaps& maps, int n, dim3 grid, bool cpml, bool coef, bool uni,
                cudaStream_t stream) {
  constexpr size_t bytes = smem_bytes<R>();
  // dynamic shared memory beyond 48 KB is opted into per kernel (and per
  // device context), so the attribute is set before every launch: a host-side
  // call of a few microseconds that needs no stream and is allowed while
  // capturing a graph
#define FDTD_TILE(CPML, COEF, UNI)                                                                         \
  do {                                                                                                     \
    auto kern = tile_step_kernel<R, CPML, COEF, UNI>;                                                      \
    const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,          \
                                               static_cast<int>(bytes));                                  \
    if (e != cudaSuccess) return static_cast<int>(e);                                                      \
    kern<<<grid, kThreads, bytes, stream>>>(p, maps, n);                                                   \
  } while (0)
  if (uni) {
    if (cpml) {
      if (coef) FDTD_TILE(true, true, true);
      else FDTD_TILE(true, false, true);
    } else {
      if (coef) FDTD_TILE(false, true, true);
      else FDTD_TILE(false, false, true);
    }
  } else {
    if (cpml) {
      if (coef) FDTD_TILE(true, true, false);
      else FDTD_TILE(true, false, false);
    } else {
      if (coef) FDTD_TILE(false, true, false);
      else FDTD_TILE(false, false, false);
    }
  }
#undef FDTD_TILE
  return static_cast<int>(cudaGetLastError());
}

}  // namespace

int tile_block_threads() { return kThreads; }

// A four-stage ring: the consumers hold planes i and i + 1 while planes i + 2
// and i + 3 are in flight.  Six- and eight-stage rings measured no faster on
// the 256^3 workloads (the march is not waiting on these loads).
int launch_tile_step(const StepParams& p, const TmaMaps& maps, int n, dim3 grid, bool cpml, bool coef, bool uni,
                     cudaStream_t stream) {
  return launch_ring<4>(p, maps, n, grid, cpml, coef, uni, stream);
}

}  // namespace fdtdb200
