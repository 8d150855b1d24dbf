// ADE pass: the Debye / Drude / Lorentz pole update of one step as a
// streaming kernel after the fused step kernel, over the cells the pole boxes
// cover.  The step kernel then writes E^{n+1} without the polarisation term
// (it is launched with no poles), and this pass, per cell,
//   - advances every pole covering the cell from E^n (the step's input buffer,
//     left intact by the ping-pong layout),
//   - subtracts dt J^{n+1} / eps of each pole from E^{n+1}, in pole order.
// That is the reference's order: the E update, then TFSF and source terms,
// then the dispersive correction (witwin/maxwell/fdtd/runtime/stepping.py:
// 2290-2316; ADE arithmetic of witwin/maxwell/fdtd/cuda/kernels/dispersive.cu:
// 18-83).  Inside the 64-register step kernel the pole loads of a cell are
// consumed as they arrive, one pole after another.  Here a thread's only
// dependent read is its tile; the pole table sits in the kernel parameters
// (constant cache) and is read once per pole per tile, and each lane loads the
// state of a pole for all its cells together.
//
// Work list: one warp per tile {row = i * NY + j, k0, k1, pole mask} of up to
// 32 * kAdeCellsPerLane cells [k0, k1) of one row; the mask holds the poles
// whose box covers row (i, j) and meets [k0, k1).  The host builds the tiles
// from the union of the pole boxes per row.  A cell that no pole of a touched
// component covers is written back unchanged (every cell lies in one tile).
#include "step_device.cuh"

namespace fdtdb200 {

namespace {

// Cells per lane: a tile is kAdeCellsPerLane * 32 consecutive z cells of a row,
// lane l taking k0 + l + 32 q.  Each pole's table entry is then read once per
// tile, and a lane has the state loads of all its cells in flight together.
// Four CTAs per SM (64 registers): measured 2.3 % faster per step on the
// dispersive workload than the unbounded 70-register build (three CTAs), and
// than two cells per lane.
constexpr int kQ = kAdeCellsPerLane;

__global__ void __launch_bounds__(256, 4) ade_pass_kernel(const __grid_constant__ AdeParams a,
                                                       const int4* __restrict__ tiles, int n_tiles) {
  const int t = static_cast<int>(blockIdx.x) * (blockDim.x >> 5) + static_cast<int>(threadIdx.x >> 5);
  if (t >= n_tiles) return;  // whole warp
  const int4 tl = __ldg(tiles + t);
  const int lane = static_cast<int>(threadIdx.x & 31);
  const int i = tl.x / a.NY;
  const int j = tl.x - i * a.NY;
  const int64_t row = static_cast<int64_t>(tl.x) * a.P;
  const unsigned mask = static_cast<unsigned>(tl.w);  // the same for every lane
  unsigned comps = 0;
  for (unsigned m = mask; m; m &= m - 1) comps |= 1u << a.poles[__ffs(m) - 1].comp;
  bool in[kQ];
#pragma unroll
  for (int q = 0; q < kQ; ++q) in[q] = tl.y + lane + 32 * q < tl.z;
  // E^n and E^{n+1} of the touched components
  float eo[kQ][3], v[kQ][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const bool use = (comps >> c) & 1u;
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
      const int64_t x = row + tl.y + lane + 32 * q;
      eo[q][c] = use && in[q] ? __ldg(a.Ein[c] + x) : 0.f;
      v[q][c] = use && in[q] ? a.Eout[c][x] : 0.f;
    }
  }
  // poles in id order (the order of the subtractions)
  for (unsigned m = mask; m; m &= m - 1) {
    const AdePole& pt = a.poles[__ffs(m) - 1];
    const int c = pt.comp, kind = pt.kind;
    const int64_t rbase = (static_cast<int64_t>(i - pt.i0) * pt.nj + (j - pt.j0)) * pt.nkk - pt.kk0;
    bool act[kQ];
    float drive[kQ], ie[kQ], pol[kQ], cur[kQ];
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
      const int k = tl.y + lane + 32 * q;
      act[q] = in[q] && k >= pt.k0 && k < pt.k1;
      drive[q] = ie[q] = pol[q] = cur[q] = 0.f;
      if (act[q]) {
        drive[q] = __ldg(pt.drive + rbase + k);
        ie[q] = __ldg(pt.inv_eps + rbase + k);
        if (kind != 1) pol[q] = pt.pol[rbase + k];
        if (kind != 0) cur[q] = pt.cur[rbase + k];
      }
    }
    const float decay = pt.decay, restoring = pt.restoring, dt = pt.dt, inv_dt = pt.inv_dt;
    // nonlinear scenes: J times this step's curl coefficient (dt 1)
    const float* nlc = a.nl_curl[c];
    const float dt_apply = nlc ? 1.0f : dt;
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
      if (!act[q]) continue;
      const int64_t o = rbase + tl.y + lane + 32 * q;
      const float ec = c == 0 ? eo[q][0] : (c == 1 ? eo[q][1] : eo[q][2]);
      float jn;
      if (kind == 0) {
        const float prev = pol[q];
        const float next = decay * prev + drive[q] * ec;
        pt.pol[o] = next;
        jn = (next - prev) * inv_dt;
        pt.cur[o] = jn;
      } else if (kind == 1) {
        jn = decay * cur[q] + drive[q] * ec;
        pt.cur[o] = jn;
      } else {
        const float pl = pol[q];
        jn = decay * cur[q] - restoring * pl + drive[q] * ec;
        pt.cur[o] = jn;
        pt.pol[o] = pl + dt * jn;
      }
      const float s = dt_apply * jn * (nlc ? __ldg(nlc + row + tl.y + lane + 32 * q) : ie[q]);
      if (c == 0) v[q][0] -= s;
      else if (c == 1) v[q][1] -= s;
      else v[q][2] -= s;
    }
  }
  // tangential E on PEC faces stays zero (scenes without TFSF,
  // witwin/maxwell/fdtd/runtime/stepping.py:2316-2318)
  if (a.pec_faces) {
    const int pf = a.pec_faces;
    const bool xf = (i == 0 && (pf & 1)) || (i == a.NX - 1 && (pf & 2));
    const bool yf = (j == 0 && (pf & 4)) || (j == a.NY - 1 && (pf & 8));
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
      const int k = tl.y + lane + 32 * q;
      const bool zf = (k == 0 && (pf & 16)) || (k == a.NZ - 1 && (pf & 32));
      if (yf || zf) v[q][0] = 0.f;
      if (xf || zf) v[q][1] = 0.f;
      if (xf || yf) v[q][2] = 0.f;
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!((comps >> c) & 1u)) continue;
#pragma unroll
    for (int q = 0; q < kQ; ++q)
      if (in[q]) __stcg(a.Eout[c] + row + tl.y + lane + 32 * q, v[q][c]);
  }
}

}  // namespace

int launch_ade_pass(const AdeParams& a, const int* tiles, int n_tiles, cudaStream_t stream) {
  if (n_tiles <= 0) return 0;
  const unsigned blocks = static_cast<unsigned>((n_tiles + 7) / 8);
  ade_pass_kernel<<<blocks, 256, 0, stream>>>(a, reinterpret_cast<const int4*>(tiles), n_tiles);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace fdtdb200
