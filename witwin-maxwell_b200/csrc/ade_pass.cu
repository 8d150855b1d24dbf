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
// (constant cache), so E^n, E^{n+1} and the state of up to four poles are
// loaded together and the pole state streams at HBM speed.
//
// Work list: one warp per tile {row = i * NY + j, k0, k1, pole mask}: lane l
// takes the cell k = k0 + l when k < k1; the mask holds the poles whose box
// covers row (i, j) and meets [k0, k1).  The host builds the tiles from the
// union of the pole boxes per row, 32 cells each.
#include "step_device.cuh"

namespace fdtdb200 {

namespace {

constexpr int kAdePoleBatch = 4;  // poles whose state loads are issued together

__global__ void __launch_bounds__(256) ade_pass_kernel(const __grid_constant__ AdeParams a,
                                                       const int4* __restrict__ tiles, int n_tiles) {
  const int t = static_cast<int>(blockIdx.x) * (blockDim.x >> 5) + static_cast<int>(threadIdx.x >> 5);
  if (t >= n_tiles) return;
  const int4 tl = __ldg(tiles + t);
  const int k = tl.y + static_cast<int>(threadIdx.x & 31);
  if (k >= tl.z) return;
  const int i = tl.x / a.NY;
  const int j = tl.x - i * a.NY;
  const int64_t x = static_cast<int64_t>(tl.x) * a.P + k;
  const unsigned mask = static_cast<unsigned>(tl.w);
  // poles covering this lane's cell, and the components they touch
  unsigned cov = 0, comps = 0;
  for (unsigned m = mask; m; m &= m - 1) {
    const int b = __ffs(m) - 1;
    if (k >= a.poles[b].k0 && k < a.poles[b].k1) {
      cov |= 1u << b;
      comps |= 1u << a.poles[b].comp;
    }
  }
  float eo[3], v[3];
  for (int c = 0; c < 3; ++c) {
    eo[c] = ((comps >> c) & 1u) ? __ldg(a.Ein[c] + x) : 0.f;
    v[c] = ((comps >> c) & 1u) ? a.Eout[c][x] : 0.f;
  }
  for (unsigned m = cov; m;) {
    int ids[kAdePoleBatch];
    int64_t offs[kAdePoleBatch];
    float drive[kAdePoleBatch], ie[kAdePoleBatch], pol[kAdePoleBatch], cur[kAdePoleBatch];
#pragma unroll
    for (int u = 0; u < kAdePoleBatch; ++u) {
      ids[u] = -1;
      offs[u] = 0;
      drive[u] = ie[u] = pol[u] = cur[u] = 0.f;
      if (m) {
        const int b = __ffs(m) - 1;
        m &= m - 1;
        const AdePole& pt = a.poles[b];
        const int64_t o = (static_cast<int64_t>(i - pt.i0) * pt.nj + (j - pt.j0)) * pt.nkk + (k - pt.kk0);
        ids[u] = b;
        offs[u] = o;
        drive[u] = __ldg(pt.drive + o);
        ie[u] = __ldg(pt.inv_eps + o);
        if (pt.kind != 1) pol[u] = pt.pol[o];
        if (pt.kind != 0) cur[u] = pt.cur[o];
      }
    }
#pragma unroll
    for (int u = 0; u < kAdePoleBatch; ++u) {
      if (ids[u] < 0) continue;
      const AdePole& pt = a.poles[ids[u]];
      const int64_t o = offs[u];
      const int c = pt.comp;
      const float ec = c == 0 ? eo[0] : (c == 1 ? eo[1] : eo[2]);
      float jn;
      if (pt.kind == 0) {
        const float prev = pol[u];
        const float next = pt.decay * prev + drive[u] * ec;
        pt.pol[o] = next;
        jn = (next - prev) * pt.inv_dt;
        pt.cur[o] = jn;
      } else if (pt.kind == 1) {
        jn = pt.decay * cur[u] + drive[u] * ec;
        pt.cur[o] = jn;
      } else {
        const float pl = pol[u];
        jn = pt.decay * cur[u] - pt.restoring * pl + drive[u] * ec;
        pt.cur[o] = jn;
        pt.pol[o] = pl + pt.dt * jn;
      }
      const float s = pt.dt * jn * ie[u];
      if (c == 0) v[0] -= s;
      else if (c == 1) v[1] -= s;
      else v[2] -= s;
    }
  }
  for (int c = 0; c < 3; ++c)
    if ((comps >> c) & 1u) __stcg(a.Eout[c] + x, v[c]);
}

}  // namespace

int launch_ade_pass(const AdeParams& a, const int* tiles, int n_tiles, cudaStream_t stream) {
  if (n_tiles <= 0) return 0;
  const unsigned blocks = static_cast<unsigned>((n_tiles + 7) / 8);
  ade_pass_kernel<<<blocks, 256, 0, stream>>>(a, reinterpret_cast<const int4*>(tiles), n_tiles);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace fdtdb200
