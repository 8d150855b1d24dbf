// Wrap kernel of periodic and Bloch-periodic faces: the E update of the cells
// the fused step kernel defers (edge mode kModeDeferred), run after the step
// kernels of both field channels have written the whole new H.
//
// A backward difference along a wrapped axis at the low face reads the last H
// plane with the phase e^{-ikL}, and at the high face (the image of the low
// face) reads the first H plane with e^{+ikL}
// (witwin/maxwell/fdtd/cuda/kernels/electric.cu:124-168, bloch_backward_diff_axis
// with phase_positive / phase_negative); a periodic face is the same with phase
// 1.  The complex field is carried as two real channels (real and imaginary
// part, each a full engine): the phase couples them only here.  Along an axis
// that does not wrap the difference is the standard one, zero on a NONE or PML
// face (electric.cu:23-40 boundary_diff_low / high, as the reference's
// Bloch-x/y standard-z kernels, electric.cu:1164-1229).  CPML psi of the
// non-wrapped axes, ADE poles and E-phase injection terms of the deferred cells
// are applied as in the step kernel, per channel.
#include "step_device.cuh"

namespace fdtdb200 {

namespace {

struct Cplx {
  float re, im;
};

__device__ __forceinline__ int64_t wcell(const StepParams& p, int i, int j, int k) {
  return (static_cast<int64_t>(i) * p.NY + j) * p.P + k;
}

__device__ __forceinline__ float inv_e_at(const StepParams& p, int axis, int idx) {
  return p.uniform_grid ? p.inv_e_u[axis] : __ldg(p.inv_e[axis] + idx);
}

// Backward difference of H component hc along `axis` for the E cell (i, j, k),
// both channels (im ignored when !cplx); TS: the stored field type, each channel
// read with its own scale (p: real channel, q: imaginary channel).
template <typename TS>
__device__ Cplx bdiff(const StepParams& p, const StepParams& q, const WrapFields& fr, const WrapFields& fi, bool cplx,
                      int hc, int axis, int i, int j, int k, float pc, float ps) {
  const int N = axis == 0 ? p.NX : (axis == 1 ? p.NY : p.NZ);
  const int coord = axis == 0 ? i : (axis == 1 ? j : k);
  const float inv = inv_e_at(p, axis, coord);
  auto at = [&](int c) {
    return axis == 0 ? wcell(p, c, j, k) : (axis == 1 ? wcell(p, i, c, k) : wcell(p, i, j, c));
  };
  const float* hr = fr.hnew[hc];
  const float* hi = cplx ? fi.hnew[hc] : nullptr;
  const float sr = p.fscale[3 + hc], si = q.fscale[3 + hc];
  auto val = [&](int c) { return Cplx{ldf<TS>(hr, at(c), true, sr), hi ? ldf<TS>(hi, at(c), true, si) : 0.0f}; };
  if (wraps(p.bnd[2 * axis])) {
    if (coord == 0) {
      const Cplx lo = val(0), h = val(N - 2);
      // phase_negative: e^{-ikL} times the last plane
      const Cplx sh{pc * h.re + ps * h.im, pc * h.im - ps * h.re};
      return {(lo.re - sh.re) * inv, (lo.im - sh.im) * inv};
    }
    if (coord == N - 1) {
      const Cplx lo = val(0), h = val(N - 2);
      // phase_positive: e^{+ikL} times the first plane
      const Cplx sh{pc * lo.re - ps * lo.im, ps * lo.re + pc * lo.im};
      return {(sh.re - h.re) * inv, (sh.im - h.im) * inv};
    }
  } else if (coord == 0 || coord == N - 1) {
    return {0.0f, 0.0f};
  }
  const Cplx cur = val(coord), prev = val(coord - 1);
  return {(cur.re - prev.re) * inv, (cur.im - prev.im) * inv};
}

// CPML psi of term `which` (0: a-axis, 1: b-axis) of E component c at (i, j, k)
// on the channel's own psi arrays; returns the stretched difference.
__device__ float psi_term(const StepParams& p, int c, int which, int axis, int i, int j, int k, float d) {
  if (!p.cpml) return d;
  const int coord = axis == 0 ? i : (axis == 1 ? j : k);
  const int extent = axis == 0 ? p.NX : (axis == 1 ? p.NY : p.NZ);
  const int s = slab_coord(p, axis, coord, extent);
  if (s < 0) return d;
  const int off = axis == 0 ? xslab_off(p, s, j, k) : (axis == 1 ? yslab_off(p, i, s, k) : zslab_off(p, i, j, k));
  const Prof pr = prof(p.eb[axis], p.ec[axis], p.eik[axis], coord);
  return psi_step(d, pr.b, pr.c, pr.ik, p.psiE[c][which], p.psiE[c][which], off, true);
}

__device__ __forceinline__ float coef_at(const float* arr, float u, int64_t x) { return arr ? __ldg(arr + x) : u; }

// The E update of the deferred components at (i, j, k) for one channel; TS the
// stored field type, TA the ADE pole state type.
template <typename TS, typename TA>
__device__ void wrap_cell_channel(const StepParams& p, const WrapFields& f, const Cplx (&d)[3][2], const int (&m)[3],
                                  int n, int i, int j, int k, bool imag) {
  const int64_t x = wcell(p, i, j, k);
  float v[3] = {0.f, 0.f, 0.f};
  float eo[3];
  for (int c = 0; c < 3; ++c) eo[c] = ldf<TS>(f.eold[c], x, true, p.fscale[c]);
  unsigned mask = 0;
  // component c: its two derivative terms a (which 0) and b (which 1) along
  // Ex: y, z; Ey: x, z; Ez: x, y; Ex = (a - b), Ey = (b - a), Ez = (a - b)
  const int ax[3][2] = {{1, 2}, {0, 2}, {0, 1}};
  for (int c = 0; c < 3; ++c) {
    if (m[c] != kModeDeferred) continue;
    mask |= 1u << c;
    float a = imag ? d[c][0].im : d[c][0].re;
    float b = imag ? d[c][1].im : d[c][1].re;
    a = psi_term(p, c, 0, ax[c][0], i, j, k, a);
    b = psi_term(p, c, 1, ax[c][1], i, j, k, b);
    const float g = coef_at(p.edecay[c], p.edecay_u[c], x);
    const float cc = coef_at(p.ecurl[c], p.ecurl_u[c], x);
    v[c] = eo[c] * g + cc * (c == 1 ? (b - a) : (a - b));
  }
  if (!mask) return;
  if (p.n_poles && (__ldg(p.plane_bits + i) & kPlanePoles)) {
    unsigned lane_poles = 0;
    const int np_ = min(p.n_poles, 32);
    for (int b = 0; b < np_; ++b) {
      const PoleTerm& pt = p.poles[b];
      if (j >= pt.j0 && j < pt.j1 && k >= pt.k0 && k < pt.k1) lane_poles |= 1u << b;
    }
    ade<TA>(p, lane_poles, i, j, k, eo[0], eo[1], eo[2], v[0], v[1], v[2], mask);
  }
  if (p.n_terms[0]) {
    const bool sx = __ldg(p.plane_bits + i) & kPlaneETerms;
    const bool sy = list_nonempty(p.term_index[0], 1, j);
    const bool sz = list_nonempty(p.term_index[0], 2, k);
    if (sx || sy || sz) add_terms(p, 0, 0, n, i, j, k, sx, sy, sz, v[0], v[1], v[2]);
  }
  for (int c = 0; c < 3; ++c)
    if ((mask >> c) & 1u) stf<TS>(f.enew[c], x, v[c], p.finv[c]);
}

// One thread per cell of the wrap faces: the two x faces (whole planes) when x
// wraps, then the two y faces (rows, without the x-face cells already counted).
template <typename TS, typename TA>
__global__ void wrap_fixup_kernel(const StepParams pr, const StepParams pim, const WrapFields fr, const WrapFields fi,
                                  int cplx, float pcx, float psx, float pcy, float psy, int n) {
  const StepParams& p = pr;
  if (p.step_base) n += __ldg(p.step_base);
  const int NX = p.NX, NY = p.NY, NZ = p.NZ;
  const bool xw = wraps(p.bnd[0]), yw = wraps(p.bnd[2]);
  const int64_t nxa = xw ? 2ll * NY * NZ : 0;
  const int ix_lo = xw ? 1 : 0, ix_hi = xw ? NX - 1 : NX;  // rows of the y faces: i in [ix_lo, ix_hi)
  const int64_t nyb = yw ? 2ll * (ix_hi - ix_lo) * NZ : 0;
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= nxa + nyb) return;
  int i, j, k;
  if (t < nxa) {
    const int64_t plane = static_cast<int64_t>(NY) * NZ;
    i = t < plane ? 0 : NX - 1;
    const int64_t r = t % plane;
    j = static_cast<int>(r / NZ);
    k = static_cast<int>(r % NZ);
  } else {
    const int64_t u = t - nxa;
    const int64_t face = static_cast<int64_t>(ix_hi - ix_lo) * NZ;
    j = u < face ? 0 : NY - 1;
    const int64_t r = u % face;
    i = ix_lo + static_cast<int>(r / NZ);
    k = static_cast<int>(r % NZ);
  }
  const bool xlo = i == 0, xhi = i == NX - 1, ylo = j == 0, yhi = j == NY - 1, zlo = k == 0, zhi = k == NZ - 1;
  int m[3];
  m[0] = edge_mode(i < NX - 1 && k < NZ, ylo, yhi, zlo, zhi, p.bnd[2], p.bnd[3], p.bnd[4], p.bnd[5]);
  m[1] = edge_mode(j < NY - 1 && k < NZ, xlo, xhi, zlo, zhi, p.bnd[0], p.bnd[1], p.bnd[4], p.bnd[5]);
  m[2] = edge_mode(k < NZ - 1, xlo, xhi, ylo, yhi, p.bnd[0], p.bnd[1], p.bnd[2], p.bnd[3]);
  if (m[0] != kModeDeferred && m[1] != kModeDeferred && m[2] != kModeDeferred) return;
  const bool cx = cplx != 0;
  const float pc[3] = {pcx, pcy, 1.0f}, ps[3] = {psx, psy, 0.0f};
  // raw differences (both channels): Ex: dHz/dy, dHy/dz; Ey: dHz/dx, dHx/dz; Ez: dHy/dx, dHx/dy
  const int hsrc[3][2] = {{2, 1}, {2, 0}, {1, 0}};
  const int ax[3][2] = {{1, 2}, {0, 2}, {0, 1}};
  Cplx d[3][2];
  for (int c = 0; c < 3; ++c) {
    for (int w = 0; w < 2; ++w) {
      d[c][w] = {0.0f, 0.0f};
      if (m[c] == kModeDeferred) {
        const int a = ax[c][w];
        d[c][w] = bdiff<TS>(p, pim, fr, fi, cx, hsrc[c][w], a, i, j, k, pc[a], ps[a]);
      }
    }
  }
  wrap_cell_channel<TS, TA>(pr, fr, d, m, n, i, j, k, false);
  if (cx) wrap_cell_channel<TS, TA>(pim, fi, d, m, n, i, j, k, true);
}

}  // namespace

// Cells of the wrap faces of a grid (0 when no axis wraps).
int64_t wrap_cell_count(const StepParams& p) {
  const bool xw = wraps(p.bnd[0]), yw = wraps(p.bnd[2]);
  const int64_t nxa = xw ? 2ll * p.NY * p.NZ : 0;
  const int64_t nyb = yw ? 2ll * (xw ? p.NX - 2 : p.NX) * p.NZ : 0;
  return nxa + nyb;
}

int launch_wrap_fixup(const StepParams& pr, const StepParams* pim, const WrapFields& fr, const WrapFields* fi,
                      const float* phase_cos, const float* phase_sin, int n, cudaStream_t stream, int storage) {
  const int64_t cells = wrap_cell_count(pr);
  if (cells == 0) return 0;
  if (storage != kStoreF32 && storage != kStoreBF16) return static_cast<int>(cudaErrorInvalidValue);
  const unsigned blocks = static_cast<unsigned>((cells + 255) / 256);
  const bool cplx = pim != nullptr && fi != nullptr;
  if (storage == kStoreBF16)
    wrap_fixup_kernel<__nv_bfloat16, __nv_bfloat16><<<blocks, 256, 0, stream>>>(
        pr, cplx ? *pim : pr, fr, cplx ? *fi : fr, cplx ? 1 : 0, phase_cos[0], phase_sin[0], phase_cos[1],
        phase_sin[1], n);
  else
    wrap_fixup_kernel<float, float><<<blocks, 256, 0, stream>>>(pr, cplx ? *pim : pr, fr, cplx ? *fi : fr,
                                                                cplx ? 1 : 0, phase_cos[0], phase_sin[0],
                                                                phase_cos[1], phase_sin[1], n);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace fdtdb200
