// Reverse-time adjoint of the fused leapfrog step: the exact discrete
// transpose of one step (H update with CPML, E update with CPML and edge
// modes), plus monitor seeds and the permittivity gradient of design boxes.
//
// One forward step maps x_n = (E^n, H^{n-1/2}, psi) to x_{n+1}:
//   H' = dh H - ch (a_eff - b_eff),   a/b = forward differences of E
//   E' = de E + ce (a_eff - b_eff),   a/b = backward differences of H'
//   d_eff = ik d + psi',  psi' = b psi + c d          (CPML slab cells)
// The reverse step maps the adjoint g_{n+1} = dL/dx_{n+1} to g_n in three
// passes, as the reference's reverse kernels do
// (witwin/maxwell/fdtd/cuda/kernels/adjoint.cu:295-411, 1224-1690):
//   A (H cells): gH_mid = gH + C_H^T g(d_E)       g(d_E) from u = ce gE'
//   B (E cells): gE = de gE' - C_E^T g(d_H)        g(d_H) from v = ch gH_mid;
//                adjoint E psi updated; dL/deps accumulated in design boxes
//   C (H cells): adjoint H psi updated; gH = dh gH_mid
// with, for a slab term of effective adjoint g_eff and old adjoint psi gq:
//   g(d) = ik g_eff + c (gq + g_eff),   gq <- b (gq + g_eff).
// dL/deps of an E cell (ce = dt/eps, de = 1): the update E' = de E + ce curl
// + S - A, where every E-phase source coefficient carries the same dt/eps
// (point dipole current patches -dt/eps J, injection.py:214-396; TFSF and soft
// surface terms, the curl coefficient times an inverse spacing) and so does
// the ADE correction A (dt J' / eps, or (P' - P) / eps for Debye), so
//   dE'/deps = -(ce curl + S - A) / eps = -(E^{n+1} - de E^n) ce / dt,
// evaluated from the replayed E history of the box.  Sources are affine in the
// fields: they add nothing to the adjoint recursion itself.
#include <cuda_runtime.h>

#include "../../include/fdtd_b200.h"
#include "adjoint.cuh"
#include "step_device.cuh"

namespace fdtdb200 {

namespace {

__device__ __forceinline__ float coef(const float* arr, float uni, int64_t x) { return arr ? __ldg(arr + x) : uni; }

// E edge mode of component c at (i, j, k) (electric.cu:242-268, as the forward kernel).
__device__ __forceinline__ int e_mode(const StepParams& p, int c, int i, int j, int k) {
  const int NX = p.NX, NY = p.NY, NZ = p.NZ;
  if (i < 0 || j < 0 || k < 0) return 3;
  const bool xlo = i == 0, xhi = i == NX - 1, ylo = j == 0, yhi = j == NY - 1, zlo = k == 0, zhi = k == NZ - 1;
  if (c == 0)
    return edge_mode(i < NX - 1 && j < NY && k < NZ, ylo, yhi, zlo, zhi, p.bnd[2], p.bnd[3], p.bnd[4], p.bnd[5]);
  if (c == 1)
    return edge_mode(i < NX && j < NY - 1 && k < NZ, xlo, xhi, zlo, zhi, p.bnd[0], p.bnd[1], p.bnd[4], p.bnd[5]);
  return edge_mode(i < NX && j < NY && k < NZ - 1, xlo, xhi, ylo, yhi, p.bnd[0], p.bnd[1], p.bnd[2], p.bnd[3]);
}

__device__ __forceinline__ bool h_in_extent(const StepParams& p, int c, int i, int j, int k) {
  if (i < 0 || j < 0 || k < 0) return false;
  if (c == 0) return i < p.NX && j < p.NY - 1 && k < p.NZ - 1;
  if (c == 1) return i < p.NX - 1 && j < p.NY && k < p.NZ - 1;
  return i < p.NX - 1 && j < p.NY - 1 && k < p.NZ;
}

__device__ __forceinline__ int64_t cell(const StepParams& p, int i, int j, int k) {
  return (static_cast<int64_t>(i) * p.NY + j) * p.P + k;
}

// Slab offset of the psi element of axis `axis` at (i, j, k) with slab coordinate s.
__device__ __forceinline__ int slab_off(const StepParams& p, int axis, int s, int i, int j, int k) {
  return axis == 0 ? xslab_off(p, s, j, k) : (axis == 1 ? yslab_off(p, i, s, k) : zslab_off(p, i, j, k));
}

__device__ __forceinline__ int coord(int axis, int i, int j, int k) { return axis == 0 ? i : (axis == 1 ? j : k); }

// Adjoint of the raw derivative term `which` (0: a, 1: b) of E component c at
// (i, j, k), reading the adjoint psi (not updating it).  The effective adjoint
// is +u for the term entering the curl with a plus sign, -u otherwise.
__device__ float e_term_adjoint(const StepParams& p, const AdjParams& q, int c, int which, int i, int j, int k) {
  if (e_mode(p, c, i, j, k) != 0) return 0.0f;  // also every cell outside the component's extent
  const int64_t x = cell(p, i, j, k);
  const float u = coef(p.ecurl[c], p.ecurl_u[c], x) * q.gE[c][x];
  // Ex: +a -b;  Ey: -a +b;  Ez: +a -b
  const float g_eff = ((c == 1) ? (which == 0 ? -u : u) : (which == 0 ? u : -u));
  if (!p.cpml) return g_eff;
  const int axis = which == 0 ? (c == 0 ? 1 : 0) : (c == 2 ? 1 : 2);
  const int extent = axis == 0 ? p.NX : (axis == 1 ? p.NY : p.NZ);
  const int s = slab_coord(p, axis, coord(axis, i, j, k), extent);
  if (s < 0) return g_eff;
  const int idx = coord(axis, i, j, k);
  const float cc = __ldg(p.ec[axis] + idx), ik = __ldg(p.eik[axis] + idx);
  const float gq = q.gpsiE[c][which][slab_off(p, axis, s, i, j, k)];
  return ik * g_eff + cc * (gq + g_eff);
}

// Adjoint of the raw forward-difference term `which` of H component c at (i, j, k).
// Hx: -a +b;  Hy: +a -b;  Hz: -a +b  (H' = dh H - ch (a - b) for Hx, Hz; ch (b - a) for Hy).
__device__ float h_term_adjoint(const StepParams& p, const AdjParams& q, int c, int which, int i, int j, int k) {
  if (!h_in_extent(p, c, i, j, k)) return 0.0f;
  const int64_t x = cell(p, i, j, k);
  const float v = coef(p.hcurl[c], p.hcurl_u[c], x) * q.gH[c][x];
  const float g_eff = (c == 1) ? (which == 0 ? v : -v) : (which == 0 ? -v : v);
  if (!p.cpml) return g_eff;
  const int axis = which == 0 ? (c == 0 ? 1 : 0) : (c == 2 ? 1 : 2);
  const int extent = axis == 0 ? p.NX - 1 : (axis == 1 ? p.NY - 1 : p.NZ - 1);
  const int s = slab_coord(p, axis, coord(axis, i, j, k), extent);
  if (s < 0) return g_eff;
  const int idx = coord(axis, i, j, k);
  const float cc = __ldg(p.hc[axis] + idx), ik = __ldg(p.hik[axis] + idx);
  const float gq = q.gpsiH[c][which][slab_off(p, axis, s, i, j, k)];
  return ik * g_eff + cc * (gq + g_eff);
}

// Inverse spacing of index idx (zero outside [0, n)); on a uniform grid the
// axis value u, without a load.
template <bool kUniform>
__device__ __forceinline__ float inv_at(const float* arr, int idx, int n, float u) {
  if (kUniform) return (idx >= 0 && idx < n) ? u : 0.0f;
  return (idx >= 0 && idx < n) ? __ldg(arr + idx) : 0.0f;
}

// True when every coordinate of (i, j, k) lies in [lo_a + a0, N_a - hi_a - a1]
// with lo_a, hi_a the CPML slab lengths raised to at least `floor_` (the edge
// planes are then excluded as well).  Pass A takes a0 = 0, a1 = 2 with floor 1:
// every E neighbour an H cell reads (coordinates c and c + 1) is then an
// interior, non-slab E cell of edge mode 0, so each transposed term is +-ce gE.
// Pass B takes a0 = 1, a1 = 2 with floor 0: the H neighbours (c - 1 and c) are
// in their extent and outside the slabs, and the E cell itself has edge mode 0
// and no psi.
__device__ __forceinline__ bool plain_cell(const StepParams& p, int i, int j, int k, int floor_, int a0, int a1) {
  const int c[3] = {i, j, k};
  const int n[3] = {p.NX, p.NY, p.NZ};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int lo = max(p.cpml ? p.slab_lo[a] : 0, floor_), hi = max(p.cpml ? p.slab_hi[a] : 0, floor_);
    if (c[a] < lo + a0 || c[a] > n[a] - hi - a1) return false;
  }
  return true;
}

// ---- pass A: gH_mid = gH + C_H^T g(d_E) (in place in q.gH) ----
template <bool kUniform>
__global__ void adj_pass_a_kernel(const StepParams p, const AdjParams q) {
  {
    // one thread per cell: k from the x-dimension, rows and planes from y and z
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if (k >= p.P) return;
    const int64_t x = (static_cast<int64_t>(i) * p.NY + j) * p.P + k;
    const float* iex = p.inv_e[0];
    const float* iey = p.inv_e[1];
    const float* iez = p.inv_e[2];
    if (plain_cell(p, i, j, k, 1, 0, 2)) {
      // the same sums as below with every term +-u, u = ce gE of the neighbour
      const int64_t sy = p.P, sx = static_cast<int64_t>(p.NY) * p.P;
      const float uxk = coef(p.ecurl[0], p.ecurl_u[0], x) * q.gE[0][x];
      const float uxk1 = coef(p.ecurl[0], p.ecurl_u[0], x + 1) * q.gE[0][x + 1];
      const float uxj1 = coef(p.ecurl[0], p.ecurl_u[0], x + sy) * q.gE[0][x + sy];
      const float uyk = coef(p.ecurl[1], p.ecurl_u[1], x) * q.gE[1][x];
      const float uyk1 = coef(p.ecurl[1], p.ecurl_u[1], x + 1) * q.gE[1][x + 1];
      const float uyi1 = coef(p.ecurl[1], p.ecurl_u[1], x + sx) * q.gE[1][x + sx];
      const float uzj1 = coef(p.ecurl[2], p.ecurl_u[2], x + sy) * q.gE[2][x + sy];
      const float uzi1 = coef(p.ecurl[2], p.ecurl_u[2], x + sx) * q.gE[2][x + sx];
      const float uz = coef(p.ecurl[2], p.ecurl_u[2], x) * q.gE[2][x];
      const float ez0 = inv_at<kUniform>(iez, k, p.NZ, p.inv_e_u[2]), ez1 = inv_at<kUniform>(iez, k + 1, p.NZ, p.inv_e_u[2]);
      const float ey0 = inv_at<kUniform>(iey, j, p.NY, p.inv_e_u[1]), ey1 = inv_at<kUniform>(iey, j + 1, p.NY, p.inv_e_u[1]);
      const float ex0 = inv_at<kUniform>(iex, i, p.NX, p.inv_e_u[0]), ex1 = inv_at<kUniform>(iex, i + 1, p.NX, p.inv_e_u[0]);
      float g = q.gH[0][x];
      g += ez0 * uyk - ez1 * uyk1;
      g += ey0 * -uz - ey1 * -uzj1;
      q.gH[0][x] = g;
      g = q.gH[1][x];
      g += ez0 * -uxk - ez1 * -uxk1;
      g += ex0 * uz - ex1 * uzi1;
      q.gH[1][x] = g;
      g = q.gH[2][x];
      g += ey0 * uxk - ey1 * uxj1;
      g += ex0 * -uyk - ex1 * -uyi1;
      q.gH[2][x] = g;
      return;
    }
    if (h_in_extent(p, 0, i, j, k)) {  // Hx: Ey d1b (z), Ez d2b (y)
      float g = q.gH[0][x];
      g += inv_at<kUniform>(iez, k, p.NZ, p.inv_e_u[2]) * e_term_adjoint(p, q, 1, 1, i, j, k) -
           inv_at<kUniform>(iez, k + 1, p.NZ, p.inv_e_u[2]) * e_term_adjoint(p, q, 1, 1, i, j, k + 1);
      g += inv_at<kUniform>(iey, j, p.NY, p.inv_e_u[1]) * e_term_adjoint(p, q, 2, 1, i, j, k) -
           inv_at<kUniform>(iey, j + 1, p.NY, p.inv_e_u[1]) * e_term_adjoint(p, q, 2, 1, i, j + 1, k);
      q.gH[0][x] = g;
    }
    if (h_in_extent(p, 1, i, j, k)) {  // Hy: Ex d0b (z), Ez d2a (x)
      float g = q.gH[1][x];
      g += inv_at<kUniform>(iez, k, p.NZ, p.inv_e_u[2]) * e_term_adjoint(p, q, 0, 1, i, j, k) -
           inv_at<kUniform>(iez, k + 1, p.NZ, p.inv_e_u[2]) * e_term_adjoint(p, q, 0, 1, i, j, k + 1);
      g += inv_at<kUniform>(iex, i, p.NX, p.inv_e_u[0]) * e_term_adjoint(p, q, 2, 0, i, j, k) -
           inv_at<kUniform>(iex, i + 1, p.NX, p.inv_e_u[0]) * e_term_adjoint(p, q, 2, 0, i + 1, j, k);
      q.gH[1][x] = g;
    }
    if (h_in_extent(p, 2, i, j, k)) {  // Hz: Ex d0a (y), Ey d1a (x)
      float g = q.gH[2][x];
      g += inv_at<kUniform>(iey, j, p.NY, p.inv_e_u[1]) * e_term_adjoint(p, q, 0, 0, i, j, k) -
           inv_at<kUniform>(iey, j + 1, p.NY, p.inv_e_u[1]) * e_term_adjoint(p, q, 0, 0, i, j + 1, k);
      g += inv_at<kUniform>(iex, i, p.NX, p.inv_e_u[0]) * e_term_adjoint(p, q, 1, 0, i, j, k) -
           inv_at<kUniform>(iex, i + 1, p.NX, p.inv_e_u[0]) * e_term_adjoint(p, q, 1, 0, i + 1, j, k);
      q.gH[2][x] = g;
    }
  }
}

// ---- pass B: gE = de gE' - C_E^T g(d_H); adjoint E psi; design gradient ----
// kPoles: the scene has ADE poles (their transpose is compiled only then: in
// the per-component loop it slows the pole-free kernel by a third).  The
// pole-free kernel runs twelve 128-thread CTAs per SM (40 registers, no
// spills): the pass is latency-bound, and 48 resident warps against 32 at 64
// registers took the backward of the 160x160x96 design workload from 910 to
// 782 ms.  The pole kernel spills at that budget and runs five CTAs per SM
// (at most 102 registers, 70-72 used).
template <bool kUniform, bool kPoles>
__global__ void __launch_bounds__(128, kPoles ? 5 : 12) adj_pass_b_kernel(const StepParams p, const AdjParams q) {
  {
    // one thread per cell: k from the x-dimension, rows and planes from y and z
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if (k >= p.P) return;
    const int64_t x = (static_cast<int64_t>(i) * p.NY + j) * p.P + k;
    const float* ihx = p.inv_h[0];
    const float* ihy = p.inv_h[1];
    const float* ihz = p.inv_h[2];
    // interior cells: the same sums with every term +-v, v = ch gH of the neighbour
    const bool plain = plain_cell(p, i, j, k, 0, 1, 2);
    float vx0 = 0.f, vxk = 0.f, vxj = 0.f, vy0 = 0.f, vyk = 0.f, vyi = 0.f, vz0 = 0.f, vzj = 0.f, vzi = 0.f;
    float hz0 = 0.f, hz1 = 0.f, hy0 = 0.f, hy1 = 0.f, hx0 = 0.f, hx1 = 0.f;
    if (plain) {
      const int64_t sy = p.P, sx = static_cast<int64_t>(p.NY) * p.P;
      vx0 = coef(p.hcurl[0], p.hcurl_u[0], x) * q.gH[0][x];
      vxk = coef(p.hcurl[0], p.hcurl_u[0], x - 1) * q.gH[0][x - 1];
      vxj = coef(p.hcurl[0], p.hcurl_u[0], x - sy) * q.gH[0][x - sy];
      vy0 = coef(p.hcurl[1], p.hcurl_u[1], x) * q.gH[1][x];
      vyk = coef(p.hcurl[1], p.hcurl_u[1], x - 1) * q.gH[1][x - 1];
      vyi = coef(p.hcurl[1], p.hcurl_u[1], x - sx) * q.gH[1][x - sx];
      vz0 = coef(p.hcurl[2], p.hcurl_u[2], x) * q.gH[2][x];
      vzj = coef(p.hcurl[2], p.hcurl_u[2], x - sy) * q.gH[2][x - sy];
      vzi = coef(p.hcurl[2], p.hcurl_u[2], x - sx) * q.gH[2][x - sx];
      hz0 = inv_at<kUniform>(ihz, k, p.NZ - 1, p.inv_h_u[2]);
      hz1 = inv_at<kUniform>(ihz, k - 1, p.NZ - 1, p.inv_h_u[2]);
      hy0 = inv_at<kUniform>(ihy, j, p.NY - 1, p.inv_h_u[1]);
      hy1 = inv_at<kUniform>(ihy, j - 1, p.NY - 1, p.inv_h_u[1]);
      hx0 = inv_at<kUniform>(ihx, i, p.NX - 1, p.inv_h_u[0]);
      hx1 = inv_at<kUniform>(ihx, i - 1, p.NX - 1, p.inv_h_u[0]);
    }
    for (int c = 0; c < 3; ++c) {
      const int m = plain ? 0 : e_mode(p, c, i, j, k);
      if (m == 3 || k >= p.NZ) continue;
      const float gp = q.gE[c][x];
      float g = m == 0 ? coef(p.edecay[c], p.edecay_u[c], x) * gp : (m == 1 ? gp : 0.0f);
      // H-update terms reading this E cell (forward differences of E)
      if (plain) {
        if (c == 0) {
          g += -hz0 * -vy0 + hz1 * -vyk;
          g += -hy0 * vz0 + hy1 * vzj;
        } else if (c == 1) {
          g += -hz0 * vx0 + hz1 * vxk;
          g += -hx0 * -vz0 + hx1 * -vzi;
        } else {
          g += -hy0 * -vx0 + hy1 * -vxj;
          g += -hx0 * vy0 + hx1 * vyi;
        }
      } else if (c == 0) {  // Hy cyb (z), Hz czb (y)
        g += -inv_at<kUniform>(ihz, k, p.NZ - 1, p.inv_h_u[2]) * h_term_adjoint(p, q, 1, 1, i, j, k) +
             inv_at<kUniform>(ihz, k - 1, p.NZ - 1, p.inv_h_u[2]) * h_term_adjoint(p, q, 1, 1, i, j, k - 1);
        g += -inv_at<kUniform>(ihy, j, p.NY - 1, p.inv_h_u[1]) * h_term_adjoint(p, q, 2, 1, i, j, k) +
             inv_at<kUniform>(ihy, j - 1, p.NY - 1, p.inv_h_u[1]) * h_term_adjoint(p, q, 2, 1, i, j - 1, k);
      } else if (c == 1) {  // Hx cxb (z), Hz cza (x)
        g += -inv_at<kUniform>(ihz, k, p.NZ - 1, p.inv_h_u[2]) * h_term_adjoint(p, q, 0, 1, i, j, k) +
             inv_at<kUniform>(ihz, k - 1, p.NZ - 1, p.inv_h_u[2]) * h_term_adjoint(p, q, 0, 1, i, j, k - 1);
        g += -inv_at<kUniform>(ihx, i, p.NX - 1, p.inv_h_u[0]) * h_term_adjoint(p, q, 2, 0, i, j, k) +
             inv_at<kUniform>(ihx, i - 1, p.NX - 1, p.inv_h_u[0]) * h_term_adjoint(p, q, 2, 0, i - 1, j, k);
      } else {  // Hx cxa (y), Hy cya (x)
        g += -inv_at<kUniform>(ihy, j, p.NY - 1, p.inv_h_u[1]) * h_term_adjoint(p, q, 0, 0, i, j, k) +
             inv_at<kUniform>(ihy, j - 1, p.NY - 1, p.inv_h_u[1]) * h_term_adjoint(p, q, 0, 0, i, j - 1, k);
        g += -inv_at<kUniform>(ihx, i, p.NX - 1, p.inv_h_u[0]) * h_term_adjoint(p, q, 1, 0, i, j, k) +
             inv_at<kUniform>(ihx, i - 1, p.NX - 1, p.inv_h_u[0]) * h_term_adjoint(p, q, 1, 0, i - 1, j, k);
      }
      if (m == 0) {
        const float ce = coef(p.ecurl[c], p.ecurl_u[c], x);
        const float u = ce * gp;
        if (p.cpml && !plain) {
          for (int w = 0; w < 2; ++w) {
            const int axis = w == 0 ? (c == 0 ? 1 : 0) : (c == 2 ? 1 : 2);
            const int extent = axis == 0 ? p.NX : (axis == 1 ? p.NY : p.NZ);
            const int s = slab_coord(p, axis, coord(axis, i, j, k), extent);
            if (s < 0) continue;
            const float g_eff = (c == 1) ? (w == 0 ? -u : u) : (w == 0 ? u : -u);
            const float b = __ldg(p.eb[axis] + coord(axis, i, j, k));
            float* gq = q.gpsiE[c][w] + slab_off(p, axis, s, i, j, k);
            *gq = b * (*gq + g_eff);
          }
        }
        const DesignBox& d = q.design[c];
        if (d.grad && i >= d.lo[0] && i < d.hi[0] && j >= d.lo[1] && j < d.hi[1] && k >= d.lo[2] && k < d.hi[2]) {
          const int64_t l = (static_cast<int64_t>(i - d.lo[0]) * (d.hi[1] - d.lo[1]) + (j - d.lo[1])) *
                                (d.hi[2] - d.lo[2]) + (k - d.lo[2]);
          const float e_next = d.hist[static_cast<int64_t>(q.hist_slot + 1) * d.cells + l];
          const float e_now = d.hist[static_cast<int64_t>(q.hist_slot) * d.cells + l];
          const float de = coef(p.edecay[c], p.edecay_u[c], x);
          d.grad[l] += -gp * (e_next - de * e_now) * ce * q.inv_dt;
        }
      }
      // ADE poles of this component at this cell (every E mode: the forward
      // subtracts dt J' / eps after the edge treatment, dispersive.cu:18-83).
      // With u = gE' the adjoint of E^{n+1} and the pole's carried adjoint
      // state of step n + 1:
      //   Drude:   J' = a J + b E;             E' -= dt inv J'
      //   Lorentz: J' = a J - r P + b E; P' = P + dt J';  E' -= dt inv J'
      //   Debye:   P' = a P + b E;             E' -= inv (P' - P)
      if (kPoles && (__ldg(p.plane_bits + i) & kPlanePoles)) {
        // a PEC cell that the forward zeroes after the ADE correction
        // (pec_clamp) passes no adjoint to the pole currents
        const float gpc = (m == 2 && p.pec_clamp) ? 0.0f : gp;
        const int pb = __ldg(p.pole_plane_ptr + i), pe = __ldg(p.pole_plane_ptr + i + 1);
        for (int xx = pb; xx < pe; ++xx) {
          const int id = __ldg(p.pole_plane_ids + xx);
          const PoleTerm& pt = p.poles[id];
          if (pt.comp != c || j < pt.j0 || j >= pt.j1 || k < pt.k0 || k >= pt.k1) continue;
          const int64_t o = (static_cast<int64_t>(i - pt.i0) * (pt.j1 - pt.j0) + (j - pt.j0)) * pt.nkk + (k - pt.kk0);
          const float inv = __ldg(pt.inv_eps + o), b = __ldg(pt.drive + o);
          if (pt.kind == 1) {
            float* gj = q.gcur[id] + o;
            const float ge = *gj - pt.dt * inv * gpc;
            g += b * ge;
            *gj = pt.decay * ge;
          } else if (pt.kind == 2) {
            float* gj = q.gcur[id] + o;
            float* gq = q.gpol[id] + o;
            const float ge = *gj + pt.dt * *gq - pt.dt * inv * gpc;
            g += b * ge;
            *gj = pt.decay * ge;
            *gq = *gq - pt.restoring * ge;
          } else {
            float* gq = q.gpol[id] + o;
            const float ge = *gq - inv * gpc;
            g += b * ge;
            *gq = pt.decay * ge + inv * gpc;
          }
        }
      }
      q.gE[c][x] = g;
    }
  }
}

// ---- pass C: adjoint H psi; gH = dh gH_mid ----
__global__ void adj_pass_c_kernel(const StepParams p, const AdjParams q) {
  {
    // one thread per cell: k from the x-dimension, rows and planes from y and z
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if (k >= p.P) return;
    const int64_t x = (static_cast<int64_t>(i) * p.NY + j) * p.P + k;
    // cells outside every slab have nothing to do when no H component decays
    bool unit = true;
    for (int c = 0; c < 3; ++c) unit = unit && !p.hdecay[c] && p.hdecay_u[c] == 1.0f;
    if (unit && plain_cell(p, i, j, k, 0, 0, 2)) return;
    for (int c = 0; c < 3; ++c) {
      if (!h_in_extent(p, c, i, j, k)) continue;
      // With unit magnetic decay (no magnetic loss) gH = gH_mid already: only
      // CPML slab cells have work (their adjoint psi).
      if (!p.hdecay[c] && p.hdecay_u[c] == 1.0f) {
        bool slab = false;
        if (p.cpml) {
          for (int w = 0; w < 2; ++w) {
            const int axis = w == 0 ? (c == 0 ? 1 : 0) : (c == 2 ? 1 : 2);
            const int extent = axis == 0 ? p.NX - 1 : (axis == 1 ? p.NY - 1 : p.NZ - 1);
            slab = slab || slab_coord(p, axis, coord(axis, i, j, k), extent) >= 0;
          }
        }
        if (!slab) continue;
      }
      const float gm = q.gH[c][x];
      if (p.cpml) {
        const float v = coef(p.hcurl[c], p.hcurl_u[c], x) * gm;
        for (int w = 0; w < 2; ++w) {
          const int axis = w == 0 ? (c == 0 ? 1 : 0) : (c == 2 ? 1 : 2);
          const int extent = axis == 0 ? p.NX - 1 : (axis == 1 ? p.NY - 1 : p.NZ - 1);
          const int s = slab_coord(p, axis, coord(axis, i, j, k), extent);
          if (s < 0) continue;
          const float g_eff = (c == 1) ? (w == 0 ? v : -v) : (w == 0 ? -v : v);
          const float b = __ldg(p.hb[axis] + coord(axis, i, j, k));
          float* gq = q.gpsiH[c][w] + slab_off(p, axis, s, i, j, k);
          *gq = b * (*gq + g_eff);
        }
      }
      q.gH[c][x] = coef(p.hdecay[c], p.hdecay_u[c], x) * gm;
    }
  }
}

// Monitor seeds of step n: the adjoint of the sampled value of every slot,
// sum_f (g_re[f][slot] w_re[n][f] + g_im[f][slot] w_im[n][f]), added to the
// adjoint field at the slot's cell (E^{n+1} with w_e, H^{n+1/2} with w_h).
__global__ void adj_seed_kernel(const StepParams p, const AdjParams q, const RegionFlush* regions, int n_regions,
                                const float2* w_e, const float2* w_h, int n_freq, int n) {
  const int r = blockIdx.y;
  if (r >= n_regions) return;
  const RegionFlush rf = regions[r];
  const float2* w = (rf.is_h ? w_h : w_e) + static_cast<int64_t>(n) * n_freq;
  float* field = rf.is_h ? q.gH[rf.comp - 3] : q.gE[rf.comp];
  for (int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; s < rf.count;
       s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t slot = rf.base + s;
    float acc = 0.0f;
    for (int f = 0; f < n_freq; ++f) {
      const float2 wf = w[f];
      const int64_t o = static_cast<int64_t>(f) * q.n_samples + slot;
      acc += q.seed_re[o] * wf.x + q.seed_im[o] * wf.y;
    }
    const int lk = static_cast<int>(s % rf.nk);
    const int lj = static_cast<int>((s / rf.nk) % rf.nj);
    const int li = static_cast<int>(s / (static_cast<int64_t>(rf.nk) * rf.nj));
    field[cell(p, rf.i0 + li, rf.j0 + lj, rf.k0 + lk)] += acc;
  }
}

// Copy the current E of every design box into history slot `slot`.  Index
// arithmetic in 32 bits: a design box holds fewer than 2^31 cells (the host
// rejects larger ones).
__global__ void design_record_kernel(const StepParams p, const AdjParams q, int slot) {
  const int c = blockIdx.y;
  const DesignBox& d = q.design[c];
  if (!d.grad) return;
  const float* e = p.Ein[c];
  const int nj = d.hi[1] - d.lo[1], nk = d.hi[2] - d.lo[2];
  const int cells = static_cast<int>(d.cells);
  float* hist = d.hist + static_cast<int64_t>(slot) * d.cells;
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < cells; l += gridDim.x * blockDim.x) {
    const int r = l / nk;
    const int k = d.lo[2] + (l - r * nk);
    const int i = d.lo[0] + r / nj;
    const int j = d.lo[1] + (r - (r / nj) * nj);
    hist[l] = e[cell(p, i, j, k)];
  }
}

unsigned grid_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return static_cast<unsigned>(b);
}

}  // namespace

int launch_adjoint_step(const StepParams& p, const AdjParams& q, const RegionFlush* regions, int n_regions,
                        const float2* w_e, const float2* w_h, int n_freq, int n, cudaStream_t stream) {
  if (n_regions > 0 && q.seed_re) {
    dim3 grid(64, n_regions);
    adj_seed_kernel<<<grid, 256, 0, stream>>>(p, q, regions, n_regions, w_e, w_h, n_freq, n);
  }
  const dim3 cells((p.P + 127) / 128, p.NY, p.NX);
  const bool poles = p.n_poles > 0;
  if (p.uniform_grid) {
    adj_pass_a_kernel<true><<<cells, 128, 0, stream>>>(p, q);
    if (poles) adj_pass_b_kernel<true, true><<<cells, 128, 0, stream>>>(p, q);
    else adj_pass_b_kernel<true, false><<<cells, 128, 0, stream>>>(p, q);
  } else {
    adj_pass_a_kernel<false><<<cells, 128, 0, stream>>>(p, q);
    if (poles) adj_pass_b_kernel<false, true><<<cells, 128, 0, stream>>>(p, q);
    else adj_pass_b_kernel<false, false><<<cells, 128, 0, stream>>>(p, q);
  }
  adj_pass_c_kernel<<<cells, 128, 0, stream>>>(p, q);
  return static_cast<int>(cudaGetLastError());
}

int launch_design_record(const StepParams& p, const AdjParams& q, int slot, cudaStream_t stream) {
  int64_t cells = 0;
  for (int c = 0; c < 3; ++c)
    if (q.design[c].grad && q.design[c].cells > cells) cells = q.design[c].cells;
  if (cells == 0) return 0;
  design_record_kernel<<<dim3(grid_for(cells), 3), 256, 0, stream>>>(p, q, slot);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace fdtdb200
