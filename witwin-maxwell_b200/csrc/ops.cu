// Per-op kernels with the semantics of the reference's torch ops
// (witwin/maxwell/fdtd/cuda/extension.cpp:2059-2196).  They let a caller
// re-point the reference's NativeFDTDModule op by op; the fused engine is the
// fast path.  Each kernel is one thread per output element over a flattened
// index (z fastest), 256-thread blocks, launched on the caller's stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/fdtd_b200.h"
#include "common.cuh"

using namespace fdtdb200;

namespace {

int op_fail(int code, const char* msg) {
  set_last_error(msg);
  return code;
}

int op_launch_check(const char* what) {
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    set_last_error(std::string(what) + ": " + cudaGetErrorString(err));
    return FDTD_ERR_CUDA;
  }
  return 0;
}

constexpr int kThreads = 256;

unsigned blocks_for(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  if (b < 1) b = 1;
  if (b > (1 << 20)) b = 1 << 20;
  return static_cast<unsigned>(b);
}

__device__ __forceinline__ void unflatten(int64_t x, int ny, int nz, int& i, int& j, int& k) {
  k = static_cast<int>(x % nz);
  const int64_t r = x / nz;
  j = static_cast<int>(r % ny);
  i = static_cast<int>(r / ny);
}

struct CpmlArgs {
  float* psi_a;
  float* psi_b;
  const float *ika, *ba, *ca, *ikb, *bb, *cb;
  int a_low, a_hstart, a_hlen, b_low, b_hstart, b_hlen;
};

__device__ __forceinline__ float psi_advance(int mode, float* psi, const float* b, const float* c, int axis, int i,
                                             int j, int k, int ny, int nz, int coord, int low, int hstart,
                                             int hlen, float d) {
  int64_t o;
  if (mode == 1) {
    o = off3(i, j, k, ny, nz);
  } else {
    const int local = slab_local(coord, low, hstart, hlen);
    if (local < 0) return 0.0f;
    const int clen = low + hlen;
    o = axis == 0 ? off3(local, j, k, ny, nz) : (axis == 1 ? off3(i, local, k, clen, nz) : off3(i, j, local, ny, clen));
  }
  const float v = b[coord] * psi[o] + c[coord] * d;
  psi[o] = v;
  return v;
}

// witwin/maxwell/fdtd/cuda/kernels/magnetic.cu:20-212
__global__ void op_magnetic_kernel(int comp, int mode, int nx, int ny, int nz, float* field, const float* first,
                                   const float* second, const float* decay, const float* curl, float decay_u,
                                   float curl_u, const float* inv_a, const float* inv_b, CpmlArgs cp) {
  const int64_t total = static_cast<int64_t>(nx) * ny * nz;
  const int A = comp == 0 ? 1 : 0, B = comp == 2 ? 1 : 2;
  const int sy2 = ny + (A == 1), sz2 = nz + (A == 2);
  const int sy1 = ny + (B == 1), sz1 = nz + (B == 2);
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int i, j, k;
    unflatten(x, ny, nz, i, j, k);
    const int ca_ = A == 0 ? i : (A == 1 ? j : k);
    const int cb_ = B == 0 ? i : (B == 1 ? j : k);
    const float da = (second[off3(i + (A == 0), j + (A == 1), k + (A == 2), sy2, sz2)] - second[off3(i, j, k, sy2, sz2)]) * inv_a[ca_];
    const float db = (first[off3(i + (B == 0), j + (B == 1), k + (B == 2), sy1, sz1)] - first[off3(i, j, k, sy1, sz1)]) * inv_b[cb_];
    float ea = da, eb = db;
    if (mode != 0) {
      const float pa = psi_advance(mode, cp.psi_a, cp.ba, cp.ca, A, i, j, k, ny, nz, ca_, cp.a_low, cp.a_hstart, cp.a_hlen, da);
      const float pb = psi_advance(mode, cp.psi_b, cp.bb, cp.cb, B, i, j, k, ny, nz, cb_, cp.b_low, cp.b_hstart, cp.b_hlen, db);
      ea = da * cp.ika[ca_] + pa;
      eb = db * cp.ikb[cb_] + pb;
    }
    const float c = comp == 1 ? (eb - ea) : (ea - eb);
    const float dv = decay ? decay[x] : decay_u;
    const float cv = curl ? curl[x] : curl_u;
    field[x] = field[x] * dv - cv * c;
  }
}

__device__ __forceinline__ float bdiff(const float* src, int axis, int i, int j, int k, int tsize, int sy, int sz,
                                       int lo, int hi, const float* inv) {
  const int coord = axis == 0 ? i : (axis == 1 ? j : k);
  const float iv = inv[coord];
  if (coord == 0 || coord + 1 == tsize) {
    const int last = tsize - 2;
    const int64_t l = axis == 0 ? off3(0, j, k, sy, sz) : (axis == 1 ? off3(i, 0, k, sy, sz) : off3(i, j, 0, sy, sz));
    const int64_t h = axis == 0 ? off3(last, j, k, sy, sz) : (axis == 1 ? off3(i, last, k, sy, sz) : off3(i, j, last, sy, sz));
    const int mode = coord == 0 ? lo : hi;
    if (mode == BND_PERIODIC) return (src[l] - src[h]) * iv;
    if (mode == BND_PMC) return coord == 0 ? 2.0f * src[l] * iv : -2.0f * src[h] * iv;
    return 0.0f;
  }
  const int64_t cur = off3(i, j, k, sy, sz);
  const int64_t prv = axis == 0 ? off3(i - 1, j, k, sy, sz) : (axis == 1 ? off3(i, j - 1, k, sy, sz) : off3(i, j, k - 1, sy, sz));
  return (src[cur] - src[prv]) * iv;
}

// Bloch-periodic backward difference along `axis` of the complex source
// (re, im) at the target cell (i, j, k), target extent tsize along the axis:
// across the wrap the far face enters with the phase e^{-ikL} at the low end
// and the near face with e^{+ikL} at the high end
// (witwin/maxwell/fdtd/cuda/kernels/electric.cu:120-240, 356-453).
__device__ __forceinline__ void bloch_bdiff(const float* re, const float* im, int axis, int i, int j, int k, int tsize,
                                            int sy, int sz, float pc, float ps, const float* inv, float& dr, float& di) {
  const int coord = axis == 0 ? i : (axis == 1 ? j : k);
  const float iv = inv[coord];
  if (coord == 0 || coord + 1 == tsize) {
    const int last = tsize - 2;
    const int64_t l = axis == 0 ? off3(0, j, k, sy, sz) : (axis == 1 ? off3(i, 0, k, sy, sz) : off3(i, j, 0, sy, sz));
    const int64_t h = axis == 0 ? off3(last, j, k, sy, sz) : (axis == 1 ? off3(i, last, k, sy, sz) : off3(i, j, last, sy, sz));
    if (coord == 0) {
      const float nr = pc * re[h] + ps * im[h], ni = pc * im[h] - ps * re[h];
      dr = (re[l] - nr) * iv;
      di = (im[l] - ni) * iv;
    } else {
      const float pr = pc * re[l] - ps * im[l], pi = ps * re[l] + pc * im[l];
      dr = (pr - re[h]) * iv;
      di = (pi - im[h]) * iv;
    }
    return;
  }
  const int64_t cur = off3(i, j, k, sy, sz);
  const int64_t prv = axis == 0 ? off3(i - 1, j, k, sy, sz) : (axis == 1 ? off3(i, j - 1, k, sy, sz) : off3(i, j, k - 1, sy, sz));
  dr = (re[cur] - re[prv]) * iv;
  di = (im[cur] - im[prv]) * iv;
}

// witwin/maxwell/fdtd/cuda/kernels/electric.cu:18-119, 242-311, 462-941
__global__ void op_electric_kernel(int comp, int mode, int nx, int ny, int nz, float* field, const float* first,
                                   const float* second, const float* decay, const float* curl, float decay_u,
                                   float curl_u, const float* inv_a, const float* inv_b, int a_lo, int a_hi,
                                   int b_lo, int b_hi, CpmlArgs cp) {
  const int64_t total = static_cast<int64_t>(nx) * ny * nz;
  const int A = comp == 0 ? 1 : 0, B = comp == 2 ? 1 : 2;
  const int sy2 = ny - (A == 1), sz2 = nz - (A == 2);
  const int sy1 = ny - (B == 1), sz1 = nz - (B == 2);
  const int size_a = A == 0 ? nx : (A == 1 ? ny : nz);
  const int size_b = B == 0 ? nx : (B == 1 ? ny : nz);
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int i, j, k;
    unflatten(x, ny, nz, i, j, k);
    const int ca_ = A == 0 ? i : (A == 1 ? j : k);
    const int cb_ = B == 0 ? i : (B == 1 ? j : k);
    const bool pec = (ca_ == 0 && a_lo == BND_PEC) || (ca_ + 1 == size_a && a_hi == BND_PEC) ||
                     (cb_ == 0 && b_lo == BND_PEC) || (cb_ + 1 == size_b && b_hi == BND_PEC);
    if (pec) {
      field[x] = 0.0f;
      continue;
    }
    const bool ina = (ca_ == 0 && (a_lo == BND_NONE || a_lo == BND_PML)) ||
                     (ca_ + 1 == size_a && (a_hi == BND_NONE || a_hi == BND_PML));
    const bool inb = (cb_ == 0 && (b_lo == BND_NONE || b_lo == BND_PML)) ||
                     (cb_ + 1 == size_b && (b_hi == BND_NONE || b_hi == BND_PML));
    if (ina || inb) continue;
    const float da = bdiff(second, A, i, j, k, size_a, sy2, sz2, a_lo, a_hi, inv_a);
    const float db = bdiff(first, B, i, j, k, size_b, sy1, sz1, b_lo, b_hi, inv_b);
    float ea = da, eb = db;
    if (mode != 0) {
      const float pa = psi_advance(mode, cp.psi_a, cp.ba, cp.ca, A, i, j, k, ny, nz, ca_, cp.a_low, cp.a_hstart, cp.a_hlen, da);
      const float pb = psi_advance(mode, cp.psi_b, cp.bb, cp.cb, B, i, j, k, ny, nz, cb_, cp.b_low, cp.b_hstart, cp.b_hlen, db);
      ea = da * cp.ika[ca_] + pa;
      eb = db * cp.ikb[cb_] + pb;
    }
    const float c = comp == 1 ? (eb - ea) : (ea - eb);
    const float dv = decay ? decay[x] : decay_u;
    const float cv = curl ? curl[x] : curl_u;
    field[x] = field[x] * dv + cv * c;
  }
}

__global__ void op_debye_kernel(int64_t n, const float* e, const float* drive, float decay, float inv_dt, float* pol,
                                float* cur) {
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < n;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float prev = pol[x];
    const float next = decay * prev + drive[x] * e[x];
    pol[x] = next;
    cur[x] = (next - prev) * inv_dt;
  }
}

__global__ void op_drude_kernel(int64_t n, const float* e, const float* drive, float decay, float* cur) {
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < n;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x)
    cur[x] = decay * cur[x] + drive[x] * e[x];
}

__global__ void op_lorentz_kernel(int64_t n, const float* e, const float* drive, float decay, float restoring,
                                  float dt, float* pol, float* cur) {
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < n;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float pj = cur[x], pp = pol[x];
    const float nj = decay * pj - restoring * pp + drive[x] * e[x];
    cur[x] = nj;
    pol[x] = pp + dt * nj;
  }
}

__global__ void op_apply_pol_kernel(int64_t n, const float* cur, const float* inv_eps, float dt, float* e) {
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < n;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x)
    e[x] -= dt * cur[x] * inv_eps[x];
}

__global__ void op_patch_kernel(float* field, int fx, int fy, int fz, const float* patch, int px, int py, int pz,
                                int oi, int oj, int ok, float signal) {
  const int64_t total = static_cast<int64_t>(px) * py * pz;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int i, j, k;
    unflatten(x, py, pz, i, j, k);
    const int gi = oi + i, gj = oj + j, gk = ok + k;
    if (gi < 0 || gj < 0 || gk < 0 || gi >= fx || gj >= fy || gk >= fz) continue;
    field[off3(gi, gj, gk, fy, fz)] += signal * patch[x];
  }
}

// Complex E update on Bloch faces: E = E decay + curl (d_A second - d_B first)
// (Ey: d_B first - d_A second), both differences Bloch-wrapped, or the B (z)
// difference standard with z boundary modes (z_std: the Bloch-x/y,
// standard-z kernels), electric.cu:356-453, 1164-1528.
__global__ void op_electric_bloch_kernel(int comp, int z_std, int nx, int ny, int nz, float* er, float* ei,
                                         const float* fr, const float* fi, const float* sr, const float* si,
                                         const float* decay, const float* curl, float pca, float psa, float pcb,
                                         float psb, const float* inv_a, const float* inv_b, int z_lo, int z_hi) {
  const int64_t total = static_cast<int64_t>(nx) * ny * nz;
  const int A = comp == 0 ? 1 : 0, B = comp == 2 ? 1 : 2;
  const int sy2 = ny - (A == 1), sz2 = nz - (A == 2);
  const int sy1 = ny - (B == 1), sz1 = nz - (B == 2);
  const int size_a = A == 0 ? nx : (A == 1 ? ny : nz);
  const int size_b = B == 0 ? nx : (B == 1 ? ny : nz);
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int i, j, k;
    unflatten(x, ny, nz, i, j, k);
    float dar, dai, dbr, dbi;
    bloch_bdiff(sr, si, A, i, j, k, size_a, sy2, sz2, pca, psa, inv_a, dar, dai);
    if (z_std) {
      dbr = bdiff(fr, B, i, j, k, size_b, sy1, sz1, z_lo, z_hi, inv_b);
      dbi = bdiff(fi, B, i, j, k, size_b, sy1, sz1, z_lo, z_hi, inv_b);
    } else {
      bloch_bdiff(fr, fi, B, i, j, k, size_b, sy1, sz1, pcb, psb, inv_b, dbr, dbi);
    }
    const float cr = comp == 1 ? (dbr - dar) : (dar - dbr);
    const float ci = comp == 1 ? (dbi - dai) : (dai - dbi);
    er[x] = er[x] * decay[x] + curl[x] * cr;
    ei[x] = ei[x] * decay[x] + curl[x] * ci;
  }
}

// z-CPML correction of Ex (t axis y) or Ey (t axis x) over a region at
// (oi, oj, ok) of the full grid: psi = b psi + c dH/dz, E -/+= curl (dH/dz
// (1 / kappa - 1) + psi), skipped on inactive t faces (NONE, PEC, PML) and on
// the first and last global z planes (electric.cu:1164-1528).
__global__ void op_cpml_z_kernel(int comp, float* field, int sx, int sy, int sz, const float* h, int hy, int hz,
                                 const float* curl, float* psi, const float* ik, const float* b, const float* c,
                                 const float* inv_dz, int oi, int oj, int ok, int lo_mode, int hi_mode, int full_t,
                                 int k0, int k1) {
  const int nk = k1 - k0;
  const int64_t total = static_cast<int64_t>(sx) * sy * nk;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int li, lj, lk;
    unflatten(x, sy, nk, li, lj, lk);
    lk += k0;
    const int gi = oi + li, gj = oj + lj, gk = ok + lk;
    const int t = comp == 0 ? gj : gi;
    const bool lo_off = lo_mode == BND_NONE || lo_mode == BND_PEC || lo_mode == BND_PML;
    const bool hi_off = hi_mode == BND_NONE || hi_mode == BND_PEC || hi_mode == BND_PML;
    if ((lo_off && t == 0) || (hi_off && t + 1 == full_t)) continue;
    const float d = (h[off3(gi, gj, gk, hy, hz)] - h[off3(gi, gj, gk - 1, hy, hz)]) * inv_dz[gk];
    const int64_t o = off3(li, lj, lk, sy, sz);
    const float v = b[gk] * psi[o] + c[gk] * d;
    psi[o] = v;
    // the z difference enters Ex's curl with a minus sign and Ey's with a plus
    const float corr = curl[o] * (d * (ik[gk] - 1.0f) + v);
    field[o] = comp == 0 ? field[o] - corr : field[o] + corr;
  }
}

// Face projection of a periodic (im == nullptr: average of the two faces) or
// Bloch field (the low face least-squares consistent with high = e^{ikL} low,
// then the high face set from it), projection.cu:43-125.
__global__ void op_project_kernel(float* re, float* im, int nx, int ny, int nz, int axis, float pc, float ps) {
  const int da = axis == 0 ? ny : nx, db = axis == 2 ? ny : nz;
  const int64_t total = static_cast<int64_t>(da) * db;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int a = static_cast<int>(x / db), bb = static_cast<int>(x % db);
    int64_t lo, hi;
    if (axis == 0) {
      lo = off3(0, a, bb, ny, nz);
      hi = lo + static_cast<int64_t>(nx - 1) * ny * nz;
    } else if (axis == 1) {
      lo = off3(a, 0, bb, ny, nz);
      hi = lo + static_cast<int64_t>(ny - 1) * nz;
    } else {
      lo = off3(a, bb, 0, ny, nz);
      hi = lo + nz - 1;
    }
    if (!im) {
      const float avg = 0.5f * (re[lo] + re[hi]);
      re[lo] = avg;
      re[hi] = avg;
      continue;
    }
    const float lr = re[lo], li = im[lo], hr = re[hi], hi_i = im[hi];
    const float pr = 0.5f * (lr + pc * hr + ps * hi_i);
    const float pi = 0.5f * (li + pc * hi_i - ps * hr);
    re[lo] = pr;
    im[lo] = pi;
    re[hi] = pc * pr - ps * pi;
    im[hi] = ps * pr + pc * pi;
  }
}

// CW-phased patch: value = signal_cos * patch_cos + signal_sin * patch_sin
// (witwin/maxwell/fdtd/cuda/kernels/sources.cu:156-171).
__global__ void op_cw_patch_kernel(float* field, int fx, int fy, int fz, const float* pc, const float* ps, int px,
                                   int py, int pz, int oi, int oj, int ok, float sc, float ss) {
  const int64_t total = static_cast<int64_t>(px) * py * pz;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int i, j, k;
    unflatten(x, py, pz, i, j, k);
    const int gi = oi + i, gj = oj + j, gk = ok + k;
    if (gi < 0 || gj < 0 || gk < 0 || gi >= fx || gj >= fy || gk >= fz) continue;
    field[off3(gi, gj, gk, fy, fz)] += sc * pc[x] + ss * ps[x];
  }
}

// Time-shifted patch: value = patch * w(time - delay[cell]) with the analytic
// waveform w of kind 0 (CW: A cos(omega t + phase)), 1 (Gaussian pulse:
// A exp(-(tau inv_sigma)^2 / 2) cos(omega tau + phase), tau = t - wdelay) or
// 2 (Ricker: A (1 - 2 a^2) exp(-a^2), a = pi f tau); with the causal gate a cell
// adds nothing before its activation time (witwin/maxwell/fdtd/cuda/kernels/
// sources.cu:173-221, waveforms.py:83-107).
__global__ void op_shifted_patch_kernel(float* field, int fx, int fy, int fz, const float* patch, const float* delay,
                                        const float* activation, int gate, int px, int py, int pz, int oi, int oj,
                                        int ok, int kind, float time, float omega, float inv_sigma, float pi_f,
                                        float amplitude, float phase, float wdelay) {
  const int64_t total = static_cast<int64_t>(px) * py * pz;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int i, j, k;
    unflatten(x, py, pz, i, j, k);
    const int gi = oi + i, gj = oj + j, gk = ok + k;
    if (gi < 0 || gj < 0 || gk < 0 || gi >= fx || gj >= fy || gk >= fz) continue;
    if (gate && time < activation[x]) continue;
    const float t = time - delay[x];
    float w;
    if (kind == 0) {
      w = amplitude * cosf(omega * t + phase);
    } else if (kind == 1) {
      const float tau = t - wdelay;
      const float a = tau * inv_sigma;
      w = amplitude * expf(-0.5f * a * a) * cosf(omega * tau + phase);
    } else {
      const float a = pi_f * (t - wdelay);
      w = amplitude * (1.0f - 2.0f * a * a) * expf(-a * a);
    }
    field[off3(gi, gj, gk, fy, fz)] += w * patch[x];
  }
}

__global__ void op_line_patch_kernel(float* field, int fx, int fy, int fz, const float* coeff, int px, int py, int pz,
                                     int oi, int oj, int ok, const float* inc, const int64_t* sidx, int axis,
                                     float scale) {
  const int64_t total = static_cast<int64_t>(px) * py * pz;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int i, j, k;
    unflatten(x, py, pz, i, j, k);
    const int gi = oi + i, gj = oj + j, gk = ok + k;
    if (gi < 0 || gj < 0 || gk < 0 || gi >= fx || gj >= fy || gk >= fz) continue;
    const int a = axis == 0 ? i : (axis == 1 ? j : k);
    field[off3(gi, gj, gk, fy, fz)] += coeff[x] * inc[sidx[a]] * scale;
  }
}

__global__ void op_aux_h_kernel(int ne, float* h, const float* e, const float* hd, const float* hc) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x < ne - 1) h[x] = hd[x] * h[x] - hc[x] * (e[x + 1] - e[x]);
}

__global__ void op_aux_e_kernel(int ne, float* e, const float* h, const float* ed, const float* ec, int src,
                                float value) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= ne) return;
  if (x == ne - 1) {
    e[x] = 0.0f;  // checked before the source cell, as the reference's op does
  } else if (x == src) {
    e[x] = value;
  } else if (x >= 1) {
    e[x] = ed[x] * e[x] - ec[x] * (h[x] - h[x - 1]);
  }
}

__global__ void op_points_kernel(const float* field, int fy, int fz, int np, const int* pi, const int* pj,
                                 const int* pk, float* re, float* im, float wc, float ws) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const float v = field[off3(pi[p], pj[p], pk[p], fy, fz)];
  re[p] += v * wc;
  im[p] += v * ws;
}

__global__ void op_plane_kernel(const float* field, int fx, int fy, int fz, int axis, int index, float* re, float* im,
                                float wc, float ws) {
  const int da = axis == 0 ? fy : fx;
  const int db = axis == 2 ? fy : fz;
  const int64_t total = static_cast<int64_t>(da) * db;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int a = static_cast<int>(x / db), b = static_cast<int>(x % db);
    int64_t o;
    if (axis == 0) o = off3(index, a, b, fy, fz);
    else if (axis == 1) o = off3(a, index, b, fy, fz);
    else o = off3(a, b, index, fy, fz);
    const float v = field[o];
    re[x] += v * wc;
    im[x] += v * ws;
  }
}

__global__ void op_dft_volume_kernel(int64_t n, int nf, const float* field, float* re, float* im, const float* wc,
                                     const float* ws) {
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < n;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float v = field[x];
    for (int f = 0; f < nf; ++f) {
      re[static_cast<int64_t>(f) * n + x] += v * wc[f];
      im[static_cast<int64_t>(f) * n + x] += v * ws[f];
    }
  }
}

__global__ void op_clamp_kernel(float* field, int fx, int fy, int fz, int axis, int side) {
  const int n[3] = {fx, fy, fz};
  const int idx = side == 0 ? 0 : n[axis] - 1;
  const int da = axis == 0 ? fy : fx;
  const int db = axis == 2 ? fy : fz;
  const int64_t total = static_cast<int64_t>(da) * db;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int a = static_cast<int>(x / db), b = static_cast<int>(x % db);
    int64_t o;
    if (axis == 0) o = off3(idx, a, b, fy, fz);
    else if (axis == 1) o = off3(a, idx, b, fy, fz);
    else o = off3(a, b, idx, fy, fz);
    field[o] = 0.0f;
  }
}

CpmlArgs make_cpml(float* psi_a, float* psi_b, const float* ika, const float* ba, const float* ca, const float* ikb,
                   const float* bb, const float* cb, const int* slab) {
  CpmlArgs c{};
  c.psi_a = psi_a;
  c.psi_b = psi_b;
  c.ika = ika;
  c.ba = ba;
  c.ca = ca;
  c.ikb = ikb;
  c.bb = bb;
  c.cb = cb;
  if (slab) {
    c.a_low = slab[0];
    c.a_hstart = slab[1];
    c.a_hlen = slab[2];
    c.b_low = slab[3];
    c.b_hstart = slab[4];
    c.b_hlen = slab[5];
  }
  return c;
}

bool cpml_args_ok(int mode, float* psi_a, float* psi_b, const float* ika, const float* ba, const float* ca,
                  const float* ikb, const float* bb, const float* cb, const int* slab) {
  if (mode == 0) return true;
  if (!psi_a || !psi_b || !ika || !ba || !ca || !ikb || !bb || !cb) return false;
  return mode == 1 || slab != nullptr;
}

// Instantaneous nonlinear coefficients of E component comp (kernels/
// dispersive.cu:165-400): E collocated onto comp's Yee edge (own component
// direct, the other two 4-point averaged with clamped indices), then the Kerr
// curl (general = 0: curl = dt / eps_eff * decay) or the general decay / curl
// pair (general = 1; dec is then the external decay).
struct NlShapes {
  int s[3][3];  // Ex, Ey, Ez array shapes
};

__device__ __forceinline__ float nl_at(const float* f, const NlShapes& sh, int c, int i, int j, int k) {
  i = min(max(i, 0), sh.s[c][0] - 1);
  j = min(max(j, 0), sh.s[c][1] - 1);
  k = min(max(k, 0), sh.s[c][2] - 1);
  return f[off3(i, j, k, sh.s[c][1], sh.s[c][2])];
}

__global__ void op_nonlinear_kernel(int comp, int general, NlShapes sh, const float* ex, const float* ey,
                                    const float* ez, const float* eps, const float* dec, const float* sig_s,
                                    const float* chi2, const float* chi3, const float* tpa, float dt, float eps0,
                                    float* out_decay, float* out_curl) {
  const int dx = sh.s[comp][0], dy = sh.s[comp][1], dz = sh.s[comp][2];
  const int64_t n = static_cast<int64_t>(dx) * dy * dz;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < n;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int i, j, k;
    unflatten(x, dy, dz, i, j, k);
    float vx, vy, vz;
    if (comp == 0) {
      vx = ex[x];
      vy = 0.25f * (nl_at(ey, sh, 1, i, j - 1, k) + nl_at(ey, sh, 1, i, j, k) + nl_at(ey, sh, 1, i + 1, j - 1, k) +
                    nl_at(ey, sh, 1, i + 1, j, k));
      vz = 0.25f * (nl_at(ez, sh, 2, i, j, k - 1) + nl_at(ez, sh, 2, i, j, k) + nl_at(ez, sh, 2, i + 1, j, k - 1) +
                    nl_at(ez, sh, 2, i + 1, j, k));
    } else if (comp == 1) {
      vx = 0.25f * (nl_at(ex, sh, 0, i - 1, j, k) + nl_at(ex, sh, 0, i, j, k) + nl_at(ex, sh, 0, i - 1, j + 1, k) +
                    nl_at(ex, sh, 0, i, j + 1, k));
      vy = ey[x];
      vz = 0.25f * (nl_at(ez, sh, 2, i, j, k - 1) + nl_at(ez, sh, 2, i, j, k) + nl_at(ez, sh, 2, i, j + 1, k - 1) +
                    nl_at(ez, sh, 2, i, j + 1, k));
    } else {
      vx = 0.25f * (nl_at(ex, sh, 0, i - 1, j, k) + nl_at(ex, sh, 0, i, j, k) + nl_at(ex, sh, 0, i - 1, j, k + 1) +
                    nl_at(ex, sh, 0, i, j, k + 1));
      vy = 0.25f * (nl_at(ey, sh, 1, i, j - 1, k) + nl_at(ey, sh, 1, i, j, k) + nl_at(ey, sh, 1, i, j - 1, k + 1) +
                    nl_at(ey, sh, 1, i, j, k + 1));
      vz = ez[x];
    }
    const float fsq = vx * vx + vy * vy + vz * vz;
    const float floor_eps = 1.0e-12f * eps0;
    if (!general) {
      float eff = eps[x] + eps0 * chi3[x] * fsq;
      if (eff < floor_eps) eff = floor_eps;
      out_curl[x] = (dt / eff) * dec[x];
    } else {
      const float own = comp == 0 ? vx : (comp == 1 ? vy : vz);
      float eff = eps[x] + eps0 * (chi2[x] * own + chi3[x] * fsq);
      if (eff < floor_eps) eff = floor_eps;
      float sigma = sig_s[x] + tpa[x] * fsq;
      if (sigma < 0.0f) sigma = 0.0f;
      const float half = 0.5f * sigma * dt / eff;
      const float inv_denom = 1.0f / (1.0f + half);
      out_decay[x] = dec[x] * (1.0f - half) * inv_denom;
      out_curl[x] = dec[x] * (dt / eff) * inv_denom;
    }
  }
}

// Off-diagonal (full-tensor) anisotropic coupling of E component comp
// (kernels/aniso.cu:26-580): E_c += coeff_a <curlH_a> / 4 + coeff_b <curlH_b> / 4,
// with <curlH_d> the sum of curl(H)_d over the four d-edges around the E_c edge
// (curl from H with backward differences at each d-edge).  A sample whose
// stencil leaves a non-periodic axis is skipped; periodic axes wrap (the last
// node duplicates node 0).  Cells with both coefficients zero are untouched.
struct AnisoGrid {
  int n[3];      // node counts
  int per[3];    // periodic flags
  const float* h[3];
  const float* inv[3];
};

// Edge coordinate (array length n - 1) wrapped on a periodic axis; -1 = skip.
__device__ __forceinline__ int aniso_edge(int c, int n, int per) {
  if (c >= 0 && c < n - 1) return c;
  if (!per) return -1;
  return c < 0 ? c + (n - 1) : c - (n - 1);
}

// Backward edge pair (c - 1, c) at node coordinate c (after the periodic node map).
__device__ __forceinline__ bool aniso_pair(int& c, int n, int per, int& lo, int& hi) {
  if (per && c == n - 1) c = 0;
  hi = c;
  lo = c - 1;
  if (hi > n - 2) {
    if (!per) return false;
    hi -= n - 1;
  }
  if (lo < 0) {
    if (!per) return false;
    lo += n - 1;
  }
  return true;
}

__device__ __forceinline__ float aniso_h(const AnisoGrid& g, int c, int i, int j, int k) {
  // H shapes: Hx (n0, n1 - 1, n2 - 1), Hy (n0 - 1, n1, n2 - 1), Hz (n0 - 1, n1 - 1, n2)
  const int ny = c == 1 ? g.n[1] : g.n[1] - 1;
  const int nz = c == 2 ? g.n[2] : g.n[2] - 1;
  return __ldg(g.h[c] + off3(i, j, k, ny, nz));
}

// curl(H)_d at the d-edge (s0, s1, s2) (s_d an edge coordinate, the others
// node coordinates); false when the sample is skipped.
__device__ bool aniso_curl(const AnisoGrid& g, int d, int s0, int s1, int s2, float& value) {
  int s[3] = {s0, s1, s2};
  s[d] = aniso_edge(s[d], g.n[d], g.per[d]);
  if (s[d] < 0) return false;
  const int a = d == 0 ? 1 : 0, b = d == 2 ? 1 : 2;  // the two derivative axes, a < b
  int alo, ahi, blo, bhi;
  if (!aniso_pair(s[a], g.n[a], g.per[a], alo, ahi) || !aniso_pair(s[b], g.n[b], g.per[b], blo, bhi)) return false;
  // curl_d = d(H_b')/da - d(H_a')/db with the cyclic pairs of (d, a, b):
  //   x: dHz/dy - dHy/dz;  y: dHx/dz - dHz/dx;  z: dHy/dx - dHx/dy
  if (d == 1) {
    // dHx/dz (Hx at (s0, s1, z)) - dHz/dx (Hz at (x, s1, s2))
    const float d_z = (aniso_h(g, 0, s[0], s[1], bhi) - aniso_h(g, 0, s[0], s[1], blo)) * __ldg(g.inv[2] + s[2]);
    const float d_x = (aniso_h(g, 2, ahi, s[1], s[2]) - aniso_h(g, 2, alo, s[1], s[2])) * __ldg(g.inv[0] + s[0]);
    value = d_z - d_x;
  } else if (d == 0) {
    // dHz/dy (Hz at (s0, y, s2)) - dHy/dz (Hy at (s0, s1, z))
    const float d_y = (aniso_h(g, 2, s[0], ahi, s[2]) - aniso_h(g, 2, s[0], alo, s[2])) * __ldg(g.inv[1] + s[1]);
    const float d_z = (aniso_h(g, 1, s[0], s[1], bhi) - aniso_h(g, 1, s[0], s[1], blo)) * __ldg(g.inv[2] + s[2]);
    value = d_y - d_z;
  } else {
    // dHy/dx (Hy at (x, s1, s2)) - dHx/dy (Hx at (s0, y, s2))
    const float d_x = (aniso_h(g, 1, ahi, s[1], s[2]) - aniso_h(g, 1, alo, s[1], s[2])) * __ldg(g.inv[0] + s[0]);
    const float d_y = (aniso_h(g, 0, s[0], bhi, s[2]) - aniso_h(g, 0, s[0], blo, s[2])) * __ldg(g.inv[1] + s[1]);
    value = d_x - d_y;
  }
  return true;
}

__global__ void op_full_aniso_kernel(int comp, AnisoGrid g, const float* __restrict__ ca, const float* __restrict__ cb,
                                     float* __restrict__ e) {
  const int ex = comp == 0 ? g.n[0] - 1 : g.n[0], ey = comp == 1 ? g.n[1] - 1 : g.n[1];
  const int ez = comp == 2 ? g.n[2] - 1 : g.n[2];
  const int64_t total = static_cast<int64_t>(ex) * ey * ez;
  // the two off-axis curl components (a < b) and, per axis, the offsets of the
  // four neighbouring edges: the own axis spans {c, c + 1} (node positions
  // around the half-index edge), the curl's axis spans {c - 1, c}
  const int da = comp == 0 ? 1 : 0, db = comp == 2 ? 1 : 2;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float c_a = ca[x], c_b = cb[x];
    if (c_a == 0.0f && c_b == 0.0f) continue;
    int i, j, k;
    unflatten(x, ey, ez, i, j, k);
    const int pos[3] = {i, j, k};
    float acc[2] = {0.0f, 0.0f};
    for (int t = 0; t < 2; ++t) {
      const int d = t == 0 ? da : db;
      if ((t == 0 ? c_a : c_b) == 0.0f) continue;
      // own axis offsets {0, +1}, curl axis d offsets {-1, 0}; the lower of the
      // two axes is the outer loop (the reference's summation order)
      const int outer = min(comp, d), inner = max(comp, d);
      for (int u = 0; u < 2; ++u)
        for (int v = 0; v < 2; ++v) {
          int s[3] = {pos[0], pos[1], pos[2]};
          s[outer] += outer == comp ? u : u - 1;
          s[inner] += inner == comp ? v : v - 1;
          float sample;
          if (aniso_curl(g, d, s[0], s[1], s[2], sample)) acc[t] += sample;
        }
    }
    e[x] += 0.25f * (c_a * acc[0] + c_b * acc[1]);
  }
}

bool nl_shapes(const int* shapes, NlShapes& sh) {
  if (!shapes) return false;
  for (int c = 0; c < 3; ++c)
    for (int a = 0; a < 3; ++a) {
      sh.s[c][a] = shapes[3 * c + a];
      if (sh.s[c][a] <= 0) return false;
    }
  return true;
}

}  // namespace

extern "C" {

int fdtd_op_update_magnetic(int comp, int mode, int nx, int ny, int nz, float* field, const float* first,
                            const float* second, const float* decay, const float* curl, float decay_u,
                            float curl_u, const float* inv_a, const float* inv_b, float* psi_a, float* psi_b,
                            const float* ika, const float* ba, const float* ca, const float* ikb,
                            const float* bb, const float* cb, const int* slab, void* stream) {
  if (comp < 0 || comp > 2 || mode < 0 || mode > 2 || nx <= 0 || ny <= 0 || nz <= 0 || !field || !first ||
      !second || !inv_a || !inv_b)
    return op_fail(FDTD_ERR_INVALID_ARG, "update_magnetic: bad arguments");
  if (!cpml_args_ok(mode, psi_a, psi_b, ika, ba, ca, ikb, bb, cb, slab))
    return op_fail(FDTD_ERR_INVALID_ARG, "update_magnetic: missing CPML arguments");
  const int64_t n = static_cast<int64_t>(nx) * ny * nz;
  op_magnetic_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      comp, mode, nx, ny, nz, field, first, second, decay, curl, decay_u, curl_u, inv_a, inv_b,
      make_cpml(psi_a, psi_b, ika, ba, ca, ikb, bb, cb, slab));
  return op_launch_check("update_magnetic");
}

int fdtd_op_update_electric(int comp, int mode, int nx, int ny, int nz, float* field, const float* first,
                            const float* second, const float* decay, const float* curl, float decay_u,
                            float curl_u, const float* inv_a, const float* inv_b, const int* modes,
                            float* psi_a, float* psi_b, const float* ika, const float* ba, const float* ca,
                            const float* ikb, const float* bb, const float* cb, const int* slab, void* stream) {
  if (comp < 0 || comp > 2 || mode < 0 || mode > 2 || nx < 2 || ny < 2 || nz < 2 || !field || !first || !second ||
      !inv_a || !inv_b || !modes)
    return op_fail(FDTD_ERR_INVALID_ARG, "update_electric: bad arguments");
  for (int m = 0; m < 4; ++m)
    if (modes[m] == BND_BLOCH) return op_fail(FDTD_ERR_UNSUPPORTED, "update_electric: Bloch faces need the complex kernels");
  if (!cpml_args_ok(mode, psi_a, psi_b, ika, ba, ca, ikb, bb, cb, slab))
    return op_fail(FDTD_ERR_INVALID_ARG, "update_electric: missing CPML arguments");
  const int64_t n = static_cast<int64_t>(nx) * ny * nz;
  op_electric_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      comp, mode, nx, ny, nz, field, first, second, decay, curl, decay_u, curl_u, inv_a, inv_b, modes[0],
      modes[1], modes[2], modes[3], make_cpml(psi_a, psi_b, ika, ba, ca, ikb, bb, cb, slab));
  return op_launch_check("update_electric");
}

int fdtd_op_update_debye(int64_t n, const float* e, const float* drive, float decay, float dt, float* pol,
                         float* cur, void* stream) {
  if (n < 0 || !e || !drive || !pol || !cur || !(dt > 0.0f)) return op_fail(FDTD_ERR_INVALID_ARG, "update_debye: bad arguments");
  if (n == 0) return 0;
  op_debye_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(n, e, drive, decay, 1.0f / dt, pol, cur);
  return op_launch_check("update_debye");
}

int fdtd_op_update_drude(int64_t n, const float* e, const float* drive, float decay, float* cur, void* stream) {
  if (n < 0 || !e || !drive || !cur) return op_fail(FDTD_ERR_INVALID_ARG, "update_drude: bad arguments");
  if (n == 0) return 0;
  op_drude_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(n, e, drive, decay, cur);
  return op_launch_check("update_drude");
}

int fdtd_op_update_lorentz(int64_t n, const float* e, const float* drive, float decay, float restoring,
                           float dt, float* pol, float* cur, void* stream) {
  if (n < 0 || !e || !drive || !pol || !cur) return op_fail(FDTD_ERR_INVALID_ARG, "update_lorentz: bad arguments");
  if (n == 0) return 0;
  op_lorentz_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(n, e, drive, decay, restoring, dt, pol, cur);
  return op_launch_check("update_lorentz");
}

int fdtd_op_apply_polarization(int64_t n, const float* cur, const float* inv_eps, float dt, float* e,
                               void* stream) {
  if (n < 0 || !cur || !inv_eps || !e) return op_fail(FDTD_ERR_INVALID_ARG, "apply_polarization: bad arguments");
  if (n == 0) return 0;
  op_apply_pol_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(n, cur, inv_eps, dt, e);
  return op_launch_check("apply_polarization");
}

int fdtd_op_add_source_patch(float* field, const int* fshape, const float* patch, const int* pshape,
                             const int* offset, float signal, void* stream) {
  if (!field || !fshape || !patch || !pshape || !offset) return op_fail(FDTD_ERR_INVALID_ARG, "add_source_patch: bad arguments");
  const int64_t n = static_cast<int64_t>(pshape[0]) * pshape[1] * pshape[2];
  if (n <= 0) return 0;
  op_patch_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      field, fshape[0], fshape[1], fshape[2], patch, pshape[0], pshape[1], pshape[2], offset[0], offset[1], offset[2], signal);
  return op_launch_check("add_source_patch");
}

int fdtd_op_update_electric_bloch(int comp, int z_standard, int nx, int ny, int nz, float* e_re, float* e_im,
                                  const float* first_re, const float* first_im, const float* second_re,
                                  const float* second_im, const float* decay, const float* curl, float phase_cos_a,
                                  float phase_sin_a, float phase_cos_b, float phase_sin_b, const float* inv_a,
                                  const float* inv_b, int z_low_mode, int z_high_mode, void* stream) {
  if (comp < 0 || comp > 2 || (z_standard && comp == 2) || nx < 2 || ny < 2 || nz < 2 || !e_re || !e_im ||
      !first_re || !first_im || !second_re || !second_im || !decay || !curl || !inv_a || !inv_b)
    return op_fail(FDTD_ERR_INVALID_ARG, "update_electric_bloch: bad arguments");
  const int64_t n = static_cast<int64_t>(nx) * ny * nz;
  op_electric_bloch_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      comp, z_standard ? 1 : 0, nx, ny, nz, e_re, e_im, first_re, first_im, second_re, second_im, decay, curl,
      phase_cos_a, phase_sin_a, phase_cos_b, phase_sin_b, inv_a, inv_b, z_low_mode, z_high_mode);
  return op_launch_check("update_electric_bloch");
}

int fdtd_op_apply_cpml_z_correction(int comp, float* field, const int* fshape, const float* h, const int* hshape,
                                    const float* curl, float* psi, const float* inv_kappa, const float* b,
                                    const float* c, const float* inv_dz, const int* offset, int low_mode,
                                    int high_mode, int full_size_t, int full_size_z, void* stream) {
  if (comp < 0 || comp > 1 || !field || !fshape || !h || !hshape || !curl || !psi || !inv_kappa || !b || !c ||
      !inv_dz || !offset)
    return op_fail(FDTD_ERR_INVALID_ARG, "apply_cpml_z_correction: bad arguments");
  const int k0 = std::max(0, 1 - offset[2]);
  const int k1 = std::min(fshape[2], full_size_z - 1 - offset[2]);
  if (k1 <= k0 || fshape[0] <= 0 || fshape[1] <= 0) return 0;
  const int64_t n = static_cast<int64_t>(fshape[0]) * fshape[1] * (k1 - k0);
  op_cpml_z_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      comp, field, fshape[0], fshape[1], fshape[2], h, hshape[1], hshape[2], curl, psi, inv_kappa, b, c, inv_dz,
      offset[0], offset[1], offset[2], low_mode, high_mode, full_size_t, k0, k1);
  return op_launch_check("apply_cpml_z_correction");
}

int fdtd_op_project_periodic(float* field, const int* fshape, int axis, void* stream) {
  if (!field || !fshape || axis < 0 || axis > 2) return op_fail(FDTD_ERR_INVALID_ARG, "project_periodic: bad arguments");
  const int64_t n = static_cast<int64_t>(axis == 0 ? fshape[1] : fshape[0]) * (axis == 2 ? fshape[1] : fshape[2]);
  if (n <= 0) return 0;
  op_project_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      field, nullptr, fshape[0], fshape[1], fshape[2], axis, 1.0f, 0.0f);
  return op_launch_check("project_periodic");
}

int fdtd_op_project_bloch(float* field_re, float* field_im, const int* fshape, int axis, float phase_cos,
                          float phase_sin, void* stream) {
  if (!field_re || !field_im || !fshape || axis < 0 || axis > 2)
    return op_fail(FDTD_ERR_INVALID_ARG, "project_bloch: bad arguments");
  const int64_t n = static_cast<int64_t>(axis == 0 ? fshape[1] : fshape[0]) * (axis == 2 ? fshape[1] : fshape[2]);
  if (n <= 0) return 0;
  op_project_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      field_re, field_im, fshape[0], fshape[1], fshape[2], axis, phase_cos, phase_sin);
  return op_launch_check("project_bloch");
}

int fdtd_op_add_cw_patch(float* field, const int* fshape, const float* patch_cos, const float* patch_sin,
                         const int* pshape, const int* offset, float signal_cos, float signal_sin, void* stream) {
  if (!field || !fshape || !patch_cos || !patch_sin || !pshape || !offset)
    return op_fail(FDTD_ERR_INVALID_ARG, "add_cw_patch: bad arguments");
  const int64_t n = static_cast<int64_t>(pshape[0]) * pshape[1] * pshape[2];
  if (n <= 0) return 0;
  op_cw_patch_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      field, fshape[0], fshape[1], fshape[2], patch_cos, patch_sin, pshape[0], pshape[1], pshape[2], offset[0],
      offset[1], offset[2], signal_cos, signal_sin);
  return op_launch_check("add_cw_patch");
}

int fdtd_op_add_shifted_patch(float* field, const int* fshape, const float* patch, const float* delay,
                              const float* activation, int causal_gate, const int* pshape, const int* offset, int kind,
                              float time, float frequency, float fwidth, float amplitude, float phase, float wdelay,
                              void* stream) {
  if (!field || !fshape || !patch || !delay || !pshape || !offset || kind < 0 || kind > 2 ||
      (causal_gate && !activation))
    return op_fail(FDTD_ERR_INVALID_ARG, "add_shifted_patch: bad arguments");
  const int64_t n = static_cast<int64_t>(pshape[0]) * pshape[1] * pshape[2];
  if (n <= 0) return 0;
  constexpr double kPi = 3.141592653589793;
  const float inv_sigma = static_cast<float>(std::max(2.0 * kPi * fwidth, 1e-30));
  op_shifted_patch_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      field, fshape[0], fshape[1], fshape[2], patch, delay, activation, causal_gate ? 1 : 0, pshape[0], pshape[1],
      pshape[2], offset[0], offset[1], offset[2], kind, time, static_cast<float>(2.0 * kPi * frequency), inv_sigma,
      static_cast<float>(kPi * frequency), amplitude, phase, wdelay);
  return op_launch_check("add_shifted_patch");
}

int fdtd_op_add_line_patch(float* field, const int* fshape, const float* coeff, const int* pshape,
                           const int* offset, const float* incident, const int64_t* sample_idx, int axis,
                           float scale, void* stream) {
  if (!field || !fshape || !coeff || !pshape || !offset || !incident || !sample_idx || axis < 0 || axis > 2)
    return op_fail(FDTD_ERR_INVALID_ARG, "add_line_patch: bad arguments");
  const int64_t n = static_cast<int64_t>(pshape[0]) * pshape[1] * pshape[2];
  if (n <= 0) return 0;
  op_line_patch_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      field, fshape[0], fshape[1], fshape[2], coeff, pshape[0], pshape[1], pshape[2], offset[0], offset[1],
      offset[2], incident, sample_idx, axis, scale);
  return op_launch_check("add_line_patch");
}

int fdtd_op_aux_magnetic(int n_e, float* h, const float* e, const float* h_decay, const float* h_curl,
                         void* stream) {
  if (n_e < 2 || !h || !e || !h_decay || !h_curl) return op_fail(FDTD_ERR_INVALID_ARG, "aux_magnetic: bad arguments");
  op_aux_h_kernel<<<blocks_for(n_e), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(n_e, h, e, h_decay, h_curl);
  return op_launch_check("aux_magnetic");
}

int fdtd_op_aux_electric(int n_e, float* e, const float* h, const float* e_decay, const float* e_curl,
                         int source_index, float source_value, void* stream) {
  if (n_e < 2 || !h || !e || !e_decay || !e_curl) return op_fail(FDTD_ERR_INVALID_ARG, "aux_electric: bad arguments");
  // Interior cells read h only, so a single pass is race free.
  op_aux_e_kernel<<<blocks_for(n_e), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(n_e, e, h, e_decay, e_curl,
                                                                                         source_index, source_value);
  return op_launch_check("aux_electric");
}

int fdtd_op_point_observers(const float* field, const int* fshape, int n_points, const int* pi, const int* pj,
                            const int* pk, float* re, float* im, float wcos, float wsin, void* stream) {
  if (!field || !fshape || n_points < 0 || !pi || !pj || !pk || !re || !im)
    return op_fail(FDTD_ERR_INVALID_ARG, "point_observers: bad arguments");
  if (n_points == 0) return 0;
  op_points_kernel<<<blocks_for(n_points), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      field, fshape[1], fshape[2], n_points, pi, pj, pk, re, im, wcos, wsin);
  return op_launch_check("point_observers");
}

int fdtd_op_plane_observer(const float* field, const int* fshape, int axis, int index, float* re, float* im,
                           float wcos, float wsin, void* stream) {
  if (!field || !fshape || axis < 0 || axis > 2 || !re || !im || index < 0 || index >= fshape[axis])
    return op_fail(FDTD_ERR_INVALID_ARG, "plane_observer: bad arguments");
  const int da = axis == 0 ? fshape[1] : fshape[0];
  const int db = axis == 2 ? fshape[1] : fshape[2];
  op_plane_kernel<<<blocks_for(static_cast<int64_t>(da) * db), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      field, fshape[0], fshape[1], fshape[2], axis, index, re, im, wcos, wsin);
  return op_launch_check("plane_observer");
}

int fdtd_op_dft_volume(int64_t n, int n_freq, const float* field, float* re, float* im, const float* wcos,
                       const float* wsin, void* stream) {
  if (n < 0 || n_freq <= 0 || !field || !re || !im || !wcos || !wsin)
    return op_fail(FDTD_ERR_INVALID_ARG, "dft_volume: bad arguments");
  if (n == 0) return 0;
  op_dft_volume_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(n, n_freq, field, re, im, wcos, wsin);
  return op_launch_check("dft_volume");
}

int fdtd_op_clamp_face(float* field, const int* fshape, int axis, int side, void* stream) {
  if (!field || !fshape || axis < 0 || axis > 2 || side < 0 || side > 1)
    return op_fail(FDTD_ERR_INVALID_ARG, "clamp_face: bad arguments");
  const int da = axis == 0 ? fshape[1] : fshape[0];
  const int db = axis == 2 ? fshape[1] : fshape[2];
  op_clamp_kernel<<<blocks_for(static_cast<int64_t>(da) * db), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      field, fshape[0], fshape[1], fshape[2], axis, side);
  return op_launch_check("clamp_face");
}

int fdtd_op_update_kerr_curl(int comp, const int* shapes, const float* ex, const float* ey, const float* ez,
                             const float* eps, const float* decay, const float* chi3, float dt, float eps0,
                             float* curl, void* stream) {
  NlShapes sh;
  if (comp < 0 || comp > 2 || !nl_shapes(shapes, sh) || !ex || !ey || !ez || !eps || !decay || !chi3 || !curl)
    return op_fail(FDTD_ERR_INVALID_ARG, "update_kerr_curl: bad arguments");
  const int64_t n = static_cast<int64_t>(sh.s[comp][0]) * sh.s[comp][1] * sh.s[comp][2];
  op_nonlinear_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      comp, 0, sh, ex, ey, ez, eps, decay, nullptr, nullptr, chi3, nullptr, dt, eps0, nullptr, curl);
  return op_launch_check("update_kerr_curl");
}

int fdtd_op_update_nonlinear_coefficients(int comp, const int* shapes, const float* ex, const float* ey,
                                          const float* ez, const float* eps, const float* external_decay,
                                          const float* sigma, const float* chi2, const float* chi3, const float* tpa,
                                          float dt, float eps0, float* decay, float* curl, void* stream) {
  NlShapes sh;
  if (comp < 0 || comp > 2 || !nl_shapes(shapes, sh) || !ex || !ey || !ez || !eps || !external_decay || !sigma ||
      !chi2 || !chi3 || !tpa || !decay || !curl)
    return op_fail(FDTD_ERR_INVALID_ARG, "update_nonlinear_coefficients: bad arguments");
  const int64_t n = static_cast<int64_t>(sh.s[comp][0]) * sh.s[comp][1] * sh.s[comp][2];
  op_nonlinear_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      comp, 1, sh, ex, ey, ez, eps, external_decay, sigma, chi2, chi3, tpa, dt, eps0, decay, curl);
  return op_launch_check("update_nonlinear_coefficients");
}

int fdtd_op_update_electric_full_aniso(int comp, int nx, int ny, int nz, float* e, const float* hx, const float* hy,
                                       const float* hz, const float* coeff_a, const float* coeff_b,
                                       const float* inv_dx, const float* inv_dy, const float* inv_dz, int periodic_x,
                                       int periodic_y, int periodic_z, void* stream) {
  if (comp < 0 || comp > 2 || nx < 2 || ny < 2 || nz < 2 || !e || !hx || !hy || !hz || !coeff_a || !coeff_b ||
      !inv_dx || !inv_dy || !inv_dz)
    return op_fail(FDTD_ERR_INVALID_ARG, "update_electric_full_aniso: bad arguments");
  AnisoGrid g;
  g.n[0] = nx;
  g.n[1] = ny;
  g.n[2] = nz;
  g.per[0] = periodic_x != 0;
  g.per[1] = periodic_y != 0;
  g.per[2] = periodic_z != 0;
  g.h[0] = hx;
  g.h[1] = hy;
  g.h[2] = hz;
  g.inv[0] = inv_dx;
  g.inv[1] = inv_dy;
  g.inv[2] = inv_dz;
  const int64_t n = static_cast<int64_t>(comp == 0 ? nx - 1 : nx) * (comp == 1 ? ny - 1 : ny) * (comp == 2 ? nz - 1 : nz);
  op_full_aniso_kernel<<<blocks_for(n), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(comp, g, coeff_a, coeff_b, e);
  return op_launch_check("update_electric_full_aniso");
}

}  // extern "C"
