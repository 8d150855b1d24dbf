// Host side of the fused step engine and its C ABI (include/fdtd_b200.h).
//
// The engine owns its device state in an internal padded layout: every field
// component lives in an [NX][NY][P] array (P = NZ rounded up to a multiple of
// 4 so each z row starts on a 16-byte boundary and can be read as float4),
// cells outside a component's Yee extent are held at zero.  CPML psi arrays
// are kept only on their slabs; ADE state only on the pole boxes.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <type_traits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/fdtd_b200.h"
#include "engine.cuh"
#include "tma_step.cuh"
#include "adjoint.cuh"

namespace fdtdb200 {
template <bool kCpml, bool kCoef, bool kUniform, int kMinBlocks, bool kAde>
__global__ void warp_step_kernel(const StepParams p, int n, int slot);
int launch_classify_vec(const StepParams& p, int V, int n_kblocks, int n_chunks, unsigned char* out,
                        cudaStream_t stream);
int launch_step_reduced(const StepParams& p, int n, dim3 grid, bool cpml, bool coef, bool uni, cudaStream_t stream);
int launch_tile_step(const StepParams& p, const TmaMaps& maps, int n, dim3 grid, bool cpml, bool coef, bool uni,
                     cudaStream_t stream);
int tile_block_threads();
using VecLauncher = int (*)(const StepParams&, int, dim3, bool, bool, bool, cudaStream_t);
int launch_vec_v4(const StepParams&, int, dim3, bool, bool, bool, cudaStream_t);
int launch_vec_v2(const StepParams&, int, dim3, bool, bool, bool, cudaStream_t);
int launch_vec_r2d4(const StepParams&, int, dim3, bool, bool, bool, cudaStream_t);
int launch_vec_r2d3(const StepParams&, int, dim3, bool, bool, bool, cudaStream_t);
int launch_vec_r4d3(const StepParams&, int, dim3, bool, bool, bool, cudaStream_t);
}

using namespace fdtdb200;

namespace {

thread_local std::string g_last_error;

// An NVTX range over a host entry point (step ranges, replay, reverse,
// checkpoints, autotune): names the enqueue span on a profiler's timeline;
// without an attached tool the calls return at once.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

}  // namespace

void fdtdb200::set_last_error(const std::string& msg) { g_last_error = msg; }

namespace {

int cuda_fail(cudaError_t err, const char* what) {
  return fail(FDTD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
}

#define CUDA_TRY(expr)                              \
  do {                                              \
    cudaError_t err__ = (expr);                     \
    if (err__ != cudaSuccess) return cuda_fail(err__, #expr); \
  } while (0)

int axis_a(int comp) { return comp == 0 ? 1 : 0; }
int axis_b(int comp) { return comp == 2 ? 1 : 2; }

// Yee extent of component comp (0..2 E, 3..5 H) on a node grid.
void comp_extent(int comp, int NX, int NY, int NZ, int ext[3]) {
  const int c = comp % 3;
  const bool is_h = comp >= 3;
  int n[3] = {NX, NY, NZ};
  for (int a = 0; a < 3; ++a) {
    // E component c is half-cell (N-1) along its own axis; H component c is
    // half-cell along the two other axes.
    const bool half = is_h ? (a != c) : (a == c);
    ext[a] = half ? n[a] - 1 : n[a];
  }
}

// Dense [sx][sy][sz] <-> internal [.][NY][P] copies.  Inner coordinates
// k >= zlo move by zshift (the high segment of a z-slab psi row); every other
// array passes zlo = INT_MAX.
__global__ void pack_kernel(float* dst, const float* src, int sx, int sy, int sz, int NY, int P, int zlo,
                            int zshift) {
  const int64_t total = static_cast<int64_t>(sx) * sy * sz;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(x % sz);
    const int64_t r = x / sz;
    const int j = static_cast<int>(r % sy);
    const int i = static_cast<int>(r / sy);
    dst[(static_cast<int64_t>(i) * NY + j) * P + (k < zlo ? k : k + zshift)] = src[x];
  }
}

__global__ void unpack_kernel(float* dst, const float* src, int sx, int sy, int sz, int NY, int P, int zlo,
                              int zshift) {
  const int64_t total = static_cast<int64_t>(sx) * sy * sz;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(x % sz);
    const int64_t r = x / sz;
    const int j = static_cast<int>(r % sy);
    const int i = static_cast<int>(r / sy);
    dst[x] = src[(static_cast<int64_t>(i) * NY + j) * P + (k < zlo ? k : k + zshift)];
  }
}

constexpr int kNoRemap = 0x7fffffff;

// Dense FP32 [sx][sy][sz] <-> internal reduced-storage [.][NY][P] field
// (value = stored * scale).
template <typename TS>
__global__ void pack_field_rs_kernel(TS* dst, const float* src, int sx, int sy, int sz, int NY, int P, float inv) {
  const int64_t total = static_cast<int64_t>(sx) * sy * sz;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(x % sz);
    const int64_t r = x / sz;
    const int j = static_cast<int>(r % sy);
    const int i = static_cast<int>(r / sy);
    const float v = src[x] * inv;
    TS out;
    if constexpr (sizeof(TS) == 2 && std::is_same<TS, __half>::value) out = __float2half_rn(v);
    else out = __float2bfloat16_rn(v);
    dst[(static_cast<int64_t>(i) * NY + j) * P + k] = out;
  }
}

template <typename TS>
__global__ void unpack_field_rs_kernel(float* dst, const TS* src, int sx, int sy, int sz, int NY, int P, float scale) {
  const int64_t total = static_cast<int64_t>(sx) * sy * sz;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(x % sz);
    const int64_t r = x / sz;
    const int j = static_cast<int>(r % sy);
    const int i = static_cast<int>(r / sy);
    const TS v = src[(static_cast<int64_t>(i) * NY + j) * P + k];
    float f;
    if constexpr (std::is_same<TS, __half>::value) f = __half2float(v);
    else f = __bfloat162float(v);
    dst[x] = f * scale;
  }
}

// BF16 pole state [rows][nkk] (cells [koff, koff + nk) of each row) -> dense FP32 [rows][nk].
__global__ void unpack_pole_bf16_kernel(float* dst, const __nv_bfloat16* src, int64_t rows, int nk, int nkk, int koff) {
  const int64_t total = rows * nk;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = x / nk;
    const int k = static_cast<int>(x % nk);
    dst[x] = __bfloat162float(src[r * nkk + koff + k]);
  }
}

// Precompute the history of a 1-D incident line (one block, sequential in time).
// Restates AuxiliaryGrid1D.advance_magnetic / advance_electric,
// witwin/maxwell/fdtd/excitation/spatial.py:443-462 and sources.cu:803-839.
__global__ void aux_history_kernel(int ne, const float* e_decay, const float* e_curl, const float* h_decay,
                                   const float* h_curl, int src_index, const float* source, int n_steps,
                                   float* e_hist, float* h_hist, float* e, float* h) {
  for (int x = threadIdx.x; x < ne; x += blockDim.x) {
    e[x] = 0.0f;
    if (x < ne - 1) h[x] = 0.0f;
  }
  __syncthreads();
  for (int n = 0; n < n_steps; ++n) {
    for (int x = threadIdx.x; x < ne; x += blockDim.x) e_hist[static_cast<int64_t>(n) * ne + x] = e[x];
    for (int x = threadIdx.x; x < ne - 1; x += blockDim.x) h[x] = h_decay[x] * h[x] - h_curl[x] * (e[x + 1] - e[x]);
    __syncthreads();
    for (int x = threadIdx.x; x < ne - 1; x += blockDim.x) h_hist[static_cast<int64_t>(n) * ne + x] = h[x];
    for (int x = threadIdx.x; x < ne; x += blockDim.x) {
      if (x >= 1 && x < ne - 1 && x != src_index) e[x] = e_decay[x] * e[x] - e_curl[x] * (h[x] - h[x - 1]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      // the source cell first, then the last cell pinned to zero: a source
      // placed on the last cell is overridden, as in the reference's op
      if (src_index >= 0 && src_index < ne) e[src_index] = source[n];
      e[ne - 1] = 0.0f;
    }
    __syncthreads();
  }
}

// DFT weights in FP64: phase = omega * (n [- 1/2]) * dt reduced modulo 2*pi in
// double precision, window applied, stored as float2 (cos, sin).
// window: one weight per step (per_freq 0) or per (step, frequency) (1).
__global__ void dft_weight_kernel(int n_freq, int n_steps, const double* omega, const double* window, int per_freq,
                                  double dt, float2* w_e, float2* w_h) {
  const int64_t total = static_cast<int64_t>(n_freq) * n_steps;
  const double two_pi = 6.283185307179586476925286766559;
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int n = static_cast<int>(x / n_freq);
    const int f = static_cast<int>(x % n_freq);
    const double w = per_freq ? window[x] : window[n];
    double pe = fmod(omega[f] * dt * static_cast<double>(n), two_pi);
    double ph = fmod(omega[f] * dt * (static_cast<double>(n) - 0.5), two_pi);
    double se, ce, sh, ch;
    sincos(pe, &se, &ce);
    sincos(ph, &sh, &ch);
    w_e[x] = make_float2(static_cast<float>(w * ce), static_cast<float>(w * se));
    w_h[x] = make_float2(static_cast<float>(w * ch), static_cast<float>(w * sh));
  }
}

// Copy the monitor cells of every sample region from the current fields into
// sample slot `slot` (one CTA column per region; observers.cu:7-78 sample the
// same values: E^{n+1} and H^{n+1/2} after all corrections of the step).
struct FieldPtrs {
  const float* f[6];
  int storage;       // kStoreF32 / kStoreF16 / kStoreBF16
  float scale[6];    // stored value * scale = field value (reduced storage)
};

__device__ __forceinline__ float load_field(const FieldPtrs& fp, int comp, int64_t off) {
  if (fp.storage == kStoreF16) return __half2float(reinterpret_cast<const __half*>(fp.f[comp])[off]) * fp.scale[comp];
  if (fp.storage == kStoreBF16)
    return __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(fp.f[comp])[off]) * fp.scale[comp];
  return __ldg(fp.f[comp] + off);
}

// Cells a thread of the gather loads before it stores any: a z-normal region
// reads one value per z row (one DRAM sector each), so the gather is bound by
// load latency unless several loads are in flight per thread.
constexpr int kGatherIlp = 4;

__global__ void sample_gather_kernel(const RegionFlush* regions, const FieldPtrs fields, int NY, int P,
                                     float* samples, int64_t n_samples, int slot) {
  const RegionFlush rg = regions[blockIdx.y];
  float* out = samples + static_cast<int64_t>(slot) * n_samples + rg.base;
  // 32-bit cell arithmetic: a region holds fewer than 2^31 cells (checked at set-up)
  const int count = static_cast<int>(rg.count), nk = rg.nk, nj = rg.nj;
  const int stride = gridDim.x * blockDim.x;
  for (int x0 = blockIdx.x * blockDim.x + threadIdx.x; x0 < count; x0 += stride * kGatherIlp) {
    float v[kGatherIlp];
#pragma unroll
    for (int u = 0; u < kGatherIlp; ++u) {
      const int x = x0 + u * stride;
      v[u] = 0.0f;
      if (x < count) {
        const int r = x / nk;
        const int lk = x - r * nk;
        const int li = r / nj;
        const int lj = r - li * nj;
        v[u] = load_field(fields, rg.comp, (static_cast<int64_t>(rg.i0 + li) * NY + rg.j0 + lj) * P + rg.k0 + lk);
      }
    }
#pragma unroll
    for (int u = 0; u < kGatherIlp; ++u)
      if (x0 + u * stride < count) out[x0 + u * stride] = v[u];
  }
}

// acc[f][slot] += sum_m sample[m][slot] * w[n_base + m][f], with Kahan
// compensation of the accumulator update.
__global__ void dft_flush_kernel(const float* samples, int64_t n_samples, int cnt, int n_base, int n_freq,
                                 const float2* w_e, const float2* w_h, const RegionFlush* regions,
                                 float* acc_re, float* acc_im, float* cmp_re, float* cmp_im, const int* base_dev) {
  extern __shared__ float2 sw[];  // [cnt][n_freq]
  if (base_dev) n_base += __ldg(base_dev);
  const RegionFlush rg = regions[blockIdx.y];
  const float2* w = rg.is_h ? w_h : w_e;
  for (int x = threadIdx.x; x < cnt * n_freq; x += blockDim.x) {
    sw[x] = w[static_cast<int64_t>(n_base) * n_freq + x];
  }
  __syncthreads();
  for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < rg.count;
       p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t slot = rg.base + p;
    float s[64];
#pragma unroll 8
    for (int m = 0; m < cnt; ++m) s[m] = samples[static_cast<int64_t>(m) * n_samples + slot];
    for (int f = 0; f < n_freq; ++f) {
      float re = 0.0f, im = 0.0f;
#pragma unroll 8
      for (int m = 0; m < cnt; ++m) {
        const float2 ww = sw[m * n_freq + f];
        re = fmaf(s[m], ww.x, re);
        im = fmaf(s[m], ww.y, im);
      }
      const int64_t a = static_cast<int64_t>(f) * n_samples + slot;
      {
        const float y = re - cmp_re[a];
        const float t = acc_re[a] + y;
        cmp_re[a] = (t - acc_re[a]) - y;
        acc_re[a] = t;
      }
      {
        const float y = im - cmp_im[a];
        const float t = acc_im[a] + y;
        cmp_im[a] = (t - acc_im[a]) - y;
        acc_im[a] = t;
      }
    }
  }
}

}  // namespace

struct DevBuf {
  float* ptr = nullptr;
  size_t n = 0;
};

constexpr int kDefaultVariant = 2;
// Planes ahead of the x march whose field rows the scalar step kernels
// prefetch into L2 (0 disables).
constexpr int kDefaultPrefetch = 2;

constexpr int kMaxVariant = 10;
// The row-tile kernel (tile_kernel.cu): the default launch of FP32 engines
// without wrapped faces.
constexpr int kTileVariant = 10;
constexpr int kTileMaxChunk = 63;  // planes per chunk of the row-tile kernel (chunk + halo plane <= 64)

// z cells per lane of a launch variant (1 for the scalar kernels 1-4).
int variant_v(int variant) {
  switch (variant) {
    case 5: case 9: return 4;
    case 6: case 7: case 8: return 2;
    default: return 1;
  }
}

// Launcher of a z-vectorised variant (5: 4 cells per lane, direct loads;
// 6: 2 cells, direct; 7 / 8: 2 cells, 4- / 3-plane cp.async ring; 9: 4 cells,
// 3-plane ring).
VecLauncher vec_launcher(int variant) {
  switch (variant) {
    case 5: return launch_vec_v4;
    case 6: return launch_vec_v2;
    case 7: return launch_vec_r2d4;
    case 8: return launch_vec_r2d3;
    case 9: return launch_vec_r4d3;
    default: return nullptr;
  }
}

struct PoleHost {
  PoleTerm t;
  float *drive = nullptr, *inv_eps = nullptr, *pol = nullptr, *cur = nullptr;
  int64_t count = 0;  // cells of the box
  int64_t rows = 0;   // (i, j) rows of the box
  int nk = 0, nkk = 0, koff = 0;  // z cells, padded z pitch, offset of k0 in a padded row
  int64_t state_floats = 0;       // size of pol / cur in 4-byte words
};

struct AuxLine {
  int ne = 0, n_steps = 0;
  float* e_hist = nullptr;
  float* h_hist = nullptr;
};

// A checkpoint slot: one allocation holding every state array back to back.
struct Checkpoint {
  float* store = nullptr;
  std::vector<float*> bufs;  // views into store, in state_buffers order
  bool valid = false;
};

// Adjoint state (reverse-time pass): adjoint fields and CPML psi in the
// forward layouts, monitor seeds, design boxes with their replayed E history.
// Time-shifted patches (witwin/maxwell/fdtd/cuda/kernels/sources.cu:173-221):
// comp gets scale[cell] * w(n dt + t_offset - delay[cell]) at step n.  Each one
// is an ordinary injection term whose coefficient array the shift kernel
// rewrites before every step, with a signal table of ones.
constexpr int kMaxShifted = 8;
struct ShiftedHost {
  float* coeff;  // the injection term's coefficient array
  const float* scale;
  const float* delay;
  int64_t cells;
  double t_offset, wdelay;
  int kind;  // 0 CW, 1 Gaussian pulse
  float omega, inv_sigma, amplitude, phase;
};

struct ShiftedLaunch {
  int count;
  float* coeff[kMaxShifted];
  const float* scale[kMaxShifted];
  const float* delay[kMaxShifted];
  int64_t cells[kMaxShifted];
  float tau0[kMaxShifted];  // n dt + t_offset (- the pulse centre), formed in FP64
  int kind[kMaxShifted];
  float omega[kMaxShifted], inv_sigma[kMaxShifted], amplitude[kMaxShifted], phase[kMaxShifted];
};

// blockIdx.y picks the term; CW: A cos(omega tau + phase); Gaussian pulse:
// A exp(-(tau inv_sigma)^2 / 2) cos(omega tau + phase) (waveforms.py:83-103).
__global__ void __launch_bounds__(256) shifted_patch_kernel(const __grid_constant__ ShiftedLaunch s) {
  const int t = blockIdx.y;
  const int64_t cells = s.cells[t];
  for (int64_t c = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; c < cells;
       c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float tau = s.tau0[t] - __ldg(s.delay[t] + c);
    float w = s.amplitude[t] * cosf(s.omega[t] * tau + s.phase[t]);
    if (s.kind[t] == 1) {
      const float a = tau * s.inv_sigma[t];
      w *= expf(-0.5f * a * a);
    }
    s.coeff[t][c] = __ldg(s.scale[t] + c) * w;
  }
}

// Instantaneous nonlinear media (witwin/maxwell/fdtd/cuda/kernels/
// dispersive.cu:165-400, called before the E update, runtime/stepping.py:
// 1794-1796): before every step the E coefficients of the nonlinear cells are
// recomposed from E^n collocated onto the cell's Yee edge (the other two
// components 4-point averaged, indices clamped to their arrays):
//   Kerr only:  curl = dt / max(eps + eps0 chi3 |E|^2, 1e-12 eps0) * decay
//   general:    eps_eff = eps + eps0 (chi2 E_own + chi3 |E|^2) (same floor),
//               sigma = max(sigma_s + tpa |E|^2, 0), half = sigma dt / (2 eps_eff),
//               decay = ext (1 - half) / (1 + half), curl = ext dt / eps_eff / (1 + half).
// The work list holds only cells with a nonzero chi2, chi3 or TPA channel: on
// every other cell the formula is constant and the host stores its value once.
struct NonlinearLaunch {
  const int4* cells;  // i, j, k, component
  const float* prm;   // 6 x n (SoA): eps, decay (Kerr) or external decay, sigma_s, chi2, chi3, tpa
  int64_t n;
  const float* E[3];  // E^n
  float* decay[3];
  float* curl[3];
  int NX, NY, NZ, P;
  float dt, eps0;
  int general;
};

// E component c at (i, j, k), each index clamped into c's Yee extent
__device__ __forceinline__ float nl_sample(const NonlinearLaunch& a, int c, int i, int j, int k) {
  const int ex = c == 0 ? a.NX - 1 : a.NX, ey = c == 1 ? a.NY - 1 : a.NY, ez = c == 2 ? a.NZ - 1 : a.NZ;
  i = min(max(i, 0), ex - 1);
  j = min(max(j, 0), ey - 1);
  k = min(max(k, 0), ez - 1);
  return __ldg(a.E[c] + (static_cast<int64_t>(i) * a.NY + j) * a.P + k);
}

__global__ void __launch_bounds__(256) nonlinear_kernel(const __grid_constant__ NonlinearLaunch a) {
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < a.n;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int4 q = __ldg(a.cells + t);
    const int i = q.x, j = q.y, k = q.z, c = q.w;
    float e[3];
    e[c] = nl_sample(a, c, i, j, k);
    if (c == 0) {
      e[1] = 0.25f * (nl_sample(a, 1, i, j - 1, k) + nl_sample(a, 1, i, j, k) + nl_sample(a, 1, i + 1, j - 1, k) +
                      nl_sample(a, 1, i + 1, j, k));
      e[2] = 0.25f * (nl_sample(a, 2, i, j, k - 1) + nl_sample(a, 2, i, j, k) + nl_sample(a, 2, i + 1, j, k - 1) +
                      nl_sample(a, 2, i + 1, j, k));
    } else if (c == 1) {
      e[0] = 0.25f * (nl_sample(a, 0, i - 1, j, k) + nl_sample(a, 0, i, j, k) + nl_sample(a, 0, i - 1, j + 1, k) +
                      nl_sample(a, 0, i, j + 1, k));
      e[2] = 0.25f * (nl_sample(a, 2, i, j, k - 1) + nl_sample(a, 2, i, j, k) + nl_sample(a, 2, i, j + 1, k - 1) +
                      nl_sample(a, 2, i, j + 1, k));
    } else {
      e[0] = 0.25f * (nl_sample(a, 0, i - 1, j, k) + nl_sample(a, 0, i, j, k) + nl_sample(a, 0, i - 1, j, k + 1) +
                      nl_sample(a, 0, i, j, k + 1));
      e[1] = 0.25f * (nl_sample(a, 1, i, j - 1, k) + nl_sample(a, 1, i, j, k) + nl_sample(a, 1, i, j - 1, k + 1) +
                      nl_sample(a, 1, i, j, k + 1));
    }
    const float fsq = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
    const float eps = __ldg(a.prm + t), dec = __ldg(a.prm + a.n + t);
    const float chi3 = __ldg(a.prm + 4 * a.n + t);
    const float floor_eps = 1.0e-12f * a.eps0;
    const int64_t o = (static_cast<int64_t>(i) * a.NY + j) * a.P + k;
    if (!a.general) {
      float eff = eps + a.eps0 * chi3 * fsq;
      if (eff < floor_eps) eff = floor_eps;
      a.curl[c][o] = (a.dt / eff) * dec;
    } else {
      const float sig_s = __ldg(a.prm + 2 * a.n + t), chi2 = __ldg(a.prm + 3 * a.n + t);
      const float tpa = __ldg(a.prm + 5 * a.n + t);
      float eff = eps + a.eps0 * (chi2 * e[c] + chi3 * fsq);
      if (eff < floor_eps) eff = floor_eps;
      float sigma = sig_s + tpa * fsq;
      if (sigma < 0.0f) sigma = 0.0f;
      const float half = 0.5f * sigma * a.dt / eff;
      const float inv_denom = 1.0f / (1.0f + half);
      a.decay[c][o] = dec * (1.0f - half) * inv_denom;
      a.curl[c][o] = dec * (a.dt / eff) * inv_denom;
    }
  }
}

// Off-diagonal anisotropic coupling (witwin/maxwell/fdtd/cuda/kernels/
// aniso.cu:26-580, applied right after the E update, runtime/stepping.py:
// 1808-1811): after the step kernel, every E cell of an anisotropic box gets
//   E_c += (coeff_a <curlH_a> + coeff_b <curlH_b>) / 4
// from the new H, <curlH_d> the sum of curl(H)_d (backward differences) over
// the four d-edges around the cell; a sample whose stencil leaves the grid is
// skipped.  Boxes stay clear of the CPML slabs and of wrapped faces (the host
// checks), so plain differences are exact there.
constexpr int kMaxAniso = 3;
struct AnisoHost {
  int comp;
  int box[6];
  float* ca;  // box-dense coefficients of the two off-axis curl components (lower axis first)
  float* cb;
};

struct AnisoLaunch {
  int count;
  int comp[kMaxAniso];
  int box[kMaxAniso][6];
  const float* ca[kMaxAniso];
  const float* cb[kMaxAniso];
  const float* H[3];  // H^{n+1/2} (padded)
  float* E[3];        // E^{n+1} (padded)
  const float* inv[3];
  float inv_u[3];
  int uniform;
  int n[3];
  int NY, P;
  int pec_faces;  // PEC faces (bit f) whose tangential E stays zero (scenes without TFSF)
};

__device__ __forceinline__ float an_h(const AnisoLaunch& a, int c, int i, int j, int k) {
  return __ldg(a.H[c] + (static_cast<int64_t>(i) * a.NY + j) * a.P + k);
}

__device__ __forceinline__ float an_inv(const AnisoLaunch& a, int axis, int idx) {
  return a.uniform ? a.inv_u[axis] : __ldg(a.inv[axis] + idx);
}

// curl(H)_d at the d-edge s (non-periodic axes): false when the stencil leaves the grid
__device__ __forceinline__ bool an_curl(const AnisoLaunch& a, int d, const int* s, float& value) {
  if (s[d] < 0 || s[d] > a.n[d] - 2) return false;
  const int x = d == 0 ? 1 : 0, y = d == 2 ? 1 : 2;  // derivative axes, lower first
  if (s[x] < 1 || s[x] > a.n[x] - 2 || s[y] < 1 || s[y] > a.n[y] - 2) return false;
  if (d == 0) {  // dHz/dy - dHy/dz
    value = (an_h(a, 2, s[0], s[1], s[2]) - an_h(a, 2, s[0], s[1] - 1, s[2])) * an_inv(a, 1, s[1]) -
            (an_h(a, 1, s[0], s[1], s[2]) - an_h(a, 1, s[0], s[1], s[2] - 1)) * an_inv(a, 2, s[2]);
  } else if (d == 1) {  // dHx/dz - dHz/dx
    value = (an_h(a, 0, s[0], s[1], s[2]) - an_h(a, 0, s[0], s[1], s[2] - 1)) * an_inv(a, 2, s[2]) -
            (an_h(a, 2, s[0], s[1], s[2]) - an_h(a, 2, s[0] - 1, s[1], s[2])) * an_inv(a, 0, s[0]);
  } else {  // dHy/dx - dHx/dy
    value = (an_h(a, 1, s[0], s[1], s[2]) - an_h(a, 1, s[0] - 1, s[1], s[2])) * an_inv(a, 0, s[0]) -
            (an_h(a, 0, s[0], s[1], s[2]) - an_h(a, 0, s[0], s[1] - 1, s[2])) * an_inv(a, 1, s[1]);
  }
  return true;
}

__global__ void __launch_bounds__(256) aniso_pass_kernel(const __grid_constant__ AnisoLaunch a) {
  const int t = blockIdx.y;
  const int comp = a.comp[t];
  const int* b = a.box[t];
  const int n1 = b[3] - b[2], n2 = b[5] - b[4];
  const int64_t cells = static_cast<int64_t>(b[1] - b[0]) * n1 * n2;
  const int da = comp == 0 ? 1 : 0, db = comp == 2 ? 1 : 2;
  for (int64_t c = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; c < cells;
       c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float c_a = __ldg(a.ca[t] + c), c_b = __ldg(a.cb[t] + c);
    if (c_a == 0.0f && c_b == 0.0f) continue;
    const int k = b[4] + static_cast<int>(c % n2);
    const int j = b[2] + static_cast<int>((c / n2) % n1);
    const int i = b[0] + static_cast<int>(c / (static_cast<int64_t>(n1) * n2));
    const int pos[3] = {i, j, k};
    if (a.pec_faces) {
      // tangential E on a PEC face stays zero
      bool face = false;
      for (int ax = 0; ax < 3; ++ax) {
        if (ax == comp) continue;
        face = face || (pos[ax] == 0 && (a.pec_faces >> (2 * ax) & 1)) ||
               (pos[ax] == a.n[ax] - 1 && (a.pec_faces >> (2 * ax + 1) & 1));
      }
      if (face) continue;
    }
    float acc[2] = {0.0f, 0.0f};
    for (int q = 0; q < 2; ++q) {
      const int d = q == 0 ? da : db;
      if ((q == 0 ? c_a : c_b) == 0.0f) continue;
      // own axis offsets {0, +1}, curl axis {-1, 0}; the lower axis outermost
      const int outer = min(comp, d), inner = max(comp, d);
      for (int u = 0; u < 2; ++u)
        for (int v = 0; v < 2; ++v) {
          int s[3] = {i, j, k};
          s[outer] += outer == comp ? u : u - 1;
          s[inner] += inner == comp ? v : v - 1;
          float sample;
          if (an_curl(a, d, s, sample)) acc[q] += sample;
        }
    }
    float* e = a.E[comp] + (static_cast<int64_t>(i) * a.NY + j) * a.P + k;
    *e += 0.25f * (c_a * acc[0] + c_b * acc[1]);
  }
}

struct AdjointHost {
  bool ready = false;
  AdjParams q{};
  std::vector<float*> bufs;  // everything allocated for the adjoint
  std::vector<float*> gpol_host, gcur_host;  // adjoint pole state per pole id
  int max_segment = 0;
  int replay_n0 = -1, replay_n1 = -1;
  // Pipelined checkpoint replay (fdtd_engine_backward_replay): a second design
  // history per box, and the stream and events on which the reverse steps of
  // one segment run while the engine stream replays the segment before it.
  float* hist2[3] = {nullptr, nullptr, nullptr};
  cudaStream_t rev = nullptr;
  cudaEvent_t ev_rep[2] = {nullptr, nullptr}, ev_rev[2] = {nullptr, nullptr};
};

struct fdtd_engine {
  fdtd_grid_desc desc{};
  cudaStream_t stream = nullptr;
  int NX = 0, NY = 0, NZ = 0, P = 0, SZ = 0;
  int zlo4 = 0, zhs4 = 0;  // z-slab psi row segments (StepParams::zlo4 / zhs4)
  // Field storage (kStore*) and per-component scales (stored * scale = value);
  // scales_set: the caller fixed the scales (else finalize estimates them).
  int storage = 0;
  float fscale[6] = {1, 1, 1, 1, 1, 1};
  bool scales_set = false;
  // Graph-captured step blocks (fdtd_batch_*): while graph_base is set the
  // launches carry step indices relative to graph_n0 and read the block's base
  // step from d_base.
  int* d_base = nullptr;
  bool graph_base = false;
  int graph_n0 = 0;
  // Periodic / Bloch faces (x, y): the step kernel defers the E cells on them
  // to the wrap kernel.  bloch: some face is Bloch (complex field, stepped as
  // the real channel or imaginary channel of an fdtd_bloch pair); in_pair: the
  // pair runs the wrap kernel and the monitor gather of this engine.
  bool wrap = false;
  bool pmc = false;  // some face is PMC: the scalar warp kernels (launch variants 1-3) only
  // Instantaneous nonlinear E cells (fdtd_engine_set_nonlinear): host lists
  // until finalize, then one device work list over the three components.
  std::vector<int> nl_cells_h;     // i, j, k, component per cell
  std::vector<float> nl_prm_h[6];  // NonlinearLaunch::prm channels
  int nl_general = -1;             // -1: no nonlinear cells; 0: Kerr (curl only); 1: general (decay and curl)
  float nl_eps0 = 0.0f;
  int64_t nl_n = 0;
  int4* d_nl_cells = nullptr;
  float* d_nl_prm = nullptr;
  int nl_lo[3] = {0, 0, 0}, nl_hi[3] = {0, 0, 0};
  std::vector<AnisoHost> aniso;  // full-anisotropy boxes (fdtd_engine_set_full_aniso)
  bool replay_region = true;     // fdtd_engine_set_replay_region
  bool bloch = false;
  bool in_pair = false;
  int64_t plane = 0, vol = 0;
  int TY = 0, CX = 0;
  // Fused kernel: 1..3 = register-prefetch warp kernel with a register budget
  // of up to 128 / 64 / 85 per thread; 4 = TMA-fed kernel; 5..9 = z-vectorised
  // warp kernels (vec_launcher); 10 = row-tile kernel (shared-memory row
  // exchange, tile_kernel.cu).
  int variant = kDefaultVariant;
  int pf_dist = kDefaultPrefetch;
  int cur = 0;  // index of the buffer holding the current state
  float* E[2][3] = {};
  float* H[2][3] = {};
  float* psiE[3][2] = {};
  float* psiH[2][3][2] = {};
  int64_t psi_count[3] = {0, 0, 0};  // per axis element count of one slab array
  float* ecoef[6][2] = {};           // [comp][decay, curl] padded arrays (nullptr = uniform)
  float ucoef[6][2] = {};
  float* inv_e[3] = {};
  float* inv_h[3] = {};
  float* eb[3] = {};
  float* ec[3] = {};
  float* eik[3] = {};
  float* hb[3] = {};
  float* hc[3] = {};
  float* hik[3] = {};
  bool cpml = false;
  bool uniform_grid = false;
  float inv_e_u[3] = {0, 0, 0}, inv_h_u[3] = {0, 0, 0};
  std::vector<InjectionTerm> terms;
  std::vector<ShiftedHost> shifted;
  std::vector<float*> owned;
  std::vector<PoleHost> poles;
  std::vector<SampleRegion> regions;
  std::vector<AuxLine> lines;
  int64_t n_samples = 0, n_samples_e = 0;
  // device tables
  InjectionTerm* d_terms = nullptr;
  PoleTerm* d_poles = nullptr;
  SampleRegion* d_regions = nullptr;
  BoxIndex term_ix[2] = {};
  BoxIndex region_ix[2] = {};
  int n_terms_ph[2] = {0, 0};
  int n_regions_ph[2] = {0, 0};
  int* d_pole_ptr = nullptr;
  int* d_pole_ids = nullptr;
  // ADE pass work list (int4 tiles over the union of the pole boxes) and its switch
  const int* d_ade_tiles = nullptr;
  int n_ade_tiles = 0;
  bool ade_pass = true;
  AdeParams ade{};
  const int* d_plane_bits = nullptr;
  unsigned char* d_warp_class = nullptr;  // sized for chunk length 1 (the largest table)
  TmaMaps maps[2] = {};                    // tensor maps of E[cur], H[cur] for cur = 0, 1
  bool tma_ready = false;
  int* d_status = nullptr;                 // timeout flag written by bounded waits
  int wait_limit = 1 << 20;                // polling rounds of a bounded pipeline wait
  int class_key = 0;                      // (chunk length, lane width) the table was built for (0 = stale)
  std::vector<int*> index_bufs;
  RegionFlush* d_flush = nullptr;
  int n_flush = 0;
  int64_t max_region = 0;
  float* samples = nullptr;
  int M = 32;
  int pending = 0;
  bool range_flush = true;  // flush the buffered monitor samples at the end of every step range
  int pending_base = 0;
  // DFT
  int n_freq = 0, dft_steps = 0;
  float2* w_e = nullptr;
  float2* w_h = nullptr;
  float *acc_re = nullptr, *acc_im = nullptr, *cmp_re = nullptr, *cmp_im = nullptr;
  bool finalized = false;
  int64_t launches = 0;
  float last_ms = 0.0f;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // Inside step_range the monitor gather and the DFT flush run on a second
  // (high-priority) stream, so they overlap the next step's kernels: the
  // gather of step n reads the buffer set step n wrote, which only step n + 2
  // overwrites (ping-pong), so step n + 2 waits for ev_gat[set] and nothing
  // else waits.  The flush stays ordered behind the gathers on the same stream,
  // and the streams are joined before step_range returns.
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_gat[2] = {nullptr, nullptr};
  bool gat_pending[2] = {false, false};
  bool async_gather = false;
  std::vector<Checkpoint> checkpoints;
  AdjointHost adj;
};

namespace {

int dev_alloc(fdtd_engine* h, float** out, size_t n) {
  if (n == 0) {
    *out = nullptr;
    return 0;
  }
  CUDA_TRY(cudaMalloc(out, n * sizeof(float)));
  CUDA_TRY(cudaMemsetAsync(*out, 0, n * sizeof(float), h->stream));
  h->owned.push_back(*out);
  return 0;
}

int dev_copy(fdtd_engine* h, float** out, const float* src, size_t n) {
  int rc = dev_alloc(h, out, n);
  if (rc) return rc;
  if (n) CUDA_TRY(cudaMemcpyAsync(*out, src, n * sizeof(float), cudaMemcpyDefault, h->stream));
  return 0;
}

// Size of one field array in 4-byte words (two reduced values per word).
int64_t field_floats(const fdtd_engine* h) { return h->storage == kStoreF32 ? h->vol : (h->vol + 1) / 2; }

int64_t slab_elems(const fdtd_engine* h, int axis) {
  const int L = h->desc.pml_lo[axis] + h->desc.pml_hi[axis];
  if (L == 0) return 0;
  if (axis == 0) return static_cast<int64_t>(L) * h->NY * h->P;
  if (axis == 1) return static_cast<int64_t>(h->NX) * L * h->P;
  return static_cast<int64_t>(h->NX) * h->NY * h->SZ;
}

bool box_ok(const fdtd_engine* h, int comp, const int* box) {
  int ext[3];
  comp_extent(comp, h->NX, h->NY, h->NZ, ext);
  for (int a = 0; a < 3; ++a) {
    if (box[2 * a] < 0 || box[2 * a + 1] > ext[a] || box[2 * a] >= box[2 * a + 1]) return false;
  }
  return true;
}

// Values of n pseudo-randomly chosen in-extent cells of a padded array.
__global__ void coef_sample_kernel(const float* a, int NY, int P, int e0, int e1, int e2, int n, float* out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n) return;
  uint64_t z = 0x9E3779B97F4A7C15ull * (static_cast<uint64_t>(x) + 1);
  z ^= z >> 31;
  z *= 0xBF58476D1CE4E5B9ull;
  z ^= z >> 27;
  const uint64_t cells = static_cast<uint64_t>(e0) * e1 * e2;
  const uint64_t c = z % cells;
  const int k = static_cast<int>(c % e2);
  const int j = static_cast<int>((c / e2) % e1);
  const int i = static_cast<int>(c / (static_cast<uint64_t>(e2) * e1));
  out[x] = a[(static_cast<int64_t>(i) * NY + j) * P + k];
}

int background_value(fdtd_engine* h, int comp, const float* arr, float* out) {
  constexpr int kSamples = 4096;
  int ext[3];
  comp_extent(comp, h->NX, h->NY, h->NZ, ext);
  float* d = nullptr;
  CUDA_TRY(cudaMalloc(&d, sizeof(float) * kSamples));
  coef_sample_kernel<<<kSamples / 256, 256, 0, h->stream>>>(arr, h->NY, h->P, ext[0], ext[1], ext[2], kSamples, d);
  std::vector<float> v(kSamples);
  cudaError_t err = cudaGetLastError();
  if (err == cudaSuccess) err = cudaMemcpyAsync(v.data(), d, sizeof(float) * kSamples, cudaMemcpyDeviceToHost, h->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(h->stream);
  cudaFree(d);
  if (err != cudaSuccess) return cuda_fail(err, "coefficient background sample");
  std::sort(v.begin(), v.end());
  float best = v[0];
  int best_n = 0;
  for (int a = 0; a < kSamples;) {
    int b = a;
    while (b < kSamples && v[b] == v[a]) ++b;
    if (b - a > best_n) {
      best_n = b - a;
      best = v[a];
    }
    a = b;
  }
  *out = best;
  return 0;
}

int z_blocks(const fdtd_engine* h);

void fill_params(const fdtd_engine* h, StepParams& p) {
  std::memset(&p, 0, sizeof(p));
  p.NX = h->NX;
  p.NY = h->NY;
  p.NZ = h->NZ;
  p.P = h->P;
  p.SZ = h->SZ;
  p.storage = h->storage;
  p.uniform_grid = h->uniform_grid ? 1 : 0;
  p.step_base = h->graph_base ? h->d_base : nullptr;
  for (int c = 0; c < 6; ++c) {
    p.fscale[c] = h->fscale[c];
    p.finv[c] = 1.0f / h->fscale[c];
  }
  p.zlo4 = h->zlo4;
  p.zhs4 = h->zhs4;
  p.TY = h->TY;
  p.CX = h->CX;
  p.pf_dist = h->pf_dist;
  p.Q = h->P / 4;
  p.ROWS = 1;
  const int src = h->cur, dst = 1 - h->cur;
  for (int c = 0; c < 3; ++c) {
    p.Ein[c] = h->E[src][c];
    p.Eout[c] = h->E[dst][c];
    p.Hin[c] = h->H[src][c];
    p.Hout[c] = h->H[dst][c];
    p.edecay[c] = h->ecoef[c][0];
    p.ecurl[c] = h->ecoef[c][1];
    p.edecay_u[c] = h->ucoef[c][0];
    p.ecurl_u[c] = h->ucoef[c][1];
    p.hdecay[c] = h->ecoef[3 + c][0];
    p.hcurl[c] = h->ecoef[3 + c][1];
    p.hdecay_u[c] = h->ucoef[3 + c][0];
    p.hcurl_u[c] = h->ucoef[3 + c][1];
    p.inv_e[c] = h->inv_e[c];
    p.inv_h[c] = h->inv_h[c];
    p.inv_e_u[c] = h->inv_e_u[c];
    p.inv_h_u[c] = h->inv_h_u[c];
    p.eb[c] = h->eb[c];
    p.ec[c] = h->ec[c];
    p.eik[c] = h->eik[c];
    p.hb[c] = h->hb[c];
    p.hc[c] = h->hc[c];
    p.hik[c] = h->hik[c];
    p.slab_lo[c] = h->desc.pml_lo[c];
    p.slab_hi[c] = h->desc.pml_hi[c];
    for (int w = 0; w < 2; ++w) {
      p.psiE[c][w] = h->psiE[c][w];
      p.psiHin[c][w] = h->psiH[src][c][w];
      p.psiHout[c][w] = h->psiH[dst][c][w];
    }
  }
  for (int f = 0; f < 6; ++f) p.bnd[f] = h->desc.boundary[f];
  p.cpml = h->cpml ? 1 : 0;
  p.terms = h->d_terms;
  p.poles = h->d_poles;
  p.pole_plane_ptr = h->d_pole_ptr;
  p.pole_plane_ids = h->d_pole_ids;
  p.n_poles = static_cast<int>(h->poles.size());
  p.regions = h->d_regions;
  p.plane_bits = reinterpret_cast<const unsigned*>(h->d_plane_bits);
  p.warp_class = h->d_warp_class;
  p.status = h->d_status;
  p.wait_limit = h->wait_limit;
  p.pmc = 0;
  for (int f = 0; f < 6; ++f)
    if (h->desc.boundary[f] == FDTD_BND_PMC) p.pmc |= 1 << f;
  p.pec_clamp = h->lines.empty() ? 1 : 0;
  p.n_kb = z_blocks(h);
  for (int a = 0; a < 3; ++a) {
    p.nl_lo[a] = h->nl_lo[a];
    p.nl_hi[a] = h->nl_hi[a];
  }
  for (int ph = 0; ph < 2; ++ph) {
    p.term_index[ph] = h->term_ix[ph];
    p.n_terms[ph] = h->n_terms_ph[ph];
    p.region_index[ph] = h->region_ix[ph];
    p.n_regions[ph] = h->n_regions_ph[ph];
  }
  p.samples = h->samples;
  p.n_samples = h->n_samples;
  p.sample_block = h->M;
}

constexpr int kWarpRows = 8;   // warps (y rows) per CTA of the step kernel
constexpr int kWarpOut = 30;   // z cells produced per warp

int z_blocks(const fdtd_engine* h) {
  const int V = variant_v(h->variant);
  const int span = V == 1 ? kWarpOut : 31 * V;
  return (h->NZ + span - 1) / span;
}

void default_tiles(fdtd_engine* h) {
  h->TY = 1;
  int CX = h->desc.chunk_planes;
  if (CX <= 0 && variant_v(h->variant) > 1) {
    // Vectorised kernel (one or two 256-thread CTAs per SM): about six waves
    // of warps, chunks of at least eight planes.
    const int64_t cols = static_cast<int64_t>((h->NY + kWarpRows - 1) / kWarpRows) * z_blocks(h);
    const int per_sm = variant_v(h->variant) == 4 ? 1 : 2;  // CTAs per SM (registers / ring)
    const int64_t want_chunks = std::max<int64_t>(1, (148 * per_sm * 6 + cols - 1) / cols);
    CX = static_cast<int>(std::max<int64_t>(8, (h->NX + want_chunks - 1) / want_chunks));
  }
  if (CX <= 0 && h->variant == kTileVariant) {
    // Row-tile kernel (three 320-thread CTAs per SM): about thirteen waves of
    // CTAs; 12-13 plane chunks measured fastest at 256^3 (chunks of 29 planes
    // were 8 % slower: fewer CTAs to fill the last waves), so chunks stay short
    // down to 12 planes.
    const int64_t cols = static_cast<int64_t>((h->NY + kWarpRows - 1) / kWarpRows) * ((h->NZ + kWarpOut - 1) / kWarpOut);
    const int64_t want_chunks = std::max<int64_t>(1, (148 * 3 * 13 + cols - 1) / cols);
    CX = static_cast<int>(std::min<int64_t>(kTileMaxChunk, std::max<int64_t>(12, (h->NX + want_chunks - 1) / want_chunks)));
  }
  if (CX <= 0) {
    // Split x into chunks until the grid holds about ten waves of the
    // 64-register variant (four 256-thread CTAs per SM on 148 SMs).  Shorter
    // chunks recompute one halo plane each, which stays cheaper than idle SMs
    // down to four planes.
    const int64_t cols = static_cast<int64_t>((h->NY + kWarpRows - 1) / kWarpRows) * ((h->NZ + kWarpOut - 1) / kWarpOut);
    const int64_t want_chunks = std::max<int64_t>(1, (148 * 4 * 10 + cols - 1) / cols);
    CX = static_cast<int>(std::max<int64_t>(4, (h->NX + want_chunks - 1) / want_chunks));
  }
  h->CX = CX;
}

dim3 step_grid(const fdtd_engine* h) {
  return dim3((h->NY + kWarpRows - 1) / kWarpRows, z_blocks(h), (h->NX + h->CX - 1) / h->CX);
}

// Read (and clear) the device status word after the stream has drained.
int check_status(fdtd_engine* h) {
  int st = 0;
  CUDA_TRY(cudaMemcpyAsync(&st, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (st != 0) {
    CUDA_TRY(cudaMemsetAsync(h->d_status, 0, sizeof(int), h->stream));
    return fail(FDTD_ERR_TIMEOUT, "a bounded wait in the step kernel ran out");
  }
  return 0;
}

int launch_wrap_single(fdtd_engine* h, int n);
int launch_gather(fdtd_engine* h, int slot);

bool has_coef(const fdtd_engine* h) {
  for (int c = 0; c < 6; ++c)
    if (h->ecoef[c][0] || h->ecoef[c][1]) return true;
  return false;
}

// Build the per-warp class table for the current launch shape if it is stale.
int ensure_classified(fdtd_engine* h, const StepParams& p) {
  const dim3 grid = step_grid(h);
  const int V = variant_v(h->variant);
  const int key = h->CX * 8 + V;
  if ((h->cpml || has_coef(h)) && h->class_key != key) {
    const int err = V == 1 ? launch_classify(p, static_cast<int>(grid.y), static_cast<int>(grid.z), h->d_warp_class, h->stream)
                           : launch_classify_vec(p, V, static_cast<int>(grid.y), static_cast<int>(grid.z), h->d_warp_class,
                                                 h->stream);
    if (err != 0) return cuda_fail(static_cast<cudaError_t>(err), "classify_kernel launch");
    h->class_key = key;
  }
  return 0;
}

// The poles run in the ADE pass after the step kernel (instead of inside it)
// on FP32 storage with the scalar step kernels and no wrapped face.
bool ade_pass_active(const fdtd_engine* h) {
  return h->ade_pass && h->n_ade_tiles > 0 && h->poles.size() <= static_cast<size_t>(kAdeMaxPoles) &&
         h->storage == kStoreF32 && !h->wrap && ((h->variant >= 1 && h->variant <= 3) || h->variant == kTileVariant);
}

// The row-tile kernel has no pole code: with poles that the ADE pass cannot
// take (more than its table holds, or the pass switched off) the 64-register
// warp kernel runs instead.
bool tile_runs(const fdtd_engine* h) {
  return h->variant == kTileVariant && h->storage == kStoreF32 && !h->wrap && !h->pmc && h->tma_ready &&
         (h->poles.empty() || ade_pass_active(h));
}

int launch_shifted(fdtd_engine* h, int n) {
  ShiftedLaunch s{};
  s.count = static_cast<int>(h->shifted.size());
  int64_t most = 0;
  for (int t = 0; t < s.count; ++t) {
    const ShiftedHost& x = h->shifted[t];
    s.coeff[t] = x.coeff;
    s.scale[t] = x.scale;
    s.delay[t] = x.delay;
    s.cells[t] = x.cells;
    s.tau0[t] = static_cast<float>(n * h->desc.dt + x.t_offset - (x.kind == 1 ? x.wdelay : 0.0));
    s.kind[t] = x.kind;
    s.omega[t] = x.omega;
    s.inv_sigma[t] = x.inv_sigma;
    s.amplitude[t] = x.amplitude;
    s.phase[t] = x.phase;
    most = std::max(most, x.cells);
  }
  const int gx = static_cast<int>(std::min<int64_t>((most + 255) / 256, 4 * 148));
  shifted_patch_kernel<<<dim3(gx, s.count), 256, 0, h->stream>>>(s);
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_fail(err, "shifted_patch_kernel launch");
  ++h->launches;
  return 0;
}

int launch_nonlinear(fdtd_engine* h) {
  NonlinearLaunch a{};
  a.cells = h->d_nl_cells;
  a.prm = h->d_nl_prm;
  a.n = h->nl_n;
  for (int c = 0; c < 3; ++c) {
    a.E[c] = h->E[h->cur][c];
    a.decay[c] = h->ecoef[c][0];
    a.curl[c] = h->ecoef[c][1];
  }
  a.NX = h->NX;
  a.NY = h->NY;
  a.NZ = h->NZ;
  a.P = h->P;
  a.dt = static_cast<float>(h->desc.dt);
  a.eps0 = h->nl_eps0;
  a.general = h->nl_general;
  const int gx = static_cast<int>(std::min<int64_t>((h->nl_n + 255) / 256, 8 * 148));
  nonlinear_kernel<<<gx, 256, 0, h->stream>>>(a);
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_fail(err, "nonlinear_kernel launch");
  ++h->launches;
  return 0;
}

int launch_aniso(fdtd_engine* h, const StepParams& p) {
  AnisoLaunch a{};
  a.count = static_cast<int>(h->aniso.size());
  int64_t most = 0;
  for (int t = 0; t < a.count; ++t) {
    const AnisoHost& x = h->aniso[t];
    a.comp[t] = x.comp;
    for (int q = 0; q < 6; ++q) a.box[t][q] = x.box[q];
    a.ca[t] = x.ca;
    a.cb[t] = x.cb;
    most = std::max<int64_t>(most, static_cast<int64_t>(x.box[1] - x.box[0]) * (x.box[3] - x.box[2]) *
                                       (x.box[5] - x.box[4]));
  }
  for (int c = 0; c < 3; ++c) {
    a.H[c] = p.Hout[c];
    a.E[c] = p.Eout[c];
    a.inv[c] = h->inv_e[c];
    a.inv_u[c] = h->inv_e_u[c];
  }
  a.uniform = h->uniform_grid ? 1 : 0;
  a.n[0] = h->NX;
  a.n[1] = h->NY;
  a.n[2] = h->NZ;
  a.NY = h->NY;
  a.P = h->P;
  a.pec_faces = 0;
  if (h->lines.empty())
    for (int f = 0; f < 6; ++f)
      if (h->desc.boundary[f] == FDTD_BND_PEC) a.pec_faces |= 1 << f;
  const int gx = static_cast<int>(std::min<int64_t>((most + 255) / 256, 4 * 148));
  aniso_pass_kernel<<<dim3(gx, a.count), 256, 0, h->stream>>>(a);
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_fail(err, "aniso_pass_kernel launch");
  ++h->launches;
  return 0;
}

// region: node box (x0, x1, y0, y1, z0, z1) to which the warp kernel's task
// grid is restricted (a sub-grid of whole row blocks, z blocks and chunks that
// covers it), or nullptr for the full step.  Only the scalar warp kernels take
// a region (region_ok); cells outside it keep stale values.
int launch_step(fdtd_engine* h, int n, int slot, const int* region = nullptr) {
  if (!h->shifted.empty()) {
    const int rc = launch_shifted(h, n);
    if (rc) return rc;
  }
  if (h->nl_n > 0) {
    const int rc = launch_nonlinear(h);
    if (rc) return rc;
  }
  StepParams p;
  fill_params(h, p);
  dim3 grid = step_grid(h);
  if (region) {
    const unsigned rb0 = static_cast<unsigned>(region[2] / kWarpRows), kb0 = static_cast<unsigned>(region[4] / kWarpOut);
    const unsigned ch0 = static_cast<unsigned>(region[0] / h->CX);
    const unsigned rb1 = std::min<unsigned>(grid.x, static_cast<unsigned>((region[3] + kWarpRows - 1) / kWarpRows));
    const unsigned kb1 = std::min<unsigned>(grid.y, static_cast<unsigned>((region[5] + kWarpOut - 1) / kWarpOut));
    const unsigned ch1 = std::min<unsigned>(grid.z, static_cast<unsigned>((region[1] + h->CX - 1) / h->CX));
    if (rb1 <= rb0 || kb1 <= kb0 || ch1 <= ch0) return fail(FDTD_ERR_INVALID_ARG, "empty step region");
    p.rb0 = static_cast<int>(rb0);
    p.kb0 = static_cast<int>(kb0);
    p.ch0 = static_cast<int>(ch0);
    grid = dim3(rb1 - rb0, kb1 - kb0, ch1 - ch0);
  }
  const bool ade_pass = ade_pass_active(h);
  bool coef = false;
  for (int c = 0; c < 6; ++c) coef = coef || h->ecoef[c][0] || h->ecoef[c][1];
  const int block = kWarpRows * 32;
  if (h->variant == 4 && !h->tma_ready)
    return fail(FDTD_ERR_UNSUPPORTED, "TMA step kernel unavailable (no tensor-map driver entry point)");
  {
    const int rc = ensure_classified(h, p);
    if (rc) return rc;
  }
  if (ade_pass) p.n_poles = 0;  // the step kernel skips the poles
  if (h->async_gather && h->gat_pending[1 - h->cur]) {
    // the set this step writes was read by the gather of two steps ago
    CUDA_TRY(cudaStreamWaitEvent(h->stream, h->ev_gat[1 - h->cur], 0));
    h->gat_pending[1 - h->cur] = false;
  }
  if (h->storage != kStoreF32) {
    const int err = launch_step_reduced(p, n, grid, h->cpml, coef, h->uniform_grid, h->stream);
    if (err != 0) return cuda_fail(static_cast<cudaError_t>(err), "warp_step_kernel_rs launch");
  } else if (!region && tile_runs(h)) {
    // the row-tile kernel, then (scenes with CPML) the warp kernel over the
    // CTAs that meet a slab, which the row-tile kernel leaves alone
    const int err = launch_tile_step(p, h->maps[h->cur], n, grid, h->cpml, coef, h->uniform_grid, h->stream);
    if (err != 0) return cuda_fail(static_cast<cudaError_t>(err), "tile_step_kernel launch");
    if (h->cpml) {
      ++h->launches;
      StepParams q = p;
      q.shell_only = 1;
#define FDTD_SHELL(COEF, UNI) warp_step_kernel<true, COEF, UNI, 4, false><<<grid, block, 0, h->stream>>>(q, n, slot)
      if (h->uniform_grid) {
        if (coef) FDTD_SHELL(true, true);
        else FDTD_SHELL(false, true);
      } else {
        if (coef) FDTD_SHELL(true, false);
        else FDTD_SHELL(false, false);
      }
#undef FDTD_SHELL
      const cudaError_t e2 = cudaGetLastError();
      if (e2 != cudaSuccess) return cuda_fail(e2, "warp_step_kernel (CPML shell) launch");
    }
  } else if (VecLauncher vl = region ? nullptr : vec_launcher(h->variant)) {
    const int err = vl(p, n, grid, h->cpml, coef, h->uniform_grid, h->stream);
    if (err != 0) return cuda_fail(static_cast<cudaError_t>(err), "vec_step_kernel launch");
  } else {
#define FDTD_LAUNCH(CPML, COEF, UNI)                                                                  \
  do {                                                                                           \
    if (h->variant == 4)                                                                          \
      tma_step_kernel<CPML, COEF, UNI><<<grid, kTmaThreads, tma_smem_bytes(), h->stream>>>(p, h->maps[h->cur], n); \
    else if ((h->variant == 2 || h->variant == kTileVariant) && ade_pass) warp_step_kernel<CPML, COEF, UNI, 4, false><<<grid, block, 0, h->stream>>>(p, n, slot); \
    else if (h->variant == 2 || h->variant == kTileVariant) warp_step_kernel<CPML, COEF, UNI, 4, true><<<grid, block, 0, h->stream>>>(p, n, slot); \
    else if (h->variant == 3 && ade_pass) warp_step_kernel<CPML, COEF, UNI, 3, false><<<grid, block, 0, h->stream>>>(p, n, slot); \
    else if (h->variant == 3) warp_step_kernel<CPML, COEF, UNI, 3, true><<<grid, block, 0, h->stream>>>(p, n, slot); \
    else warp_step_kernel<CPML, COEF, UNI, 1, true><<<grid, block, 0, h->stream>>>(p, n, slot);            \
  } while (0)
  if (h->uniform_grid) {
    if (h->cpml) {
      if (coef) FDTD_LAUNCH(true, true, true);
      else FDTD_LAUNCH(true, false, true);
    } else {
      if (coef) FDTD_LAUNCH(false, true, true);
      else FDTD_LAUNCH(false, false, true);
    }
  } else {
    if (h->cpml) {
      if (coef) FDTD_LAUNCH(true, true, false);
      else FDTD_LAUNCH(true, false, false);
    } else {
      if (coef) FDTD_LAUNCH(false, true, false);
      else FDTD_LAUNCH(false, false, false);
    }
  }
#undef FDTD_LAUNCH
  }
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_fail(err, "warp_step_kernel launch");
  ++h->launches;
  if (!h->aniso.empty()) {
    const int rc = launch_aniso(h, p);
    if (rc) return rc;
  }
  if (ade_pass) {
    for (int c = 0; c < 3; ++c) {
      h->ade.Ein[c] = p.Ein[c];
      h->ade.Eout[c] = p.Eout[c];
    }
    const int e2 = launch_ade_pass(h->ade, h->d_ade_tiles, h->n_ade_tiles, h->stream);
    if (e2 != 0) return cuda_fail(static_cast<cudaError_t>(e2), "ade_pass_kernel launch");
    ++h->launches;
  }
  h->cur = 1 - h->cur;
  if (h->in_pair) return 0;  // the Bloch pair runs the wrap kernel and the gather
  if (h->wrap) {
    const int rc = launch_wrap_single(h, n);
    if (rc) return rc;
  }
  return launch_gather(h, slot);
}

// Wrap kernel of a real periodic engine after its step (phase 1 on every axis).
int launch_wrap_single(fdtd_engine* h, int n) {
  StepParams p;
  fill_params(h, p);
  WrapFields f;
  for (int c = 0; c < 3; ++c) {
    f.eold[c] = h->E[1 - h->cur][c];
    f.enew[c] = h->E[h->cur][c];
    f.hnew[c] = h->H[h->cur][c];
  }
  const float pc[3] = {1.0f, 1.0f, 1.0f}, ps[3] = {0.0f, 0.0f, 0.0f};
  const int err = launch_wrap_fixup(p, nullptr, f, nullptr, pc, ps, n, h->stream, h->storage);
  if (err != 0) return cuda_fail(static_cast<cudaError_t>(err), "wrap_fixup_kernel launch");
  ++h->launches;
  return 0;
}

// Copy the monitor cells of the current state into sample slot `slot` (no-op for slot < 0).
int launch_gather(fdtd_engine* h, int slot) {
  cudaError_t err = cudaSuccess;
  if (h->n_flush > 0 && h->samples && slot >= 0) {
    FieldPtrs fields;
    for (int c = 0; c < 3; ++c) {
      fields.f[c] = h->E[h->cur][c];
      fields.f[3 + c] = h->H[h->cur][c];
    }
    fields.storage = h->storage;
    for (int c = 0; c < 6; ++c) fields.scale[c] = h->fscale[c];
    const int gx = static_cast<int>(std::min<int64_t>((h->max_region + 256 * kGatherIlp - 1) / (256 * kGatherIlp), 2048));
    cudaStream_t s = h->stream;
    if (h->async_gather) {
      CUDA_TRY(cudaEventRecord(h->ev_fork, h->stream));
      CUDA_TRY(cudaStreamWaitEvent(h->aux, h->ev_fork, 0));
      s = h->aux;
    }
    sample_gather_kernel<<<dim3(std::max(gx, 1), h->n_flush), 256, 0, s>>>(
        h->d_flush, fields, h->NY, h->P, h->samples, h->n_samples, slot);
    err = cudaGetLastError();
    if (err != cudaSuccess) return cuda_fail(err, "sample_gather_kernel launch");
    if (h->async_gather) {
      CUDA_TRY(cudaEventRecord(h->ev_gat[h->cur], h->aux));
      h->gat_pending[h->cur] = true;
    }
    ++h->launches;
  }
  return 0;
}

int flush_samples(fdtd_engine* h) {
  if (h->pending == 0) return 0;
  if (h->n_freq > 0 && h->n_flush > 0 && h->n_samples > 0) {
    if (h->pending_base + h->pending > h->dft_steps)
      return fail(FDTD_ERR_STATE, "DFT weight table shorter than the stepped range");
    const int threads = 256;
    const int gx = static_cast<int>(std::min<int64_t>((h->max_region + threads - 1) / threads, 4096));
    const dim3 grid(std::max(gx, 1), h->n_flush);
    const size_t smem = sizeof(float2) * static_cast<size_t>(h->pending) * h->n_freq;
    // In a captured step block the weights start at the block's device-side base step.
    const int n_base = h->graph_base ? h->pending_base - h->graph_n0 : h->pending_base;
    dft_flush_kernel<<<grid, threads, smem, h->async_gather ? h->aux : h->stream>>>(h->samples, h->n_samples, h->pending, n_base, h->n_freq,
                                                           h->w_e, h->w_h, h->d_flush, h->acc_re, h->acc_im,
                                                           h->cmp_re, h->cmp_im, h->graph_base ? h->d_base : nullptr);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return cuda_fail(err, "dft_flush_kernel launch");
    ++h->launches;
  }
  h->pending_base += h->pending;
  h->pending = 0;
  return 0;
}

template <typename T>
int upload_vec(fdtd_engine* h, T** dptr, const std::vector<T>& v) {
  if (*dptr) cudaFree(*dptr);
  *dptr = nullptr;
  if (v.empty()) return 0;
  CUDA_TRY(cudaMalloc(dptr, v.size() * sizeof(T)));
  CUDA_TRY(cudaMemcpyAsync(*dptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, h->stream));
  return 0;
}

// CSR over x planes of the boxes [i0, i1).
template <typename T>
void build_plane_csr(int NX, const std::vector<T>& items, std::vector<int>& ptr, std::vector<int>& ids) {
  ptr.assign(NX + 1, 0);
  for (const auto& t : items)
    for (int i = t.i0; i < t.i1; ++i) ptr[i + 1]++;
  for (int i = 0; i < NX; ++i) ptr[i + 1] += ptr[i];
  ids.assign(ptr[NX], 0);
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (size_t x = 0; x < items.size(); ++x)
    for (int i = items[x].i0; i < items[x].i1; ++i) ids[fill[i]++] = static_cast<int>(x);
}

int upload_ints(fdtd_engine* h, const std::vector<int>& v, const int** out) {
  int* d = nullptr;
  const size_t n = std::max<size_t>(v.size(), 1);
  CUDA_TRY(cudaMalloc(&d, n * sizeof(int)));
  CUDA_TRY(cudaMemsetAsync(d, 0, n * sizeof(int), h->stream));
  if (!v.empty()) CUDA_TRY(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  h->index_bufs.push_back(d);
  *out = d;
  return 0;
}

// Build the per-axis CSR index of the selected items (see BoxIndex): each item
// goes to the axis with the fewest planes / rows / float4 quads.
template <typename T>
int build_box_index(fdtd_engine* h, const std::vector<T>& items, const std::vector<int>& select, BoxIndex& out) {
  const int dims[3] = {h->NX, h->NY, h->P};
  std::vector<int> ptr[3], ids[3];
  std::vector<int> axis_of(select.size());
  for (size_t s = 0; s < select.size(); ++s) {
    const T& t = items[select[s]];
    const int ext[3] = {t.i1 - t.i0, t.j1 - t.j0, t.k1 - t.k0};
    int a = 0;
    if (ext[1] < ext[a]) a = 1;
    if (ext[2] < ext[a]) a = 2;
    axis_of[s] = a;
  }
  for (int a = 0; a < 3; ++a) {
    ptr[a].assign(dims[a] + 1, 0);
    for (size_t s = 0; s < select.size(); ++s) {
      if (axis_of[s] != a) continue;
      const T& t = items[select[s]];
      const int lo = a == 0 ? t.i0 : (a == 1 ? t.j0 : t.k0);
      const int hi = a == 0 ? t.i1 : (a == 1 ? t.j1 : t.k1);
      for (int c = lo; c < hi; ++c) ptr[a][c + 1]++;
    }
    for (int c = 0; c < dims[a]; ++c) ptr[a][c + 1] += ptr[a][c];
    ids[a].assign(ptr[a][dims[a]], 0);
    std::vector<int> fill(ptr[a].begin(), ptr[a].end() - 1);
    for (size_t s = 0; s < select.size(); ++s) {
      if (axis_of[s] != a) continue;
      const T& t = items[select[s]];
      const int lo = a == 0 ? t.i0 : (a == 1 ? t.j0 : t.k0);
      const int hi = a == 0 ? t.i1 : (a == 1 ? t.j1 : t.k1);
      for (int c = lo; c < hi; ++c) ids[a][fill[c]++] = select[s];
    }
    int rc = upload_ints(h, ptr[a], &out.ptr[a]);
    if (!rc) rc = upload_ints(h, ids[a], &out.ids[a]);
    if (rc) return rc;
  }
  return 0;
}

}  // namespace

extern "C" {

const char* fdtd_last_error(void) { return g_last_error.c_str(); }
const char* fdtd_version(void) { return "fdtd_b200 0.1.0 (sm_100a)"; }

int fdtd_engine_create(const fdtd_grid_desc* desc, void* stream, fdtd_engine** out) {
  if (!desc || !out) return fail(FDTD_ERR_INVALID_ARG, "null descriptor or output pointer");
  *out = nullptr;
  if (desc->nx < 3 || desc->ny < 3 || desc->nz < 3)
    return fail(FDTD_ERR_INVALID_ARG, "grid needs at least 3 nodes per axis");
  if (!(desc->dt > 0.0)) return fail(FDTD_ERR_INVALID_ARG, "dt must be positive");
  for (int f = 0; f < 6; ++f) {
    const int b = desc->boundary[f];
    const bool wrap = b == FDTD_BND_PERIODIC || b == FDTD_BND_BLOCH;
    if (b != FDTD_BND_NONE && b != FDTD_BND_PML && b != FDTD_BND_PEC && b != FDTD_BND_PMC && !wrap)
      return fail(FDTD_ERR_INVALID_ARG, "unknown boundary code");
    if (wrap && f >= 4) return fail(FDTD_ERR_UNSUPPORTED, "periodic and Bloch faces are supported on x and y");
    if (b == FDTD_BND_PMC && (f % 2 == 0 ? desc->pml_lo[f / 2] : desc->pml_hi[f / 2]) != 0)
      return fail(FDTD_ERR_INVALID_ARG, "a PMC face has no CPML slab");
  }
  {
    bool pmc = false, wraps = false;
    for (int f = 0; f < 6; ++f) {
      pmc = pmc || desc->boundary[f] == FDTD_BND_PMC;
      wraps = wraps || desc->boundary[f] == FDTD_BND_PERIODIC || desc->boundary[f] == FDTD_BND_BLOCH;
    }
    if (pmc && wraps) return fail(FDTD_ERR_UNSUPPORTED, "PMC faces with periodic or Bloch faces are not supported");
  }
  for (int a = 0; a < 2; ++a) {
    const int lo = desc->boundary[2 * a], hi = desc->boundary[2 * a + 1];
    const bool wlo = lo == FDTD_BND_PERIODIC || lo == FDTD_BND_BLOCH, whi = hi == FDTD_BND_PERIODIC || hi == FDTD_BND_BLOCH;
    if ((wlo || whi) && lo != hi) return fail(FDTD_ERR_INVALID_ARG, "both faces of a periodic or Bloch axis must match");
    if (wlo && desc->pml_lo[a] + desc->pml_hi[a] != 0)
      return fail(FDTD_ERR_INVALID_ARG, "a periodic or Bloch axis has no CPML slabs");
  }
  const int n[3] = {desc->nx, desc->ny, desc->nz};
  for (int a = 0; a < 3; ++a) {
    if (desc->pml_lo[a] < 0 || desc->pml_hi[a] < 0 || desc->pml_lo[a] + desc->pml_hi[a] > n[a] - 1)
      return fail(FDTD_ERR_INVALID_ARG, "CPML slab lengths exceed the axis");
  }
  fdtd_engine* h = new fdtd_engine();
  h->desc = *desc;
  for (int f = 0; f < 4; ++f) {
    if (desc->boundary[f] == FDTD_BND_PERIODIC || desc->boundary[f] == FDTD_BND_BLOCH) h->wrap = true;
    if (desc->boundary[f] == FDTD_BND_BLOCH) h->bloch = true;
  }
  for (int f = 0; f < 6; ++f)
    if (desc->boundary[f] == FDTD_BND_PMC) h->pmc = true;
  h->stream = static_cast<cudaStream_t>(stream);
  h->NX = desc->nx;
  h->NY = desc->ny;
  h->NZ = desc->nz;
  h->P = (desc->nz + 3) / 4 * 4;
  {
    // z-slab psi rows: low slab at [0, zlo4), high slab cells k >= zhs4 at
    // zlo4 + k - zhs4, with zlo4 = lo rounded up and zhs4 = the first high-slab
    // cell of any component rounded down to multiples of four.  When the two
    // segments would overlap the rows are kept whole (zlo4 = zhs4 = P).
    const int lo = desc->pml_lo[2], hi = desc->pml_hi[2];
    h->zlo4 = (lo + 3) / 4 * 4;
    h->zhs4 = (desc->nz - 1 - hi) / 4 * 4;
    if (h->zhs4 < h->zlo4) h->zlo4 = h->zhs4 = h->P;
    h->SZ = (lo + hi > 0) ? h->zlo4 + (h->P - h->zhs4) : 0;
  }
  h->plane = static_cast<int64_t>(h->NY) * h->P;
  h->vol = h->plane * h->NX;
  h->M = desc->sample_block > 0 ? std::min(desc->sample_block, 64) : 32;
  h->cpml = false;
  for (int a = 0; a < 3; ++a)
    if (desc->pml_lo[a] + desc->pml_hi[a] > 0) h->cpml = true;
  int rc = 0;
  for (int b = 0; b < 2 && !rc; ++b)
    for (int c = 0; c < 3 && !rc; ++c) {
      rc = dev_alloc(h, &h->E[b][c], h->vol);
      if (!rc) rc = dev_alloc(h, &h->H[b][c], h->vol);
    }
  for (int c = 0; c < 3 && !rc; ++c) {
    const int ax[2] = {axis_a(c), axis_b(c)};
    for (int w = 0; w < 2 && !rc; ++w) {
      const int64_t cnt = slab_elems(h, ax[w]);
      rc = dev_alloc(h, &h->psiE[c][w], cnt);
      if (!rc) rc = dev_alloc(h, &h->psiH[0][c][w], cnt);
      if (!rc) rc = dev_alloc(h, &h->psiH[1][c][w], cnt);
    }
  }
  for (int c = 0; c < 6; ++c) {
    h->ucoef[c][0] = 1.0f;
    h->ucoef[c][1] = 0.0f;
  }
  if (!rc) {
    cudaError_t e1 = cudaEventCreate(&h->ev0);
    cudaError_t e2 = cudaEventCreate(&h->ev1);
    if (e1 != cudaSuccess || e2 != cudaSuccess) rc = cuda_fail(e1 != cudaSuccess ? e1 : e2, "cudaEventCreate");
  }
  if (!rc) {
    int least = 0, greatest = 0;
    cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&h->aux, cudaStreamNonBlocking, greatest);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_gat[0], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_gat[1], cudaEventDisableTiming);
    if (e != cudaSuccess) rc = cuda_fail(e, "gather stream and events");
  }
  if (rc) {
    fdtd_engine_destroy(h);
    return rc;
  }
  // The row-tile kernel is the default where it measured fastest: FP32 scenes
  // without CPML or wrapped faces (256^3 vacuum: 0.201 against 0.253 ms).  With
  // CPML the slab CTAs run in the warp kernel either way and the hybrid launch
  // measured no faster (CPML vacuum 0.389 against 0.393 ms, the dispersive
  // workload 0.520 against 0.509 ms), so those engines keep variant 2.
  if (!h->wrap && !h->cpml && !h->pmc) h->variant = kTileVariant;
  default_tiles(h);
  *out = h;
  return 0;
}

int fdtd_engine_destroy(fdtd_engine* h) {
  if (!h) return 0;
  cudaStreamSynchronize(h->stream);
  for (float* p : h->owned) cudaFree(p);
  for (auto& pl : h->poles) {
    cudaFree(pl.drive);
    cudaFree(pl.inv_eps);
    cudaFree(pl.pol);
    cudaFree(pl.cur);
  }
  for (auto& l : h->lines) {
    cudaFree(l.e_hist);
    cudaFree(l.h_hist);
  }
  for (auto& ck : h->checkpoints) cudaFree(ck.store);
  cudaFree(h->d_terms);
  cudaFree(h->d_poles);
  cudaFree(h->d_regions);
  for (int* p : h->index_bufs) cudaFree(p);
  cudaFree(h->d_flush);
  cudaFree(h->d_warp_class);
  for (float* p : h->adj.bufs) cudaFree(p);
  cudaFree(h->d_status);
  cudaFree(h->d_base);
  cudaFree(h->samples);
  cudaFree(h->w_e);
  cudaFree(h->w_h);
  cudaFree(h->acc_re);
  cudaFree(h->acc_im);
  cudaFree(h->cmp_re);
  cudaFree(h->cmp_im);
  if (h->aux) cudaStreamSynchronize(h->aux);
  for (cudaEvent_t e : {h->ev_fork, h->ev_join, h->ev_gat[0], h->ev_gat[1]})
    if (e) cudaEventDestroy(e);
  if (h->aux) cudaStreamDestroy(h->aux);
  if (h->adj.rev) cudaStreamSynchronize(h->adj.rev);
  for (cudaEvent_t e : {h->adj.ev_rep[0], h->adj.ev_rep[1], h->adj.ev_rev[0], h->adj.ev_rev[1]})
    if (e) cudaEventDestroy(e);
  if (h->adj.rev) cudaStreamDestroy(h->adj.rev);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  delete h;
  return 0;
}

int fdtd_engine_set_storage(fdtd_engine* h, int kind, const float* scales) {
  if (!h || kind < kStoreF32 || kind > kStoreBF16) return fail(FDTD_ERR_INVALID_ARG, "bad storage kind");
  if (h->finalized || !h->poles.empty() || !h->checkpoints.empty())
    return fail(FDTD_ERR_STATE, "storage must be chosen right after fdtd_engine_create");
  if (h->wrap && kind == kStoreF16)
    return fail(FDTD_ERR_UNSUPPORTED, "periodic and Bloch faces need FP32 or BF16 storage");
  if (scales) {
    for (int c = 0; c < 6; ++c) {
      int e = 0;
      if (!(scales[c] > 0.0f) || !std::isfinite(scales[c]) || std::frexp(scales[c], &e) != 0.5f)
        return fail(FDTD_ERR_INVALID_ARG, "storage scales must be positive powers of two");
    }
  }
  if (kind != h->storage) {
    // Re-allocate the four field buffer sets in the new element size (zeroed).
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 3; ++c)
        for (float** buf : {&h->E[b][c], &h->H[b][c]}) {
          auto it = std::find(h->owned.begin(), h->owned.end(), *buf);
          if (it != h->owned.end()) h->owned.erase(it);
          cudaFree(*buf);
          *buf = nullptr;
        }
    h->storage = kind;
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 3; ++c) {
        int rc = dev_alloc(h, &h->E[b][c], static_cast<size_t>(field_floats(h)));
        if (!rc) rc = dev_alloc(h, &h->H[b][c], static_cast<size_t>(field_floats(h)));
        if (rc) return rc;
      }
    h->cur = 0;
  }
  for (int c = 0; c < 6; ++c) h->fscale[c] = scales ? scales[c] : 1.0f;
  h->scales_set = scales != nullptr;
  if (kind != kStoreF32) h->variant = 2;
  return 0;
}

int fdtd_engine_get_storage(fdtd_engine* h, int* kind, float* scales) {
  if (!h) return fail(FDTD_ERR_INVALID_ARG, "null engine");
  if (kind) *kind = h->storage;
  if (scales)
    for (int c = 0; c < 6; ++c) scales[c] = h->fscale[c];
  return 0;
}

int fdtd_engine_set_spacing(fdtd_engine* h, int axis, const float* inv_e, const float* inv_h) {
  if (!h || axis < 0 || axis > 2 || !inv_e || !inv_h) return fail(FDTD_ERR_INVALID_ARG, "bad spacing arguments");
  const int n[3] = {h->NX, h->NY, h->NZ};
  int rc = dev_copy(h, &h->inv_e[axis], inv_e, n[axis]);
  if (!rc) rc = dev_copy(h, &h->inv_h[axis], inv_h, n[axis] - 1);
  return rc;
}

int fdtd_engine_set_cpml(fdtd_engine* h, int axis, const float* b_e, const float* c_e, const float* ik_e,
                         const float* b_h, const float* c_h, const float* ik_h) {
  if (!h || axis < 0 || axis > 2 || !b_e || !c_e || !ik_e || !b_h || !c_h || !ik_h)
    return fail(FDTD_ERR_INVALID_ARG, "bad CPML profile arguments");
  const int n[3] = {h->NX, h->NY, h->NZ};
  int rc = dev_copy(h, &h->eb[axis], b_e, n[axis]);
  if (!rc) rc = dev_copy(h, &h->ec[axis], c_e, n[axis]);
  if (!rc) rc = dev_copy(h, &h->eik[axis], ik_e, n[axis]);
  if (!rc) rc = dev_copy(h, &h->hb[axis], b_h, n[axis] - 1);
  if (!rc) rc = dev_copy(h, &h->hc[axis], c_h, n[axis] - 1);
  if (!rc) rc = dev_copy(h, &h->hik[axis], ik_h, n[axis] - 1);
  return rc;
}

int fdtd_engine_set_coefficients(fdtd_engine* h, int comp, const float* decay, float decay_uniform,
                                 const float* curl, float curl_uniform) {
  if (!h || comp < 0 || comp > 5) return fail(FDTD_ERR_INVALID_ARG, "bad coefficient arguments");
  if (h->finalized) return fail(FDTD_ERR_STATE, "engine already finalized");
  int ext[3];
  comp_extent(comp, h->NX, h->NY, h->NZ, ext);
  const float* src[2] = {decay, curl};
  h->ucoef[comp][0] = decay_uniform;
  h->ucoef[comp][1] = curl_uniform;
  for (int w = 0; w < 2; ++w) {
    if (!src[w]) {
      h->ecoef[comp][w] = nullptr;
      continue;
    }
    int rc = dev_alloc(h, &h->ecoef[comp][w], h->vol);
    if (rc) return rc;
    pack_kernel<<<1024, 256, 0, h->stream>>>(h->ecoef[comp][w], src[w], ext[0], ext[1], ext[2], h->NY, h->P, kNoRemap, 0);
    CUDA_TRY(cudaGetLastError());
  }
  return 0;
}

int fdtd_engine_pack_field(fdtd_engine* h, int comp, const float* src) {
  if (!h || comp < 0 || comp > 5 || !src) return fail(FDTD_ERR_INVALID_ARG, "bad pack arguments");
  int ext[3];
  comp_extent(comp, h->NX, h->NY, h->NZ, ext);
  float* dst = comp < 3 ? h->E[h->cur][comp] : h->H[h->cur][comp - 3];
  const float inv = 1.0f / h->fscale[comp];
  if (h->storage == kStoreF16)
    pack_field_rs_kernel<__half><<<1024, 256, 0, h->stream>>>(reinterpret_cast<__half*>(dst), src, ext[0], ext[1],
                                                              ext[2], h->NY, h->P, inv);
  else if (h->storage == kStoreBF16)
    pack_field_rs_kernel<__nv_bfloat16><<<1024, 256, 0, h->stream>>>(reinterpret_cast<__nv_bfloat16*>(dst), src,
                                                                     ext[0], ext[1], ext[2], h->NY, h->P, inv);
  else
    pack_kernel<<<1024, 256, 0, h->stream>>>(dst, src, ext[0], ext[1], ext[2], h->NY, h->P, kNoRemap, 0);
  CUDA_TRY(cudaGetLastError());
  return 0;
}

int fdtd_engine_unpack_field(fdtd_engine* h, int comp, float* dst) {
  if (!h || comp < 0 || comp > 5 || !dst) return fail(FDTD_ERR_INVALID_ARG, "bad unpack arguments");
  int ext[3];
  comp_extent(comp, h->NX, h->NY, h->NZ, ext);
  const float* src = comp < 3 ? h->E[h->cur][comp] : h->H[h->cur][comp - 3];
  if (h->storage == kStoreF16)
    unpack_field_rs_kernel<__half><<<1024, 256, 0, h->stream>>>(dst, reinterpret_cast<const __half*>(src), ext[0],
                                                                ext[1], ext[2], h->NY, h->P, h->fscale[comp]);
  else if (h->storage == kStoreBF16)
    unpack_field_rs_kernel<__nv_bfloat16><<<1024, 256, 0, h->stream>>>(
        dst, reinterpret_cast<const __nv_bfloat16*>(src), ext[0], ext[1], ext[2], h->NY, h->P, h->fscale[comp]);
  else
    unpack_kernel<<<1024, 256, 0, h->stream>>>(dst, src, ext[0], ext[1], ext[2], h->NY, h->P, kNoRemap, 0);
  CUDA_TRY(cudaGetLastError());
  return 0;
}

// Inner-coordinate remap of a z-slab psi array of a component with z extent
// `ext_z`: slab coordinate s >= zlo (the high slab) sits at s + zshift.
static void zslab_remap(const fdtd_engine* h, int ext_z, int* zlo, int* zshift) {
  const int lo = h->desc.pml_lo[2], hi = h->desc.pml_hi[2];
  *zlo = lo;
  *zshift = h->zlo4 - lo + (ext_z - hi) - h->zhs4;
}

static int psi_geometry(fdtd_engine* h, int comp, int which, float** buf, int shape[3], int* pitch_y,
                        int* pitch_z, int* zlo, int* zshift) {
  const int c = comp % 3;
  const int axis = which == 0 ? axis_a(c) : axis_b(c);
  int ext[3];
  comp_extent(comp, h->NX, h->NY, h->NZ, ext);
  const int L = h->desc.pml_lo[axis] + h->desc.pml_hi[axis];
  shape[0] = ext[0];
  shape[1] = ext[1];
  shape[2] = ext[2];
  shape[axis] = L;
  *buf = comp < 3 ? h->psiE[c][which] : h->psiH[h->cur][c][which];
  // internal pitches: x slab [L][NY][P], y slab [NX][L][P], z slab [NX][NY][SZ]
  *pitch_y = axis == 1 ? L : h->NY;
  *pitch_z = axis == 2 ? h->SZ : h->P;
  *zlo = kNoRemap;
  *zshift = 0;
  if (axis == 2) zslab_remap(h, ext[2], zlo, zshift);
  return L;
}

int fdtd_engine_pack_psi(fdtd_engine* h, int comp, int which, const float* src) {
  if (!h || comp < 0 || comp > 5 || which < 0 || which > 1 || !src)
    return fail(FDTD_ERR_INVALID_ARG, "bad psi pack arguments");
  float* buf;
  int shape[3], py, pz, zlo, zshift;
  if (psi_geometry(h, comp, which, &buf, shape, &py, &pz, &zlo, &zshift) == 0) return 0;
  pack_kernel<<<1024, 256, 0, h->stream>>>(buf, src, shape[0], shape[1], shape[2], py, pz, zlo, zshift);
  CUDA_TRY(cudaGetLastError());
  return 0;
}

int fdtd_engine_unpack_psi(fdtd_engine* h, int comp, int which, float* dst) {
  if (!h || comp < 0 || comp > 5 || which < 0 || which > 1 || !dst)
    return fail(FDTD_ERR_INVALID_ARG, "bad psi unpack arguments");
  float* buf;
  int shape[3], py, pz, zlo, zshift;
  if (psi_geometry(h, comp, which, &buf, shape, &py, &pz, &zlo, &zshift) == 0) return 0;
  unpack_kernel<<<1024, 256, 0, h->stream>>>(dst, buf, shape[0], shape[1], shape[2], py, pz, zlo, zshift);
  CUDA_TRY(cudaGetLastError());
  return 0;
}

int fdtd_engine_add_pole(fdtd_engine* h, int comp, int kind, const int* box, const float* drive,
                         const float* inv_eps, float decay, float restoring, int* pole_id) {
  if (!h || comp < 0 || comp > 2 || kind < 0 || kind > 2 || !box || !drive || !inv_eps)
    return fail(FDTD_ERR_INVALID_ARG, "bad pole arguments");
  if (h->finalized) return fail(FDTD_ERR_STATE, "engine already finalized");
  if (!box_ok(h, comp, box)) return fail(FDTD_ERR_INVALID_ARG, "pole box outside the component extent");
  PoleHost ph;
  // Stored with the z range padded to multiples of four (zero drive and 1/eps
  // in the padding) so the vectorised step kernel reads whole lane groups.
  const int nk = box[5] - box[4];
  const int kk0 = box[4] & ~3, kk1 = (box[5] + 3) & ~3;
  const int nkk = kk1 - kk0;
  const int64_t rows = static_cast<int64_t>(box[1] - box[0]) * (box[3] - box[2]);
  ph.count = rows * nk;
  ph.rows = rows;
  ph.nk = nk;
  ph.nkk = nkk;
  ph.koff = box[4] - kk0;
  const size_t bytes = static_cast<size_t>(rows) * nkk * sizeof(float);
  // state arrays: BF16 with BF16 field storage, FP32 otherwise
  ph.state_floats =
      static_cast<int64_t>((static_cast<size_t>(rows) * nkk * (h->storage == kStoreBF16 ? 2 : 4) + 3) / 4);
  const size_t sbytes = static_cast<size_t>(ph.state_floats) * sizeof(float);
  CUDA_TRY(cudaMalloc(&ph.drive, bytes));
  CUDA_TRY(cudaMalloc(&ph.inv_eps, bytes));
  CUDA_TRY(cudaMalloc(&ph.pol, sbytes));
  CUDA_TRY(cudaMalloc(&ph.cur, sbytes));
  CUDA_TRY(cudaMemsetAsync(ph.drive, 0, bytes, h->stream));
  CUDA_TRY(cudaMemsetAsync(ph.inv_eps, 0, bytes, h->stream));
  CUDA_TRY(cudaMemsetAsync(ph.pol, 0, sbytes, h->stream));
  CUDA_TRY(cudaMemsetAsync(ph.cur, 0, sbytes, h->stream));
  CUDA_TRY(cudaMemcpy2DAsync(ph.drive + ph.koff, nkk * sizeof(float), drive, nk * sizeof(float), nk * sizeof(float),
                             rows, cudaMemcpyDefault, h->stream));
  CUDA_TRY(cudaMemcpy2DAsync(ph.inv_eps + ph.koff, nkk * sizeof(float), inv_eps, nk * sizeof(float),
                             nk * sizeof(float), rows, cudaMemcpyDefault, h->stream));
  PoleTerm& t = ph.t;
  t.comp = comp;
  t.kind = kind;
  t.i0 = box[0];
  t.i1 = box[1];
  t.j0 = box[2];
  t.j1 = box[3];
  t.k0 = box[4];
  t.k1 = box[5];
  t.kk0 = kk0;
  t.nkk = nkk;
  t.decay = decay;
  t.restoring = restoring;
  t.dt = static_cast<float>(h->desc.dt);
  t.inv_dt = static_cast<float>(1.0 / h->desc.dt);
  t.drive = ph.drive;
  t.inv_eps = ph.inv_eps;
  t.pol = ph.pol;
  t.cur = ph.cur;
  h->poles.push_back(ph);
  if (pole_id) *pole_id = static_cast<int>(h->poles.size()) - 1;
  return 0;
}

int fdtd_engine_pole_state(fdtd_engine* h, int pole_id, float* pol_out, float* cur_out) {
  if (!h || pole_id < 0 || pole_id >= static_cast<int>(h->poles.size()))
    return fail(FDTD_ERR_INVALID_ARG, "bad pole id");
  const PoleHost& ph = h->poles[pole_id];
  if (h->storage == kStoreBF16) {
    if (pol_out)
      unpack_pole_bf16_kernel<<<256, 256, 0, h->stream>>>(pol_out, reinterpret_cast<const __nv_bfloat16*>(ph.pol),
                                                          ph.rows, ph.nk, ph.nkk, ph.koff);
    if (cur_out)
      unpack_pole_bf16_kernel<<<256, 256, 0, h->stream>>>(cur_out, reinterpret_cast<const __nv_bfloat16*>(ph.cur),
                                                          ph.rows, ph.nk, ph.nkk, ph.koff);
    CUDA_TRY(cudaGetLastError());
    return 0;
  }
  const size_t w = ph.nk * sizeof(float), pitch = ph.nkk * sizeof(float);
  if (pol_out)
    CUDA_TRY(cudaMemcpy2DAsync(pol_out, w, ph.pol + ph.koff, pitch, w, ph.rows, cudaMemcpyDefault, h->stream));
  if (cur_out)
    CUDA_TRY(cudaMemcpy2DAsync(cur_out, w, ph.cur + ph.koff, pitch, w, ph.rows, cudaMemcpyDefault, h->stream));
  return 0;
}

int fdtd_engine_set_pole_state(fdtd_engine* h, int pole_id, const float* pol, const float* cur) {
  if (!h || pole_id < 0 || pole_id >= static_cast<int>(h->poles.size()))
    return fail(FDTD_ERR_INVALID_ARG, "bad pole id");
  if (h->storage == kStoreBF16) return fail(FDTD_ERR_UNSUPPORTED, "pole state is BF16 here: set it through FP32 storage");
  const PoleHost& ph = h->poles[pole_id];
  const size_t w = ph.nk * sizeof(float), pitch = ph.nkk * sizeof(float);
  if (pol) CUDA_TRY(cudaMemcpy2DAsync(ph.pol + ph.koff, pitch, pol, w, w, ph.rows, cudaMemcpyDefault, h->stream));
  if (cur) CUDA_TRY(cudaMemcpy2DAsync(ph.cur + ph.koff, pitch, cur, w, w, ph.rows, cudaMemcpyDefault, h->stream));
  return 0;
}

int fdtd_engine_add_patch(fdtd_engine* h, int comp, const int* box, const float* coeff, const float* signal,
                          int n_signal, float scale) {
  if (!h || comp < 0 || comp > 5 || !box || !coeff || !signal || n_signal <= 0)
    return fail(FDTD_ERR_INVALID_ARG, "bad patch arguments");
  if (h->finalized) return fail(FDTD_ERR_STATE, "engine already finalized");
  if (!box_ok(h, comp, box)) return fail(FDTD_ERR_INVALID_ARG, "patch box outside the component extent");
  InjectionTerm t{};
  t.comp = comp;
  t.i0 = box[0];
  t.i1 = box[1];
  t.j0 = box[2];
  t.j1 = box[3];
  t.k0 = box[4];
  t.k1 = box[5];
  const int64_t cnt = static_cast<int64_t>(t.i1 - t.i0) * (t.j1 - t.j0) * (t.k1 - t.k0);
  float* c = nullptr;
  float* s = nullptr;
  int rc = dev_copy(h, &c, coeff, cnt);
  if (!rc) rc = dev_copy(h, &s, signal, n_signal);
  if (rc) return rc;
  t.coeff = c;
  t.signal = s;
  t.aux_len = n_signal;  // bound of the signal table
  t.scale = scale;
  h->terms.push_back(t);
  return 0;
}

int fdtd_engine_add_shifted_patch(fdtd_engine* h, int comp, const int* box, const float* scale, const float* delay,
                                  double t_offset, int kind, double frequency, double fwidth, double amplitude,
                                  double phase, double wdelay, int n_steps) {
  if (!h || comp < 0 || comp > 5 || !box || !scale || !delay || kind < 0 || kind > 1 || n_steps <= 0)
    return fail(FDTD_ERR_INVALID_ARG, "bad shifted patch arguments");
  if (h->finalized) return fail(FDTD_ERR_STATE, "engine already finalized");
  if (static_cast<int>(h->shifted.size()) >= kMaxShifted) return fail(FDTD_ERR_UNSUPPORTED, "too many shifted patches");
  if (!box_ok(h, comp, box)) return fail(FDTD_ERR_INVALID_ARG, "patch box outside the component extent");
  const int64_t cnt = static_cast<int64_t>(box[1] - box[0]) * (box[3] - box[2]) * (box[5] - box[4]);
  float *c = nullptr, *sc = nullptr, *dl = nullptr, *ones = nullptr;
  int rc = dev_copy(h, &c, scale, cnt);  // the step-0 coefficients are replaced before the first step
  if (!rc) rc = dev_copy(h, &sc, scale, cnt);
  if (!rc) rc = dev_copy(h, &dl, delay, cnt);
  if (!rc) {
    const std::vector<float> one(static_cast<size_t>(n_steps), 1.0f);
    rc = dev_copy(h, &ones, one.data(), one.size());
    if (!rc) CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  if (rc) return rc;
  InjectionTerm t{};
  t.comp = comp;
  t.i0 = box[0];
  t.i1 = box[1];
  t.j0 = box[2];
  t.j1 = box[3];
  t.k0 = box[4];
  t.k1 = box[5];
  t.coeff = c;
  t.signal = ones;
  t.aux_len = n_steps;
  t.scale = 1.0f;
  h->terms.push_back(t);
  constexpr double kTwoPi = 6.283185307179586;
  ShiftedHost x{};
  x.coeff = c;
  x.scale = sc;
  x.delay = dl;
  x.cells = cnt;
  x.t_offset = t_offset;
  x.wdelay = wdelay;
  x.kind = kind;
  x.omega = static_cast<float>(kTwoPi * frequency);
  x.inv_sigma = static_cast<float>(std::max(kTwoPi * fwidth, 1e-30));
  x.amplitude = static_cast<float>(amplitude);
  x.phase = static_cast<float>(phase);
  h->shifted.push_back(x);
  return 0;
}

int fdtd_engine_set_nonlinear(fdtd_engine* h, int comp, int n_cells, const int* cells, const float* params,
                              int general, float eps0) {
  if (!h || comp < 0 || comp > 2 || n_cells < 0 || (n_cells > 0 && (!cells || !params)) || general < 0 ||
      general > 1 || !(eps0 > 0.0f))
    return fail(FDTD_ERR_INVALID_ARG, "bad nonlinear arguments");
  if (h->finalized) return fail(FDTD_ERR_STATE, "engine already finalized");
  if (h->nl_general >= 0 && h->nl_general != general)
    return fail(FDTD_ERR_INVALID_ARG, "nonlinear components disagree on the general form");
  if (h->storage != kStoreF32) return fail(FDTD_ERR_UNSUPPORTED, "nonlinear media with reduced field storage");
  h->nl_general = general;
  h->nl_eps0 = eps0;
  if (n_cells == 0) return 0;
  std::vector<int> ijk(static_cast<size_t>(3) * n_cells);
  std::vector<float> prm(static_cast<size_t>(6) * n_cells);
  CUDA_TRY(cudaMemcpy(ijk.data(), cells, sizeof(int) * ijk.size(), cudaMemcpyDefault));
  CUDA_TRY(cudaMemcpy(prm.data(), params, sizeof(float) * prm.size(), cudaMemcpyDefault));
  int ext[3];
  comp_extent(comp, h->NX, h->NY, h->NZ, ext);
  for (int t = 0; t < n_cells; ++t) {
    for (int a = 0; a < 3; ++a) {
      const int v = ijk[3 * t + a];
      if (v < 0 || v >= ext[a]) return fail(FDTD_ERR_INVALID_ARG, "nonlinear cell outside the component extent");
      h->nl_cells_h.push_back(v);
    }
    h->nl_cells_h.push_back(comp);
    for (int q = 0; q < 6; ++q) h->nl_prm_h[q].push_back(prm[6 * static_cast<size_t>(t) + q]);
  }
  return 0;
}

int fdtd_engine_set_full_aniso(fdtd_engine* h, int comp, const int* box, const float* coeff_a, const float* coeff_b) {
  if (!h || comp < 0 || comp > 2 || !box || !coeff_a || !coeff_b)
    return fail(FDTD_ERR_INVALID_ARG, "bad full-anisotropy arguments");
  if (h->finalized) return fail(FDTD_ERR_STATE, "engine already finalized");
  if (static_cast<int>(h->aniso.size()) >= kMaxAniso) return fail(FDTD_ERR_UNSUPPORTED, "one anisotropic box per component");
  for (const auto& x : h->aniso)
    if (x.comp == comp) return fail(FDTD_ERR_UNSUPPORTED, "one anisotropic box per component");
  if (!box_ok(h, comp, box)) return fail(FDTD_ERR_INVALID_ARG, "anisotropic box outside the component extent");
  if (h->wrap) return fail(FDTD_ERR_UNSUPPORTED, "full anisotropy with periodic or Bloch faces");
  if (h->storage != kStoreF32) return fail(FDTD_ERR_UNSUPPORTED, "full anisotropy with reduced field storage");
  const int n[3] = {h->NX, h->NY, h->NZ};
  for (int ax = 0; ax < 3; ++ax) {
    // the box and its curl stencils (one cell around it) stay clear of the CPML slabs
    if (h->desc.pml_lo[ax] > 0 && box[2 * ax] < h->desc.pml_lo[ax] + 1)
      return fail(FDTD_ERR_UNSUPPORTED, "anisotropic box within a cell of a CPML slab");
    if (h->desc.pml_hi[ax] > 0 && box[2 * ax + 1] > n[ax] - 1 - h->desc.pml_hi[ax] - 1)
      return fail(FDTD_ERR_UNSUPPORTED, "anisotropic box within a cell of a CPML slab");
  }
  const int64_t cnt = static_cast<int64_t>(box[1] - box[0]) * (box[3] - box[2]) * (box[5] - box[4]);
  AnisoHost x{};
  x.comp = comp;
  for (int q = 0; q < 6; ++q) x.box[q] = box[q];
  int rc = dev_copy(h, &x.ca, coeff_a, cnt);
  if (!rc) rc = dev_copy(h, &x.cb, coeff_b, cnt);
  if (!rc) CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (rc) return rc;
  h->aniso.push_back(x);
  return 0;
}

int fdtd_engine_add_aux_line(fdtd_engine* h, int n_e, const float* e_decay, const float* e_curl,
                             const float* h_decay, const float* h_curl, int source_index, const float* source,
                             int n_steps, int* line_id) {
  if (!h || n_e < 4 || !e_decay || !e_curl || !h_decay || !h_curl || !source || n_steps <= 0)
    return fail(FDTD_ERR_INVALID_ARG, "bad auxiliary line arguments");
  AuxLine l;
  l.ne = n_e;
  l.n_steps = n_steps;
  CUDA_TRY(cudaMalloc(&l.e_hist, sizeof(float) * static_cast<size_t>(n_steps) * n_e));
  CUDA_TRY(cudaMalloc(&l.h_hist, sizeof(float) * static_cast<size_t>(n_steps) * n_e));
  float *ed, *ecu, *hd, *hcu, *src, *e, *hh;
  int rc = dev_copy(h, &ed, e_decay, n_e);
  if (!rc) rc = dev_copy(h, &ecu, e_curl, n_e);
  if (!rc) rc = dev_copy(h, &hd, h_decay, n_e - 1);
  if (!rc) rc = dev_copy(h, &hcu, h_curl, n_e - 1);
  if (!rc) rc = dev_copy(h, &src, source, n_steps);
  if (!rc) rc = dev_alloc(h, &e, n_e);
  if (!rc) rc = dev_alloc(h, &hh, n_e);
  if (rc) return rc;
  aux_history_kernel<<<1, 256, 0, h->stream>>>(n_e, ed, ecu, hd, hcu, source_index, src, n_steps, l.e_hist,
                                               l.h_hist, e, hh);
  CUDA_TRY(cudaGetLastError());
  h->lines.push_back(l);
  if (line_id) *line_id = static_cast<int>(h->lines.size()) - 1;
  return 0;
}

int fdtd_engine_add_line_patch(fdtd_engine* h, int comp, const int* box, const float* coeff, int line_id,
                               int sample_kind, const int* sample_index, int sample_axis, float scale) {
  if (!h || comp < 0 || comp > 5 || !box || !coeff || !sample_index || sample_axis < 0 || sample_axis > 2 ||
      line_id < 0 || line_id >= static_cast<int>(h->lines.size()) || sample_kind < 0 || sample_kind > 1)
    return fail(FDTD_ERR_INVALID_ARG, "bad line patch arguments");
  if (h->finalized) return fail(FDTD_ERR_STATE, "engine already finalized");
  if (!box_ok(h, comp, box)) return fail(FDTD_ERR_INVALID_ARG, "line patch box outside the component extent");
  InjectionTerm t{};
  t.comp = comp;
  t.i0 = box[0];
  t.i1 = box[1];
  t.j0 = box[2];
  t.j1 = box[3];
  t.k0 = box[4];
  t.k1 = box[5];
  const int64_t cnt = static_cast<int64_t>(t.i1 - t.i0) * (t.j1 - t.j0) * (t.k1 - t.k0);
  const int axis_len = box[2 * sample_axis + 1] - box[2 * sample_axis];
  float* c = nullptr;
  int rc = dev_copy(h, &c, coeff, cnt);
  if (rc) return rc;
  const AuxLine& l = h->lines[line_id];
  // Every sample index must address a stored entry of the line history: E
  // histories hold n_e values per step, H histories n_e - 1.
  std::vector<int> host_idx(axis_len);
  CUDA_TRY(cudaMemcpy(host_idx.data(), sample_index, sizeof(int) * axis_len, cudaMemcpyDefault));
  const int limit = sample_kind == 0 ? l.ne : l.ne - 1;
  for (int v : host_idx)
    if (v < 0 || v >= limit) return fail(FDTD_ERR_INVALID_ARG, "line patch sample index outside the incident line");
  int* idx = nullptr;
  CUDA_TRY(cudaMalloc(&idx, sizeof(int) * axis_len));
  CUDA_TRY(cudaMemcpyAsync(idx, host_idx.data(), sizeof(int) * axis_len, cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->owned.push_back(reinterpret_cast<float*>(idx));
  t.coeff = c;
  t.signal = nullptr;
  t.aux_hist = sample_kind == 0 ? l.e_hist : l.h_hist;
  t.sample_index = idx;
  t.aux_len = l.ne;
  t.sample_axis = sample_axis;
  t.scale = scale;
  h->terms.push_back(t);
  return 0;
}

int fdtd_engine_add_sample_region(fdtd_engine* h, int comp, const int* box, int64_t* base) {
  if (!h || comp < 0 || comp > 5 || !box) return fail(FDTD_ERR_INVALID_ARG, "bad sample region arguments");
  if (h->finalized) return fail(FDTD_ERR_STATE, "engine already finalized");
  if (!box_ok(h, comp, box)) return fail(FDTD_ERR_INVALID_ARG, "sample region outside the component extent");
  if (static_cast<int64_t>(box[1] - box[0]) * (box[3] - box[2]) * (box[5] - box[4]) >= (int64_t(1) << 31))
    return fail(FDTD_ERR_INVALID_ARG, "a sample region holds at most 2^31 - 1 cells");
  SampleRegion r{};
  r.comp = comp;
  r.i0 = box[0];
  r.i1 = box[1];
  r.j0 = box[2];
  r.j1 = box[3];
  r.k0 = box[4];
  r.k1 = box[5];
  r.base = h->n_samples;
  h->n_samples += static_cast<int64_t>(r.i1 - r.i0) * (r.j1 - r.j0) * (r.k1 - r.k0);
  h->regions.push_back(r);
  if (base) *base = r.base;
  return 0;
}

namespace {

int set_dft_impl(fdtd_engine* h, int n_freq, const double* omega, int n_steps, const double* window, int per_freq) {
  if (!h || n_freq <= 0 || n_freq > 256 || !omega || n_steps <= 0 || !window)
    return fail(FDTD_ERR_INVALID_ARG, "bad DFT arguments");
  h->n_freq = n_freq;
  h->dft_steps = n_steps;
  cudaFree(h->w_e);
  cudaFree(h->w_h);
  CUDA_TRY(cudaMalloc(&h->w_e, sizeof(float2) * static_cast<size_t>(n_freq) * n_steps));
  CUDA_TRY(cudaMalloc(&h->w_h, sizeof(float2) * static_cast<size_t>(n_freq) * n_steps));
  const size_t n_window = static_cast<size_t>(n_steps) * (per_freq ? n_freq : 1);
  double *d_omega = nullptr, *d_window = nullptr;
  CUDA_TRY(cudaMalloc(&d_omega, sizeof(double) * n_freq));
  CUDA_TRY(cudaMalloc(&d_window, sizeof(double) * n_window));
  CUDA_TRY(cudaMemcpyAsync(d_omega, omega, sizeof(double) * n_freq, cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(cudaMemcpyAsync(d_window, window, sizeof(double) * n_window, cudaMemcpyHostToDevice, h->stream));
  dft_weight_kernel<<<256, 256, 0, h->stream>>>(n_freq, n_steps, d_omega, d_window, per_freq, h->desc.dt, h->w_e,
                                                h->w_h);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  cudaFree(d_omega);
  cudaFree(d_window);
  return 0;
}

}  // namespace

int fdtd_engine_set_dft(fdtd_engine* h, int n_freq, const double* omega, int n_steps, const double* window) {
  return set_dft_impl(h, n_freq, omega, n_steps, window, 0);
}

int fdtd_engine_set_dft_windows(fdtd_engine* h, int n_freq, const double* omega, int n_steps, const double* window) {
  return set_dft_impl(h, n_freq, omega, n_steps, window, 1);
}

namespace {

float host_absmax(const std::vector<float>& v) {
  float m = 0.0f;
  for (float x : v) m = std::max(m, std::fabs(x));
  return m;
}

// FP16 storage scales from the sources: the E peak is bounded by the incident
// line's E history (TFSF) and, for soft sources, by max|coeff| times the sum of
// |signal| over the table; the H peak by the line's H history and E / eta0.
// Each scale maps its estimate to [32, 64), leaving three decades of headroom
// below the FP16 maximum 65504 and keeping six decades of values above the
// FP16 normal range.
int estimate_scales(fdtd_engine* h) {
  double e_peak = 0.0, h_peak = 0.0;
  for (const auto& t : h->terms) {
    const int64_t cells = static_cast<int64_t>(t.i1 - t.i0) * (t.j1 - t.j0) * (t.k1 - t.k0);
    std::vector<float> coeff(static_cast<size_t>(cells));
    CUDA_TRY(cudaMemcpy(coeff.data(), t.coeff, sizeof(float) * cells, cudaMemcpyDeviceToHost));
    const double cmax = host_absmax(coeff) * std::fabs(t.scale);
    if (t.signal) {
      std::vector<float> sig(static_cast<size_t>(t.aux_len));
      CUDA_TRY(cudaMemcpy(sig.data(), t.signal, sizeof(float) * t.aux_len, cudaMemcpyDeviceToHost));
      double sum = 0.0;
      for (float x : sig) sum += std::fabs(x);
      if (t.comp < 3) e_peak = std::max(e_peak, cmax * sum);
      else h_peak = std::max(h_peak, cmax * sum);
    }
  }
  for (const auto& l : h->lines) {
    const size_t n = static_cast<size_t>(l.n_steps) * l.ne;
    std::vector<float> v(n);
    CUDA_TRY(cudaMemcpy(v.data(), l.e_hist, sizeof(float) * n, cudaMemcpyDeviceToHost));
    e_peak = std::max(e_peak, static_cast<double>(host_absmax(v)));
    CUDA_TRY(cudaMemcpy(v.data(), l.h_hist, sizeof(float) * n, cudaMemcpyDeviceToHost));
    h_peak = std::max(h_peak, static_cast<double>(host_absmax(v)));
  }
  constexpr double kEta0 = 376.730313668;
  h_peak = std::max(h_peak, e_peak / kEta0);
  auto pick = [](double peak) {
    if (!(peak > 0.0) || !std::isfinite(peak)) return 1.0f;
    int e = 0;
    std::frexp(peak, &e);  // peak in [2^(e-1), 2^e)
    return static_cast<float>(std::ldexp(1.0, e - 6));
  };
  for (int c = 0; c < 3; ++c) {
    h->fscale[c] = pick(e_peak);
    h->fscale[3 + c] = pick(h_peak);
  }
  return 0;
}

}  // namespace

int fdtd_engine_finalize(fdtd_engine* h) {
  if (!h) return fail(FDTD_ERR_INVALID_ARG, "null engine");
  if (h->finalized) return 0;
  if (h->storage == kStoreF16 && !h->scales_set) {
    const int rc = estimate_scales(h);
    if (rc) return rc;
  }
  for (int a = 0; a < 3; ++a) {
    if (!h->inv_e[a] || !h->inv_h[a]) return fail(FDTD_ERR_STATE, "spacing not set on every axis");
    if (h->cpml && (!h->eb[a] || !h->hb[a])) return fail(FDTD_ERR_STATE, "CPML profile not set on every axis");
  }
  {
    // uniform grid: every inverse spacing of an axis (dual and primal) equal
    bool uni = true;
    const int nn[3] = {h->NX, h->NY, h->NZ};
    for (int a = 0; a < 3 && uni; ++a) {
      std::vector<float> ve(nn[a]), vh(nn[a] - 1);
      CUDA_TRY(cudaMemcpy(ve.data(), h->inv_e[a], sizeof(float) * nn[a], cudaMemcpyDeviceToHost));
      CUDA_TRY(cudaMemcpy(vh.data(), h->inv_h[a], sizeof(float) * (nn[a] - 1), cudaMemcpyDeviceToHost));
      for (float v : ve) uni = uni && v == ve[0];
      for (float v : vh) uni = uni && v == ve[0];
      h->inv_e_u[a] = ve[0];
      h->inv_h_u[a] = vh[0];
    }
    h->uniform_grid = uni;
  }
  int rc = upload_vec(h, &h->d_terms, h->terms);
  if (rc) return rc;
  for (int ph = 0; ph < 2; ++ph) {
    std::vector<int> sel;
    for (size_t x = 0; x < h->terms.size(); ++x)
      if ((h->terms[x].comp >= 3) == (ph == 1)) sel.push_back(static_cast<int>(x));
    h->n_terms_ph[ph] = static_cast<int>(sel.size());
    rc = build_box_index(h, h->terms, sel, h->term_ix[ph]);
    if (rc) return rc;
  }
  if (!h->aniso.empty() && (!h->poles.empty() || h->nl_general >= 0))
    return fail(FDTD_ERR_UNSUPPORTED, "full anisotropy with dispersive or nonlinear media");
  if (h->nl_general >= 0) {
    // nonlinear cells: their coefficient arrays must exist (the host passes
    // arrays, not uniform values), poles run in the ADE pass, FP32 storage
    for (int c = 0; c < 3; ++c)
      if (!h->ecoef[c][1] || (h->nl_general == 1 && !h->ecoef[c][0]))
        return fail(FDTD_ERR_STATE, "nonlinear media need E coefficient arrays (decay and curl)");
    if (h->storage != kStoreF32) return fail(FDTD_ERR_UNSUPPORTED, "nonlinear media with reduced field storage");
    if (h->bloch) return fail(FDTD_ERR_UNSUPPORTED, "nonlinear media on Bloch (complex) fields");
    if (!h->poles.empty()) {
      if (!h->ade_pass || h->poles.size() > static_cast<size_t>(kAdeMaxPoles))
        return fail(FDTD_ERR_UNSUPPORTED, "nonlinear media with poles need the ADE pass (at most 32 pole components)");
      if (h->variant >= 4 && h->variant != kTileVariant)
        return fail(FDTD_ERR_UNSUPPORTED, "nonlinear media with poles run launch variants 1-3 and 10");
    }
    const int64_t n = static_cast<int64_t>(h->nl_cells_h.size() / 4);
    CUDA_TRY(cudaMalloc(&h->d_nl_cells, sizeof(int4) * n));
    h->owned.push_back(reinterpret_cast<float*>(h->d_nl_cells));
    CUDA_TRY(cudaMemcpy(h->d_nl_cells, h->nl_cells_h.data(), sizeof(int4) * n, cudaMemcpyHostToDevice));
    std::vector<float> prm;
    prm.reserve(static_cast<size_t>(6 * n));
    for (int q = 0; q < 6; ++q) prm.insert(prm.end(), h->nl_prm_h[q].begin(), h->nl_prm_h[q].end());
    rc = dev_copy(h, &h->d_nl_prm, prm.data(), prm.size());
    if (!rc) CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (rc) return rc;
    h->nl_n = n;
    for (int a = 0; a < 3; ++a) {
      h->nl_lo[a] = INT_MAX;
      h->nl_hi[a] = -1;
    }
    for (int64_t t = 0; t < n; ++t)
      for (int a = 0; a < 3; ++a) {
        h->nl_lo[a] = std::min(h->nl_lo[a], h->nl_cells_h[4 * t + a]);
        h->nl_hi[a] = std::max(h->nl_hi[a], h->nl_cells_h[4 * t + a] + 1);
      }
    if (n == 0)
      for (int a = 0; a < 3; ++a) h->nl_lo[a] = h->nl_hi[a] = 0;
    h->nl_cells_h.clear();
    for (int q = 0; q < 6; ++q) h->nl_prm_h[q].clear();
  }
  std::vector<PoleTerm> pv;
  for (const auto& ph : h->poles) pv.push_back(ph.t);
  rc = upload_vec(h, &h->d_poles, pv);
  if (rc) return rc;
  {
    std::vector<int> ptr, ids;
    build_plane_csr(h->NX, pv, ptr, ids);
    const int* dp = nullptr;
    const int* di = nullptr;
    rc = upload_ints(h, ptr, &dp);
    if (!rc) rc = upload_ints(h, ids, &di);
    if (rc) return rc;
    h->d_pole_ptr = const_cast<int*>(dp);
    h->d_pole_ids = const_cast<int*>(di);
  }
  if (!h->poles.empty() && h->poles.size() <= static_cast<size_t>(kAdeMaxPoles)) {
    // ADE pass: the pole table, and tiles over the z range of each (i, j) row
    // covered by any pole box, cut into 32 * kAdeCellsPerLane-cell pieces (one
    // warp each), with the mask of the poles that meet each piece
    AdeParams& a = h->ade;
    a.NY = h->NY;
    a.P = h->P;
    a.NX = h->NX;
    a.NZ = h->NZ;
    a.pec_faces = 0;
    for (int c = 0; c < 3; ++c) a.nl_curl[c] = h->nl_general >= 0 ? h->ecoef[c][1] : nullptr;
    if (h->lines.empty())
      for (int f = 0; f < 6; ++f)
        if (h->desc.boundary[f] == FDTD_BND_PEC) a.pec_faces |= 1 << f;
    for (size_t b = 0; b < h->poles.size(); ++b) {
      const PoleTerm& t = h->poles[b].t;
      AdePole& q = a.poles[b];
      q.comp = t.comp;
      q.kind = t.kind;
      q.i0 = t.i0;
      q.j0 = t.j0;
      q.nj = t.j1 - t.j0;
      q.k0 = t.k0;
      q.k1 = t.k1;
      q.kk0 = t.kk0;
      q.nkk = t.nkk;
      q.decay = t.decay;
      q.restoring = t.restoring;
      q.dt = t.dt;
      q.inv_dt = t.inv_dt;
      q.drive = t.drive;
      q.inv_eps = t.inv_eps;
      q.pol = t.pol;
      q.cur = t.cur;
    }
    const int64_t rows = static_cast<int64_t>(h->NX) * h->NY;
    std::vector<int> kmin(static_cast<size_t>(rows), INT_MAX), kmax(static_cast<size_t>(rows), -1);
    std::vector<unsigned> rmask(static_cast<size_t>(rows), 0u);
    for (size_t b = 0; b < h->poles.size(); ++b) {
      const PoleTerm& t = h->poles[b].t;
      for (int i = t.i0; i < t.i1; ++i)
        for (int j = t.j0; j < t.j1; ++j) {
          const size_t r = static_cast<size_t>(i) * h->NY + j;
          kmin[r] = std::min(kmin[r], t.k0);
          kmax[r] = std::max(kmax[r], t.k1);
          rmask[r] |= 1u << b;
        }
    }
    std::vector<int> tiles;
    for (int64_t r = 0; r < rows; ++r)
      for (int k0 = kmin[r]; k0 < kmax[r]; k0 += 32 * kAdeCellsPerLane) {
        const int k1 = std::min(k0 + 32 * kAdeCellsPerLane, kmax[r]);
        unsigned m = 0;
        for (unsigned rm = rmask[r]; rm; rm &= rm - 1) {
          const int b = __builtin_ctz(rm);
          if (h->poles[b].t.k0 < k1 && h->poles[b].t.k1 > k0) m |= 1u << b;
        }
        if (!m) continue;
        tiles.push_back(static_cast<int>(r));
        tiles.push_back(k0);
        tiles.push_back(k1);
        tiles.push_back(static_cast<int>(m));
      }
    if (tiles.size() / 4 > static_cast<size_t>(INT_MAX)) return fail(FDTD_ERR_INVALID_ARG, "pole boxes too large");
    rc = upload_ints(h, tiles, &h->d_ade_tiles);
    if (rc) return rc;
    h->n_ade_tiles = static_cast<int>(tiles.size() / 4);
  }
  rc = upload_vec(h, &h->d_regions, h->regions);
  if (rc) return rc;
  for (int ph = 0; ph < 2; ++ph) {
    std::vector<int> sel;
    for (size_t x = 0; x < h->regions.size(); ++x)
      if ((h->regions[x].comp >= 3) == (ph == 1)) sel.push_back(static_cast<int>(x));
    h->n_regions_ph[ph] = static_cast<int>(sel.size());
    rc = build_box_index(h, h->regions, sel, h->region_ix[ph]);
    if (rc) return rc;
  }
  {
    // per-plane activity bits: planes whose x-indexed lists hold items
    std::vector<int> bits(h->NX, 0);
    auto mark_x = [&](const BoxIndex& ix, const std::vector<int>& ptr_host, unsigned flag) {
      (void)ix;
      for (int i = 0; i < h->NX; ++i)
        if (ptr_host[i + 1] > ptr_host[i]) bits[i] |= static_cast<int>(flag);
    };
    for (int ph = 0; ph < 2; ++ph) {
      std::vector<int> pt(h->NX + 1), pr(h->NX + 1);
      CUDA_TRY(cudaMemcpy(pt.data(), h->term_ix[ph].ptr[0], sizeof(int) * (h->NX + 1), cudaMemcpyDeviceToHost));
      CUDA_TRY(cudaMemcpy(pr.data(), h->region_ix[ph].ptr[0], sizeof(int) * (h->NX + 1), cudaMemcpyDeviceToHost));
      mark_x(h->term_ix[ph], pt, ph == 1 ? kPlaneHTerms : kPlaneETerms);
      mark_x(h->region_ix[ph], pr, ph == 1 ? kPlaneHRegions : kPlaneERegions);
    }
    for (const auto& ph : h->poles)
      for (int i = ph.t.i0; i < ph.t.i1; ++i) bits[i] |= static_cast<int>(kPlanePoles);
    rc = upload_ints(h, bits, &h->d_plane_bits);
    if (rc) return rc;
  }
  std::vector<RegionFlush> fl;
  for (const auto& r : h->regions) {
    RegionFlush f;
    f.base = r.base;
    f.count = static_cast<int64_t>(r.i1 - r.i0) * (r.j1 - r.j0) * (r.k1 - r.k0);
    f.is_h = r.comp >= 3 ? 1 : 0;
    f.comp = r.comp;
    f.i0 = r.i0;
    f.j0 = r.j0;
    f.k0 = r.k0;
    f.nj = r.j1 - r.j0;
    f.nk = r.k1 - r.k0;
    fl.push_back(f);
    h->max_region = std::max(h->max_region, f.count);
  }
  rc = upload_vec(h, &h->d_flush, fl);
  if (rc) return rc;
  h->n_flush = static_cast<int>(fl.size());
  if (h->n_samples > 0) {
    CUDA_TRY(cudaMalloc(&h->samples, sizeof(float) * static_cast<size_t>(h->M) * h->n_samples));
    if (h->n_freq > 0) {
      const size_t acc = static_cast<size_t>(h->n_freq) * h->n_samples;
      CUDA_TRY(cudaMalloc(&h->acc_re, sizeof(float) * acc));
      CUDA_TRY(cudaMalloc(&h->acc_im, sizeof(float) * acc));
      CUDA_TRY(cudaMalloc(&h->cmp_re, sizeof(float) * acc));
      CUDA_TRY(cudaMalloc(&h->cmp_im, sizeof(float) * acc));
      CUDA_TRY(cudaMemsetAsync(h->acc_re, 0, sizeof(float) * acc, h->stream));
      CUDA_TRY(cudaMemsetAsync(h->acc_im, 0, sizeof(float) * acc, h->stream));
      CUDA_TRY(cudaMemsetAsync(h->cmp_re, 0, sizeof(float) * acc, h->stream));
      CUDA_TRY(cudaMemsetAsync(h->cmp_im, 0, sizeof(float) * acc, h->stream));
    }
  }
  // The flush stages cnt x n_freq float2 weights (at most 64 x 256 x 8 B).
  CUDA_TRY(cudaFuncSetAttribute(dft_flush_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(sizeof(float2) * 64 * 256)));
  // Background value of each coefficient array (the most frequent of a
  // sample of its cells): warps whose footprint holds only background values
  // use it as a scalar instead of reading the array.
  for (int c = 0; c < 6; ++c) {
    for (int w = 0; w < 2; ++w) {
      if (!h->ecoef[c][w]) continue;
      rc = background_value(h, c, h->ecoef[c][w], &h->ucoef[c][w]);
      if (rc) return rc;
    }
  }
  {
    const int64_t kblocks = (h->NZ + kWarpOut - 1) / kWarpOut;
    CUDA_TRY(cudaMalloc(&h->d_warp_class, static_cast<size_t>(h->NX) * kblocks * h->NY));
    h->class_key = 0;
    CUDA_TRY(cudaMalloc(&h->d_status, sizeof(int)));
    CUDA_TRY(cudaMemsetAsync(h->d_status, 0, sizeof(int), h->stream));
    CUDA_TRY(cudaMalloc(&h->d_base, sizeof(int)));
    CUDA_TRY(cudaMemsetAsync(h->d_base, 0, sizeof(int), h->stream));
  }
  {
    // TMA maps of both ping-pong buffers; without the driver entry point the
    // TMA variant stays unavailable and the warp kernel runs.
    bool ok = h->storage == kStoreF32;
    for (int b = 0; b < 2 && ok; ++b) {
      for (int c = 0; c < 3 && ok; ++c) {
        ok = encode_field_map(&h->maps[b].e[c], h->E[b][c], h->NX, h->NY, h->P, tma_rows_e()) == 0 &&
             encode_field_map(&h->maps[b].h[c], h->H[b][c], h->NX, h->NY, h->P, tma_rows_h()) == 0;
      }
    }
    h->tma_ready = ok;
  }
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->finalized = true;
  return 0;
}

static int step_range_impl(fdtd_engine* h, int n0, int n1, bool record);

// Scope of the second-stream gather inside step_range: forks the gather
// stream from the engine stream on entry (work queued before the call is
// visible to it) and joins it back on join() or on any early return.
struct AsyncGather {
  fdtd_engine* h;
  bool on;
  AsyncGather(fdtd_engine* e, bool enable) : h(e), on(enable) {
    if (!on) return;
    if (cudaEventRecord(h->ev_fork, h->stream) != cudaSuccess || cudaStreamWaitEvent(h->aux, h->ev_fork, 0) != cudaSuccess) {
      on = false;
      return;
    }
    h->async_gather = true;
  }
  int join() {
    if (!on) return 0;
    on = false;
    h->async_gather = false;
    h->gat_pending[0] = h->gat_pending[1] = false;
    CUDA_TRY(cudaEventRecord(h->ev_join, h->aux));
    CUDA_TRY(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
    return 0;
  }
  ~AsyncGather() { join(); }
};

int fdtd_engine_step_range(fdtd_engine* h, int n0, int n1) {
  NvtxRange r("fdtd_engine_step_range");
  return step_range_impl(h, n0, n1, false);
}

int fdtd_engine_step_range_recorded(fdtd_engine* h, int n0, int n1) {
  NvtxRange nvtx_range("fdtd_engine_step_range_recorded");
  if (!h || !h->adj.ready) return fail(FDTD_ERR_STATE, "adjoint not initialised");
  if (n0 < 0 || n1 < n0 || n1 - n0 > h->adj.max_segment) return fail(FDTD_ERR_INVALID_ARG, "bad recorded range");
  return step_range_impl(h, n0, n1, true);
}

static int step_range_impl(fdtd_engine* h, int n0, int n1, bool record) {
  if (!h) return fail(FDTD_ERR_INVALID_ARG, "null engine");
  if (!h->finalized) return fail(FDTD_ERR_STATE, "engine not finalized");
  if (h->bloch || h->in_pair)
    return fail(FDTD_ERR_STATE, "Bloch faces carry a complex field: step the engines with fdtd_bloch_step_range");
  if (n1 < n0 || n0 < 0) return fail(FDTD_ERR_INVALID_ARG, "bad step range");
  for (const auto& t : h->terms) {
    if (t.signal && n1 > t.aux_len) return fail(FDTD_ERR_INVALID_ARG, "source signal table shorter than the range");
  }
  for (const auto& l : h->lines) {
    if (n1 > l.n_steps) return fail(FDTD_ERR_INVALID_ARG, "incident line history shorter than the range");
  }
  if (h->n_samples > 0 && h->n_freq > 0 && n1 > h->dft_steps)
    return fail(FDTD_ERR_INVALID_ARG, "DFT weight table shorter than the range");
  CUDA_TRY(cudaEventRecord(h->ev0, h->stream));
  // Gather and flush on the second stream unless the engine's stream is being
  // captured into a graph (batches capture their own single-stream steps).
  cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
  CUDA_TRY(cudaStreamIsCapturing(h->stream, &capturing));
  AsyncGather overlap(h, h->aux && h->n_flush > 0 && h->n_samples > 0 && !h->graph_base &&
                             capturing == cudaStreamCaptureStatusNone);
  if (record) {
    StepParams p;
    fill_params(h, p);
    const int err = launch_design_record(p, h->adj.q, 0, h->stream);
    if (err) return cuda_fail(static_cast<cudaError_t>(err), "design record");
  }
  for (int n = n0; n < n1; ++n) {
    if (h->pending == 0) h->pending_base = n;
    if (h->pending_base + h->pending != n) {
      int rc = flush_samples(h);
      if (rc) return rc;
      h->pending_base = n;
    }
    int rc = launch_step(h, n, h->pending);
    if (rc) return rc;
    if (record) {
      StepParams p;
      fill_params(h, p);
      const int err = launch_design_record(p, h->adj.q, n + 1 - n0, h->stream);
      if (err) return cuda_fail(static_cast<cudaError_t>(err), "design record");
    }
    if (h->n_samples > 0) {
      ++h->pending;
      if (h->pending == h->M) {
        rc = flush_samples(h);
        if (rc) return rc;
      }
    }
  }
  // The DFT of every step in the range is accumulated before the range ends,
  // so the range's device time holds all of its monitor work.
  if (h->range_flush) {
    const int rc = flush_samples(h);
    if (rc) return rc;
  }
  {
    const int rc = overlap.join();
    if (rc) return rc;
  }
  CUDA_TRY(cudaEventRecord(h->ev1, h->stream));
  CUDA_TRY(cudaEventSynchronize(h->ev1));
  CUDA_TRY(cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1));
  if (record) {
    h->adj.replay_n0 = n0;
    h->adj.replay_n1 = n1;
  }
  return check_status(h);
}

int fdtd_engine_flush(fdtd_engine* h) {
  if (!h) return fail(FDTD_ERR_INVALID_ARG, "null engine");
  return flush_samples(h);
}

int fdtd_engine_read_dft(fdtd_engine* h, float* re, float* im) {
  if (!h || !re || !im) return fail(FDTD_ERR_INVALID_ARG, "bad DFT read arguments");
  if (!h->acc_re) return fail(FDTD_ERR_STATE, "no DFT accumulators");
  int rc = flush_samples(h);
  if (rc) return rc;
  const size_t bytes = sizeof(float) * static_cast<size_t>(h->n_freq) * h->n_samples;
  CUDA_TRY(cudaMemcpyAsync(re, h->acc_re, bytes, cudaMemcpyDefault, h->stream));
  CUDA_TRY(cudaMemcpyAsync(im, h->acc_im, bytes, cudaMemcpyDefault, h->stream));
  return 0;
}

static void state_buffers(fdtd_engine* h, std::vector<std::pair<float*, size_t>>& out) {
  const int c0 = h->cur;
  for (int c = 0; c < 3; ++c) {
    out.push_back({h->E[c0][c], static_cast<size_t>(field_floats(h))});
    out.push_back({h->H[c0][c], static_cast<size_t>(field_floats(h))});
  }
  for (int c = 0; c < 3; ++c) {
    const int ax[2] = {axis_a(c), axis_b(c)};
    for (int w = 0; w < 2; ++w) {
      const size_t n = static_cast<size_t>(slab_elems(h, ax[w]));
      if (n == 0) continue;
      out.push_back({h->psiE[c][w], n});
      out.push_back({h->psiH[c0][c][w], n});
    }
  }
  for (auto& ph : h->poles) {
    out.push_back({ph.pol, static_cast<size_t>(ph.state_floats)});
    out.push_back({ph.cur, static_cast<size_t>(ph.state_floats)});
  }
}

static int checkpoint_alloc(Checkpoint& ck, const std::vector<std::pair<float*, size_t>>& bufs) {
  if (ck.store && ck.bufs.size() == bufs.size()) return 0;
  cudaFree(ck.store);
  ck.store = nullptr;
  size_t total = 0;
  for (const auto& b : bufs) total += (b.second + 63) / 64 * 64;  // 256-byte aligned views
  CUDA_TRY(cudaMalloc(&ck.store, std::max<size_t>(total, 1) * sizeof(float)));
  ck.bufs.clear();
  size_t off = 0;
  for (const auto& b : bufs) {
    ck.bufs.push_back(ck.store + off);
    off += (b.second + 63) / 64 * 64;
  }
  return 0;
}

int fdtd_engine_checkpoint_reserve(fdtd_engine* h, int n_slots) {
  if (!h || n_slots < 0 || n_slots > 1 << 20) return fail(FDTD_ERR_INVALID_ARG, "bad checkpoint count");
  if (static_cast<int>(h->checkpoints.size()) < n_slots) h->checkpoints.resize(n_slots);
  std::vector<std::pair<float*, size_t>> bufs;
  state_buffers(h, bufs);
  for (int s = 0; s < n_slots; ++s) {
    int rc = checkpoint_alloc(h->checkpoints[s], bufs);
    if (rc) return rc;
  }
  return 0;
}

int fdtd_engine_checkpoint_save(fdtd_engine* h, int slot) {
  NvtxRange nvtx_range("fdtd_engine_checkpoint_save");
  if (!h || slot < 0 || slot > 1 << 20) return fail(FDTD_ERR_INVALID_ARG, "bad checkpoint slot");
  if (static_cast<int>(h->checkpoints.size()) <= slot) h->checkpoints.resize(slot + 1);
  std::vector<std::pair<float*, size_t>> bufs;
  state_buffers(h, bufs);
  Checkpoint& ck = h->checkpoints[slot];
  int rc = checkpoint_alloc(ck, bufs);
  if (rc) return rc;
  for (size_t x = 0; x < bufs.size(); ++x)
    CUDA_TRY(cudaMemcpyAsync(ck.bufs[x], bufs[x].first, bufs[x].second * sizeof(float), cudaMemcpyDeviceToDevice,
                             h->stream));
  ck.valid = true;
  return 0;
}

int fdtd_engine_checkpoint_load(fdtd_engine* h, int slot) {
  NvtxRange nvtx_range("fdtd_engine_checkpoint_load");
  if (!h || slot < 0 || slot >= static_cast<int>(h->checkpoints.size()) || !h->checkpoints[slot].valid)
    return fail(FDTD_ERR_INVALID_ARG, "no checkpoint in that slot");
  std::vector<std::pair<float*, size_t>> bufs;
  state_buffers(h, bufs);
  Checkpoint& ck = h->checkpoints[slot];
  for (size_t x = 0; x < bufs.size(); ++x)
    CUDA_TRY(cudaMemcpyAsync(bufs[x].first, ck.bufs[x], bufs[x].second * sizeof(float), cudaMemcpyDeviceToDevice,
                             h->stream));
  return 0;
}

int fdtd_engine_autotune(fdtd_engine* h, int* tile_rows, int* chunk_planes) {
  NvtxRange nvtx_range("fdtd_engine_autotune");
  if (!h || !h->finalized) return fail(FDTD_ERR_STATE, "engine not finalized");
  int rc = flush_samples(h);
  if (rc) return rc;
  const int next_step = h->pending_base;
  // Save the state into a private checkpoint, time the candidates (their steps
  // write scratch samples into slot 0 and advance the state), then restore.
  const int slot = static_cast<int>(h->checkpoints.size());
  rc = fdtd_engine_checkpoint_save(h, slot);
  if (rc) return rc;
  const int cxs[] = {4, 6, 8, 12, 16, 24, 32, 48};
  float best = 1e30f;
  int best_ty = 1, best_cx = h->CX, best_var = h->variant;
  for (int var = 1; var <= kMaxVariant; ++var) {
    if (var == 4 && !h->tma_ready) continue;
    if (h->storage != kStoreF32 && var != 2) continue;  // reduced storage: the 64-register kernel only
    if ((h->wrap || h->pmc) && var > 3) continue;        // wrap and PMC faces: the scalar warp kernels only
    if (h->nl_n > 0 && !h->poles.empty() && var > 3 && var != kTileVariant) continue;  // nonlinear poles: the ADE pass
    for (int cx : cxs) {
      if (cx > 2 * h->NX) continue;
      h->variant = var;
      h->CX = cx;
      const int reps = 3;
      rc = launch_step(h, 0, -1);
      if (rc) return rc;
      CUDA_TRY(cudaEventRecord(h->ev0, h->stream));
      for (int r = 0; r < reps; ++r) {
        rc = launch_step(h, 0, -1);
        if (rc) return rc;
      }
      CUDA_TRY(cudaEventRecord(h->ev1, h->stream));
      CUDA_TRY(cudaEventSynchronize(h->ev1));
      float ms = 0.0f;
      CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
      if (ms < best) {
        best = ms;
        best_cx = cx;
        best_var = var;
      }
    }
  }
  h->TY = best_ty;
  h->CX = best_cx;
  h->variant = best_var;
  rc = fdtd_engine_checkpoint_load(h, slot);
  if (rc) return rc;
  cudaFree(h->checkpoints[slot].store);
  h->checkpoints.pop_back();
  h->pending = 0;
  h->pending_base = next_step;
  if (tile_rows) *tile_rows = best_ty;
  if (chunk_planes) *chunk_planes = best_cx;
  return 0;
}

int fdtd_engine_time_kernel(fdtd_engine* h, int n, int reps, float* ms) {
  if (!h || !ms || reps <= 0 || n < 0) return fail(FDTD_ERR_INVALID_ARG, "bad time_kernel arguments");
  if (!h->finalized) return fail(FDTD_ERR_STATE, "engine not finalized");
  for (const auto& t : h->terms)
    if (t.signal && n >= t.aux_len) return fail(FDTD_ERR_INVALID_ARG, "step index beyond the source table");
  for (const auto& l : h->lines)
    if (n >= l.n_steps) return fail(FDTD_ERR_INVALID_ARG, "step index beyond the incident line history");
  CUDA_TRY(cudaEventRecord(h->ev0, h->stream));
  for (int r = 0; r < reps; ++r) {
    int rc = launch_step(h, n, -1);
    if (rc) return rc;
  }
  CUDA_TRY(cudaEventRecord(h->ev1, h->stream));
  CUDA_TRY(cudaEventSynchronize(h->ev1));
  float total = 0.0f;
  CUDA_TRY(cudaEventElapsedTime(&total, h->ev0, h->ev1));
  *ms = total / static_cast<float>(reps);
  return 0;
}

int fdtd_engine_set_launch(fdtd_engine* h, int variant, int tile_rows, int chunk_planes) {
  if (!h || variant < 1 || variant > kMaxVariant || tile_rows < 0 || chunk_planes < 0)
    return fail(FDTD_ERR_INVALID_ARG, "bad launch configuration");
  (void)tile_rows;  // the warp-granular kernels have no tile height
  if (h->storage != kStoreF32 && variant != 2)
    return fail(FDTD_ERR_UNSUPPORTED, "reduced field storage runs launch variant 2 only");
  if (h->wrap && variant > 3)
    return fail(FDTD_ERR_UNSUPPORTED, "periodic and Bloch faces run launch variants 1-3 only");
  if (h->pmc && variant > 3) return fail(FDTD_ERR_UNSUPPORTED, "PMC faces run launch variants 1-3 only");
  if (h->nl_general >= 0 && !h->poles.empty() && variant > 3 && variant != kTileVariant)
    return fail(FDTD_ERR_UNSUPPORTED, "nonlinear media with poles run launch variants 1-3 and 10");
  h->variant = variant;
  if (chunk_planes > 0) h->CX = chunk_planes;
  else default_tiles(h);
  // the row-tile kernel gathers its chunk's plane bits into 64-bit masks
  if (variant == kTileVariant) h->CX = std::min(h->CX, kTileMaxChunk);
  return 0;
}

// Poles in the ADE pass after the step kernel (on) or inside it (off).
int fdtd_engine_set_ade_pass(fdtd_engine* h, int on) {
  if (!h) return fail(FDTD_ERR_INVALID_ARG, "null engine");
  if (!on && h->nl_general >= 0 && !h->poles.empty())
    return fail(FDTD_ERR_UNSUPPORTED, "nonlinear media with poles need the ADE pass");
  h->ade_pass = on != 0;
  return 0;
}

int fdtd_engine_set_replay_region(fdtd_engine* h, int on) {
  if (!h) return fail(FDTD_ERR_INVALID_ARG, "null engine");
  h->replay_region = on != 0;
  return 0;
}

int fdtd_engine_set_range_flush(fdtd_engine* h, int on) {
  if (!h) return fail(FDTD_ERR_INVALID_ARG, "null engine");
  h->range_flush = on != 0;
  return 0;
}

// One x plane of a component's current state, in the component's Yee shape
// [ny_c][nz_c], to or from a device or host buffer (one strided 2-D copy on
// the engine's stream).
static int plane_copy(fdtd_engine* h, int comp, int i, float* out, const float* in) {
  if (!h || comp < 0 || comp > 5 || (!out && !in)) return fail(FDTD_ERR_INVALID_ARG, "bad plane arguments");
  if (!h->finalized) return fail(FDTD_ERR_STATE, "engine not finalized");
  if (h->storage != kStoreF32) return fail(FDTD_ERR_UNSUPPORTED, "plane copies need FP32 field storage");
  int ext[3];
  comp_extent(comp, h->NX, h->NY, h->NZ, ext);
  if (i < 0 || i >= ext[0]) return fail(FDTD_ERR_INVALID_ARG, "plane index outside the component's x extent");
  float* base = (comp < 3 ? h->E[h->cur][comp] : h->H[h->cur][comp - 3]) + static_cast<int64_t>(i) * h->NY * h->P;
  const size_t row = sizeof(float) * ext[2], pitch = sizeof(float) * h->P;
  if (out)
    CUDA_TRY(cudaMemcpy2DAsync(out, row, base, pitch, row, ext[1], cudaMemcpyDefault, h->stream));
  else
    CUDA_TRY(cudaMemcpy2DAsync(base, pitch, in, row, row, ext[1], cudaMemcpyDefault, h->stream));
  return 0;
}

int fdtd_engine_get_plane(fdtd_engine* h, int comp, int i, float* dst) {
  return dst ? plane_copy(h, comp, i, dst, nullptr) : fail(FDTD_ERR_INVALID_ARG, "null plane buffer");
}

int fdtd_engine_set_plane(fdtd_engine* h, int comp, int i, const float* src) {
  return src ? plane_copy(h, comp, i, nullptr, src) : fail(FDTD_ERR_INVALID_ARG, "null plane buffer");
}

int fdtd_engine_set_wait_limit(fdtd_engine* h, int rounds) {
  if (!h || rounds < 0) return fail(FDTD_ERR_INVALID_ARG, "bad wait limit");
  h->wait_limit = rounds;
  return 0;
}

// L2 prefetch distance of the scalar step kernels (launch variants 1-3).
int fdtd_engine_set_prefetch(fdtd_engine* h, int planes) {
  if (!h || planes < 0 || planes > 16) return fail(FDTD_ERR_INVALID_ARG, "prefetch distance must be 0..16 planes");
  h->pf_dist = planes;
  return 0;
}

// ---------------------------------------------------------------------------
// Reverse-time adjoint (witwin/maxwell/fdtd/adjoint/native.py:48-725,
// core.py:3527-3565 segment replay, checkpoint.py:365-568)
// ---------------------------------------------------------------------------
static int adj_alloc(fdtd_engine* h, float** out, size_t n) {
  *out = nullptr;
  if (n == 0) return 0;
  CUDA_TRY(cudaMalloc(out, n * sizeof(float)));
  CUDA_TRY(cudaMemsetAsync(*out, 0, n * sizeof(float), h->stream));
  h->adj.bufs.push_back(*out);
  return 0;
}

int fdtd_engine_adjoint_init(fdtd_engine* h, const int* design_boxes, int max_segment) {
  if (!h || max_segment < 1) return fail(FDTD_ERR_INVALID_ARG, "bad adjoint arguments");
  if (!h->finalized) return fail(FDTD_ERR_STATE, "engine not finalized");
  if (h->storage != kStoreF32) return fail(FDTD_ERR_UNSUPPORTED, "the adjoint runs on FP32 field storage only");
  if (h->wrap) return fail(FDTD_ERR_UNSUPPORTED, "the adjoint of periodic and Bloch faces is not supported");
  if (h->pmc) return fail(FDTD_ERR_UNSUPPORTED, "the adjoint of PMC faces is not supported");
  if (h->nl_general >= 0) return fail(FDTD_ERR_UNSUPPORTED, "the adjoint of nonlinear media is not supported");
  if (!h->aniso.empty()) return fail(FDTD_ERR_UNSUPPORTED, "the adjoint of full anisotropy is not supported");
  if (h->adj.ready) return fail(FDTD_ERR_STATE, "adjoint already initialised");
  AdjointHost& a = h->adj;
  a.q = AdjParams{};
  for (int c = 0; c < 3; ++c) {
    int rc = adj_alloc(h, &a.q.gE[c], h->vol);
    if (!rc) rc = adj_alloc(h, &a.q.gH[c], h->vol);
    if (rc) return rc;
    const int ax[2] = {axis_a(c), axis_b(c)};
    for (int w = 0; w < 2; ++w) {
      const size_t n = static_cast<size_t>(slab_elems(h, ax[w]));
      rc = adj_alloc(h, &a.q.gpsiE[c][w], n);
      if (!rc) rc = adj_alloc(h, &a.q.gpsiH[c][w], n);
      if (rc) return rc;
    }
  }
  if (!h->poles.empty()) {
    // adjoint pole state, laid out as the forward pole state
    std::vector<float*> gp(h->poles.size()), gc(h->poles.size());
    for (size_t id = 0; id < h->poles.size(); ++id) {
      int rc = adj_alloc(h, &gp[id], static_cast<size_t>(h->poles[id].state_floats));
      if (!rc) rc = adj_alloc(h, &gc[id], static_cast<size_t>(h->poles[id].state_floats));
      if (rc) return rc;
    }
    float** dgp = nullptr;
    float** dgc = nullptr;
    CUDA_TRY(cudaMalloc(&dgp, sizeof(float*) * gp.size()));
    a.bufs.push_back(reinterpret_cast<float*>(dgp));
    CUDA_TRY(cudaMalloc(&dgc, sizeof(float*) * gc.size()));
    a.bufs.push_back(reinterpret_cast<float*>(dgc));
    CUDA_TRY(cudaMemcpy(dgp, gp.data(), sizeof(float*) * gp.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(dgc, gc.data(), sizeof(float*) * gc.size(), cudaMemcpyHostToDevice));
    a.q.gpol = dgp;
    a.q.gcur = dgc;
    a.gpol_host = gp;
    a.gcur_host = gc;
  }
  a.q.n_samples = h->n_samples;
  a.q.inv_dt = static_cast<float>(1.0 / static_cast<double>(static_cast<float>(h->desc.dt)));
  a.max_segment = max_segment;
  for (int c = 0; c < 3; ++c) {
    DesignBox& d = a.q.design[c];
    d = DesignBox{};
    if (!design_boxes) continue;
    const int* b = design_boxes + 6 * c;
    if (b[0] >= b[1] || b[2] >= b[3] || b[4] >= b[5]) continue;
    if (!box_ok(h, c, b)) return fail(FDTD_ERR_INVALID_ARG, "design box outside the component extent");
    // The gradient formula needs plain interior updates: no CPML slab or edge.
    for (int ax = 0; ax < 3; ++ax) {
      const int n_ax = ax == 0 ? h->NX : (ax == 1 ? h->NY : h->NZ);
      if (b[2 * ax] < h->desc.pml_lo[ax] || b[2 * ax + 1] > n_ax - 1 - h->desc.pml_hi[ax])
        return fail(FDTD_ERR_INVALID_ARG, "design box reaches into a CPML slab or the domain edge");
    }
    // Design cells may sit in ADE media (the design variable is then eps_inf):
    // the pole correction -dt inv J' (Drude, Lorentz) or -inv (P' - P) (Debye)
    // carries inv = 1 / eps like the curl and source terms, so
    // dE'/deps = -(E^{n+1} - de E^n) / eps covers it, and the pole states
    // themselves depend on eps only through E (witwin/maxwell/fdtd/adjoint/
    // native.py:2104-2290, reverseDispersiveCorrection3D).
    for (int ax = 0; ax < 3; ++ax) {
      d.lo[ax] = b[2 * ax];
      d.hi[ax] = b[2 * ax + 1];
    }
    d.cells = static_cast<int64_t>(b[1] - b[0]) * (b[3] - b[2]) * (b[5] - b[4]);
    if (d.cells >= INT_MAX) return fail(FDTD_ERR_INVALID_ARG, "design box holds 2^31 cells or more");
    int rc = adj_alloc(h, &d.hist, static_cast<size_t>(d.cells) * (max_segment + 1));
    if (!rc) rc = adj_alloc(h, &d.grad, static_cast<size_t>(d.cells));
    if (rc) return rc;
  }
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  a.ready = true;
  return 0;
}

int fdtd_engine_adjoint_set_seed(fdtd_engine* h, const float* g_re, const float* g_im) {
  if (!h || !h->adj.ready) return fail(FDTD_ERR_STATE, "adjoint not initialised");
  AdjointHost& a = h->adj;
  if (!g_re || !g_im) {
    a.q.seed_re = nullptr;
    a.q.seed_im = nullptr;
    return 0;
  }
  if (h->n_samples == 0 || h->n_freq == 0) return fail(FDTD_ERR_STATE, "no monitor samples to seed");
  const size_t n = static_cast<size_t>(h->n_freq) * h->n_samples;
  if (!a.q.seed_re) {
    float *re = nullptr, *im = nullptr;
    int rc = adj_alloc(h, &re, n);
    if (!rc) rc = adj_alloc(h, &im, n);
    if (rc) return rc;
    a.q.seed_re = re;
    a.q.seed_im = im;
  }
  CUDA_TRY(cudaMemcpyAsync(const_cast<float*>(a.q.seed_re), g_re, n * sizeof(float), cudaMemcpyDefault, h->stream));
  CUDA_TRY(cudaMemcpyAsync(const_cast<float*>(a.q.seed_im), g_im, n * sizeof(float), cudaMemcpyDefault, h->stream));
  return 0;
}

int fdtd_engine_replay_range(fdtd_engine* h, int n0, int n1) {
  if (!h || !h->adj.ready) return fail(FDTD_ERR_STATE, "adjoint not initialised");
  if (n0 < 0 || n1 < n0 || n1 - n0 > h->adj.max_segment) return fail(FDTD_ERR_INVALID_ARG, "bad replay range");
  for (const auto& t : h->terms)
    if (t.signal && n1 > t.aux_len) return fail(FDTD_ERR_INVALID_ARG, "source signal table shorter than the range");
  for (const auto& l : h->lines)
    if (n1 > l.n_steps) return fail(FDTD_ERR_INVALID_ARG, "incident line history shorter than the range");
  int rc = flush_samples(h);  // buffered forward samples belong to the forward run
  if (rc) return rc;
  StepParams p;
  fill_params(h, p);
  int err = launch_design_record(p, h->adj.q, 0, h->stream);
  if (err) return cuda_fail(static_cast<cudaError_t>(err), "design record");
  for (int n = n0; n < n1; ++n) {
    rc = launch_step(h, n, -1);
    if (rc) return rc;
    fill_params(h, p);
    err = launch_design_record(p, h->adj.q, n + 1 - n0, h->stream);
    if (err) return cuda_fail(static_cast<cudaError_t>(err), "design record");
  }
  h->adj.replay_n0 = n0;
  h->adj.replay_n1 = n1;
  return check_status(h);
}

int fdtd_engine_adjoint_range(fdtd_engine* h, int n1, int n0) {
  NvtxRange nvtx_range("fdtd_engine_adjoint_range");
  if (!h || !h->adj.ready) return fail(FDTD_ERR_STATE, "adjoint not initialised");
  if (n0 < 0 || n1 < n0) return fail(FDTD_ERR_INVALID_ARG, "bad adjoint range");
  AdjointHost& a = h->adj;
  bool design = false;
  for (int c = 0; c < 3; ++c) design = design || a.q.design[c].grad;
  if (design && (n0 < a.replay_n0 || n1 > a.replay_n1))
    return fail(FDTD_ERR_STATE, "adjoint range not covered by the last replay");
  if (a.q.seed_re && n1 > h->dft_steps) return fail(FDTD_ERR_INVALID_ARG, "DFT weight table shorter than the range");
  StepParams p;
  fill_params(h, p);
  for (int n = n1 - 1; n >= n0; --n) {
    AdjParams q = a.q;
    q.hist_slot = design ? n - a.replay_n0 : 0;
    const int err = launch_adjoint_step(p, q, h->d_flush, q.seed_re ? h->n_flush : 0, h->w_e, h->w_h, h->n_freq, n,
                                        h->stream);
    if (err) return cuda_fail(static_cast<cudaError_t>(err), "adjoint step");
  }
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return 0;
}

// Segments [s * stride, min((s + 1) * stride, n_steps)) from the last to the
// first.  Segment s needs its design-box E history, which a replay from
// checkpoint slot s rebuilds on the engine stream; its reverse steps run on a
// second stream.  The reverse of segment s and the replay of segment s - 1 are
// independent (the reverse reads only adjoint state, static coefficients and
// the history of segment s; the replay writes only forward state and the
// history of segment s - 1, kept in the other of two buffers), so they run at
// the same time: each is latency-bound well below the HBM roof, and together
// they use it better than one after the other.
int fdtd_engine_backward_replay(fdtd_engine* h, int n_steps, int stride) {
  NvtxRange nvtx_range("fdtd_engine_backward_replay");
  if (!h || !h->adj.ready) return fail(FDTD_ERR_STATE, "adjoint not initialised");
  AdjointHost& a = h->adj;
  if (n_steps < 1 || stride < 1 || stride > a.max_segment)
    return fail(FDTD_ERR_INVALID_ARG, "bad replay stride (at most the max_segment of fdtd_engine_adjoint_init)");
  const int S = (n_steps + stride - 1) / stride;
  if (static_cast<int>(h->checkpoints.size()) < S)
    return fail(FDTD_ERR_STATE, "one checkpoint per segment (slot s = step s * stride) is needed");
  for (int s = 0; s < S; ++s)
    if (!h->checkpoints[s].valid) return fail(FDTD_ERR_STATE, "a segment checkpoint was never saved");
  if (a.q.seed_re && n_steps > h->dft_steps) return fail(FDTD_ERR_INVALID_ARG, "DFT weight table shorter than the range");
  for (const auto& t : h->terms)
    if (t.signal && n_steps > t.aux_len) return fail(FDTD_ERR_INVALID_ARG, "source signal table shorter than the range");
  for (const auto& l : h->lines)
    if (n_steps > l.n_steps) return fail(FDTD_ERR_INVALID_ARG, "incident line history shorter than the range");
  int rc = flush_samples(h);  // buffered forward samples belong to the forward run
  if (rc) return rc;
  if (!a.rev) {
    int prio_lo = 0, prio_hi = 0;
    CUDA_TRY(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    CUDA_TRY(cudaStreamCreateWithPriority(&a.rev, cudaStreamNonBlocking, prio_lo));
    for (int b = 0; b < 2; ++b) {
      CUDA_TRY(cudaEventCreateWithFlags(&a.ev_rep[b], cudaEventDisableTiming));
      CUDA_TRY(cudaEventCreateWithFlags(&a.ev_rev[b], cudaEventDisableTiming));
    }
  }
  bool design = false;
  for (int c = 0; c < 3; ++c) {
    DesignBox& d = a.q.design[c];
    if (!d.grad) continue;
    design = true;
    if (!a.hist2[c]) {
      rc = adj_alloc(h, &a.hist2[c], static_cast<size_t>(d.cells) * (a.max_segment + 1));
      if (rc) return rc;
    }
  }
  // the history buffers of segment s: the engine's for even s, the second for odd s
  auto with_hist = [&](int s) {
    AdjParams q = a.q;
    if (s & 1)
      for (int c = 0; c < 3; ++c)
        if (q.design[c].grad) q.design[c].hist = a.hist2[c];
    return q;
  };
  // Region replay: the segment only has to reproduce E in the design boxes.
  // One step moves information by at most one cell, so step t of a T-step
  // segment (t = 1..T) updates only the tasks over the design boxes' bounding
  // box grown by T - t cells (+2 for the half-cell component offsets): every
  // cell of that region reads inputs from the previous step's larger region,
  // which were exact, so the recorded design history is the full replay's
  // (same kernel bodies per task, bit for bit).  Cells outside the region
  // keep stale values, which nothing reads before the next checkpoint load.
  const bool region_ok = h->replay_region && design && h->storage == kStoreF32 && !h->wrap &&
                         ((h->variant >= 1 && h->variant <= 3) || h->variant == kTileVariant);
  int dbox[6] = {INT_MAX, -1, INT_MAX, -1, INT_MAX, -1};
  for (int c = 0; c < 3; ++c) {
    const DesignBox& d = a.q.design[c];
    if (!d.grad) continue;
    for (int ax = 0; ax < 3; ++ax) {
      dbox[2 * ax] = std::min(dbox[2 * ax], d.lo[ax]);
      dbox[2 * ax + 1] = std::max(dbox[2 * ax + 1], d.hi[ax]);
    }
  }
  auto replay = [&](int s) -> int {
    NvtxRange seg("replay segment");
    const int n0 = s * stride, n1 = std::min(n_steps, n0 + stride);
    int r = fdtd_engine_checkpoint_load(h, s);
    if (r) return r;
    const AdjParams q = with_hist(s);
    StepParams p;
    fill_params(h, p);
    int err = design ? launch_design_record(p, q, 0, h->stream) : 0;
    if (err) return cuda_fail(static_cast<cudaError_t>(err), "design record");
    const int nn[3] = {h->NX, h->NY, h->NZ};
    for (int n = n0; n < n1; ++n) {
      if (region_ok) {
        const int m = (n1 - 1 - n) + 2;  // cells of dependence left after this step, plus the offsets
        int box[6];
        for (int ax = 0; ax < 3; ++ax) {
          box[2 * ax] = std::max(0, dbox[2 * ax] - m);
          box[2 * ax + 1] = std::min(nn[ax], dbox[2 * ax + 1] + m);
        }
        r = launch_step(h, n, -1, box);
      } else {
        r = launch_step(h, n, -1);
      }
      if (r) return r;
      if (design) {
        fill_params(h, p);
        err = launch_design_record(p, q, n + 1 - n0, h->stream);
        if (err) return cuda_fail(static_cast<cudaError_t>(err), "design record");
      }
    }
    CUDA_TRY(cudaEventRecord(a.ev_rep[s & 1], h->stream));
    return 0;
  };
  // the reverse stream starts after everything queued so far on the engine stream
  CUDA_TRY(cudaEventRecord(a.ev_rev[0], h->stream));
  CUDA_TRY(cudaStreamWaitEvent(a.rev, a.ev_rev[0], 0));
  rc = replay(S - 1);
  if (rc) return rc;
  StepParams p;
  fill_params(h, p);
  for (int s = S - 1; s >= 0; --s) {
    const int n0 = s * stride, n1 = std::min(n_steps, n0 + stride);
    CUDA_TRY(cudaStreamWaitEvent(a.rev, a.ev_rep[s & 1], 0));
    NvtxRange seg("reverse segment");
    const AdjParams qs = with_hist(s);
    for (int n = n1 - 1; n >= n0; --n) {
      AdjParams q = qs;
      q.hist_slot = design ? n - n0 : 0;
      const int err = launch_adjoint_step(p, q, h->d_flush, q.seed_re ? h->n_flush : 0, h->w_e, h->w_h, h->n_freq,
                                          n, a.rev);
      if (err) return cuda_fail(static_cast<cudaError_t>(err), "adjoint step");
    }
    CUDA_TRY(cudaEventRecord(a.ev_rev[s & 1], a.rev));
    if (s > 0) {
      // the history buffer of segment s - 1 was read by the reverse of segment s + 1
      if (s + 1 < S) CUDA_TRY(cudaStreamWaitEvent(h->stream, a.ev_rev[(s + 1) & 1], 0));
      rc = replay(s - 1);
      if (rc) return rc;
    }
  }
  CUDA_TRY(cudaStreamWaitEvent(h->stream, a.ev_rev[0], 0));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  a.replay_n0 = a.replay_n1 = -1;
  return check_status(h);
}

int fdtd_engine_adjoint_grad(fdtd_engine* h, int comp, float* out) {
  if (!h || !h->adj.ready || comp < 0 || comp > 2 || !out) return fail(FDTD_ERR_INVALID_ARG, "bad gradient read");
  const DesignBox& d = h->adj.q.design[comp];
  if (!d.grad) return fail(FDTD_ERR_STATE, "no design box for this component");
  CUDA_TRY(cudaMemcpyAsync(out, d.grad, sizeof(float) * d.cells, cudaMemcpyDefault, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return 0;
}

static int adj_geometry(fdtd_engine* h, int kind, int comp, int which, float** buf, int shape[3], int* py, int* pz,
                        int* zlo, int* zshift) {
  int ext[3];
  comp_extent(comp, h->NX, h->NY, h->NZ, ext);
  const int c = comp % 3;
  *zlo = kNoRemap;
  *zshift = 0;
  if (kind == 0) {
    *buf = comp < 3 ? h->adj.q.gE[c] : h->adj.q.gH[c];
    for (int ax = 0; ax < 3; ++ax) shape[ax] = ext[ax];
    *py = h->NY;
    *pz = h->P;
    return 1;
  }
  const int axis = which == 0 ? axis_a(c) : axis_b(c);
  const int L = h->desc.pml_lo[axis] + h->desc.pml_hi[axis];
  for (int ax = 0; ax < 3; ++ax) shape[ax] = ext[ax];
  shape[axis] = L;
  *buf = comp < 3 ? h->adj.q.gpsiE[c][which] : h->adj.q.gpsiH[c][which];
  *py = axis == 1 ? L : h->NY;
  *pz = axis == 2 ? h->SZ : h->P;
  if (axis == 2) zslab_remap(h, ext[2], zlo, zshift);
  return L;
}

// Adjoint pole state (kind 2): comp = pole id, which = 0 (adjoint of P) or 1 (adjoint of J);
// dense box-shaped [i][j][k] on the caller's side, z-padded rows in the engine.
static int adj_pole_copy(fdtd_engine* h, int id, int which, float* dst, const float* src) {
  if (id < 0 || id >= static_cast<int>(h->poles.size())) return fail(FDTD_ERR_INVALID_ARG, "bad pole id");
  const PoleHost& ph = h->poles[id];
  float* buf = which == 0 ? h->adj.gpol_host[id] : h->adj.gcur_host[id];
  const size_t w = ph.nk * sizeof(float), pitch = ph.nkk * sizeof(float);
  if (src)
    CUDA_TRY(cudaMemcpy2DAsync(buf + ph.koff, pitch, src, w, w, ph.rows, cudaMemcpyDefault, h->stream));
  else
    CUDA_TRY(cudaMemcpy2DAsync(dst, w, buf + ph.koff, pitch, w, ph.rows, cudaMemcpyDefault, h->stream));
  return 0;
}

int fdtd_engine_adjoint_pack(fdtd_engine* h, int kind, int comp, int which, const float* src) {
  if (h && h->adj.ready && kind == 2 && src && (which == 0 || which == 1))
    return adj_pole_copy(h, comp, which, nullptr, src);
  if (!h || !h->adj.ready || kind < 0 || kind > 1 || comp < 0 || comp > 5 || which < 0 || which > 1 || !src)
    return fail(FDTD_ERR_INVALID_ARG, "bad adjoint pack arguments");
  float* buf;
  int shape[3], py, pz;
  int zlo, zshift;
  if (adj_geometry(h, kind, comp, which, &buf, shape, &py, &pz, &zlo, &zshift) == 0) return 0;
  pack_kernel<<<1024, 256, 0, h->stream>>>(buf, src, shape[0], shape[1], shape[2], py, pz, zlo, zshift);
  CUDA_TRY(cudaGetLastError());
  return 0;
}

int fdtd_engine_adjoint_unpack(fdtd_engine* h, int kind, int comp, int which, float* dst) {
  if (h && h->adj.ready && kind == 2 && dst && (which == 0 || which == 1))
    return adj_pole_copy(h, comp, which, dst, nullptr);
  if (!h || !h->adj.ready || kind < 0 || kind > 1 || comp < 0 || comp > 5 || which < 0 || which > 1 || !dst)
    return fail(FDTD_ERR_INVALID_ARG, "bad adjoint unpack arguments");
  float* buf;
  int shape[3], py, pz;
  int zlo, zshift;
  if (adj_geometry(h, kind, comp, which, &buf, shape, &py, &pz, &zlo, &zshift) == 0) return 0;
  unpack_kernel<<<1024, 256, 0, h->stream>>>(dst, buf, shape[0], shape[1], shape[2], py, pz, zlo, zshift);
  CUDA_TRY(cudaGetLastError());
  return 0;
}

int fdtd_engine_get_launch(fdtd_engine* h, int* variant, int* tile_rows, int* chunk_planes) {
  if (!h) return fail(FDTD_ERR_INVALID_ARG, "null engine");
  if (variant) *variant = h->variant;
  if (tile_rows) *tile_rows = h->TY;
  if (chunk_planes) *chunk_planes = h->CX;
  return 0;
}

int fdtd_engine_info(fdtd_engine* h, int* tile_rows, int* chunk_planes, int* grid_x, int* grid_y, int* block,
                     int64_t* launches) {
  if (!h) return fail(FDTD_ERR_INVALID_ARG, "null engine");
  if (tile_rows) *tile_rows = h->TY;
  if (chunk_planes) *chunk_planes = h->CX;
  const dim3 g = step_grid(h);
  if (grid_x) *grid_x = static_cast<int>(g.x);
  if (grid_y) *grid_y = static_cast<int>(g.y * g.z);
  if (block) *block = tile_runs(h) ? tile_block_threads() : kWarpRows * 32;
  if (launches) *launches = h->launches;
  return 0;
}

int fdtd_engine_last_ms(fdtd_engine* h, float* ms) {
  if (!h || !ms) return fail(FDTD_ERR_INVALID_ARG, "bad arguments");
  *ms = h->last_ms;
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched scenes: independent engines stepped together.  A block of M steps
// (M = the engines' common monitor sample block) of every engine is captured
// once into one CUDA graph: each engine's launches go to its own stream forked
// from the batch stream, so the kernels of all scenes run concurrently and
// small scenes fill the GPU together.  The graph holds step indices relative
// to the block start; the block's base step is written to every engine's
// device-side base before each replay, so one graph serves the whole range.
// ---------------------------------------------------------------------------
namespace {
__global__ void set_bases_kernel(int* const* bases, int n, int value) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) *bases[i] = value;
}
}  // namespace

struct fdtd_batch {
  std::vector<fdtd_engine*> eng;
  cudaStream_t stream = nullptr;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> join;
  cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr;
  // capture origin: the batch stream may be the legacy default stream, on
  // which capture is not permitted
  cudaStream_t cap = nullptr;
  int** d_bases = nullptr;
  cudaGraphExec_t exec = nullptr;
  int M = 0;
  float last_ms = 0.0f;
  int64_t graph_launches = 0;
};

static void batch_release_graph(fdtd_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
}

// Capture one M-step block of every engine into b->exec.
static int batch_capture(fdtd_batch* b) {
  for (fdtd_engine* h : b->eng) {
    StepParams p;
    fill_params(h, p);
    const int rc = ensure_classified(h, p);
    if (rc) return rc;
  }
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  CUDA_TRY(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeRelaxed));
  int rc = 0;
  cudaError_t err = cudaEventRecord(b->fork, b->cap);
  for (size_t i = 0; i < b->eng.size() && err == cudaSuccess && rc == 0; ++i) {
    fdtd_engine* h = b->eng[i];
    err = cudaStreamWaitEvent(b->streams[i], b->fork, 0);
    if (err != cudaSuccess) break;
    const int64_t launches0 = h->launches;
    const int cur0 = h->cur, pending0 = h->pending, base0 = h->pending_base;
    h->stream = b->streams[i];
    h->graph_base = true;
    h->graph_n0 = 0;
    h->pending = 0;
    h->pending_base = 0;
    for (int s = 0; s < b->M && rc == 0; ++s) {
      rc = launch_step(h, s, h->n_samples > 0 ? h->pending : -1);
      if (h->n_samples > 0) ++h->pending;
    }
    if (rc == 0) rc = flush_samples(h);
    h->stream = b->stream;
    h->graph_base = false;
    h->launches = launches0;
    h->cur = cur0;  // M is even: the captured block returns the ping-pong to its start
    h->pending = pending0;
    h->pending_base = base0;
    if (rc == 0) err = cudaEventRecord(b->join[i], b->streams[i]);
    if (rc == 0 && err == cudaSuccess) err = cudaStreamWaitEvent(b->cap, b->join[i], 0);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(b->cap, &graph);
  if (rc || err != cudaSuccess || end != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    if (rc) return rc;
    return cuda_fail(err != cudaSuccess ? err : end, "batch capture");
  }
  const cudaError_t inst = cudaGraphInstantiate(&b->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (inst != cudaSuccess) {
    b->exec = nullptr;
    return cuda_fail(inst, "cudaGraphInstantiate");
  }
  return 0;
}

extern "C" {

int fdtd_batch_create(fdtd_engine* const* engines, int n, void* stream, fdtd_batch** out) {
  if (!engines || n < 1 || !out) return fail(FDTD_ERR_INVALID_ARG, "bad batch arguments");
  *out = nullptr;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  int M = -1;
  for (int i = 0; i < n; ++i) {
    fdtd_engine* h = engines[i];
    if (!h || !h->finalized) return fail(FDTD_ERR_STATE, "every batch engine must be finalized");
    if (h->stream != st) return fail(FDTD_ERR_INVALID_ARG, "batch engines must be created on the batch stream");
    if (M < 0) M = h->M;
    if (h->M != M) return fail(FDTD_ERR_INVALID_ARG, "batch engines need the same sample block");
    for (int k = 0; k < i; ++k)
      if (engines[k] == h) return fail(FDTD_ERR_INVALID_ARG, "an engine appears twice in the batch");
  }
  if (M % 2 != 0) return fail(FDTD_ERR_INVALID_ARG, "the batch step block (sample block) must be even");
  fdtd_batch* b = new fdtd_batch();
  b->eng.assign(engines, engines + n);
  b->stream = st;
  b->M = M;
  b->streams.resize(n, nullptr);
  b->join.resize(n, nullptr);
  cudaError_t err = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  if (err == cudaSuccess) err = cudaEventCreate(&b->ev0);
  if (err == cudaSuccess) err = cudaEventCreate(&b->ev1);
  if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
  for (int i = 0; i < n && err == cudaSuccess; ++i) {
    err = cudaStreamCreateWithFlags(&b->streams[i], cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming);
  }
  if (err == cudaSuccess) err = cudaMalloc(&b->d_bases, sizeof(int*) * n);
  if (err == cudaSuccess) {
    std::vector<int*> bases(n);
    for (int i = 0; i < n; ++i) bases[i] = engines[i]->d_base;
    err = cudaMemcpy(b->d_bases, bases.data(), sizeof(int*) * n, cudaMemcpyHostToDevice);
  }
  if (err != cudaSuccess) {
    const int rc = cuda_fail(err, "batch create");
    fdtd_batch_destroy(b);
    return rc;
  }
  *out = b;
  return 0;
}

int fdtd_batch_destroy(fdtd_batch* b) {
  if (!b) return 0;
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_release_graph(b);
  for (cudaStream_t s : b->streams)
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t e : b->join)
    if (e) cudaEventDestroy(e);
  if (b->cap) cudaStreamDestroy(b->cap);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  cudaFree(b->d_bases);
  delete b;
  return 0;
}

int fdtd_batch_autotune(fdtd_batch* b) {
  if (!b) return fail(FDTD_ERR_INVALID_ARG, "null batch");
  // One autotune per size class (node counts rounded to 32, CPML or not): the
  // class's first engine times the launch variants and chunk lengths, the
  // others take its pick.
  std::vector<std::pair<std::vector<int>, fdtd_engine*>> classes;
  for (fdtd_engine* h : b->eng) {
    const std::vector<int> key = {(h->NX + 16) / 32, (h->NY + 16) / 32, (h->NZ + 16) / 32, h->cpml ? 1 : 0};
    fdtd_engine* rep = nullptr;
    for (auto& c : classes)
      if (c.first == key) rep = c.second;
    if (!rep) {
      int ty = 0, cx = 0;
      const int rc = fdtd_engine_autotune(h, &ty, &cx);
      if (rc) return rc;
      classes.push_back({key, h});
    } else {
      const int rc = fdtd_engine_set_launch(h, rep->variant, 1, rep->CX);
      if (rc) return rc;
    }
  }
  batch_release_graph(b);
  return 0;
}

int fdtd_batch_step_range(fdtd_batch* b, int n0, int n1) {
  NvtxRange nvtx_range("fdtd_batch_step_range");
  if (!b) return fail(FDTD_ERR_INVALID_ARG, "null batch");
  if (n1 < n0 || n0 < 0) return fail(FDTD_ERR_INVALID_ARG, "bad step range");
  for (fdtd_engine* h : b->eng) {
    for (const auto& t : h->terms)
      if (t.signal && n1 > t.aux_len) return fail(FDTD_ERR_INVALID_ARG, "source signal table shorter than the range");
    for (const auto& l : h->lines)
      if (n1 > l.n_steps) return fail(FDTD_ERR_INVALID_ARG, "incident line history shorter than the range");
    if (h->n_samples > 0 && h->n_freq > 0 && n1 > h->dft_steps)
      return fail(FDTD_ERR_INVALID_ARG, "DFT weight table shorter than the range");
    if (h->stream != b->stream) return fail(FDTD_ERR_STATE, "a batch engine moved to another stream");
  }
  CUDA_TRY(cudaEventRecord(b->ev0, b->stream));
  // Monitor samples are flushed into the DFT sums in the same groups as
  // fdtd_engine_step_range would (every 32 steps and at the end of the range),
  // so a batch gives the spectra of the engines stepped one by one.  Samples
  // left pending by other calls, or engines whose pending counts differ, are
  // flushed first.
  bool aligned = true;
  for (fdtd_engine* h : b->eng) {
    if (h->pending > 0 && h->pending_base + h->pending != n0) {
      const int rc = flush_samples(h);
      if (rc) return rc;
    }
    aligned = aligned && h->pending == b->eng[0]->pending;
  }
  if (!aligned) {
    for (fdtd_engine* h : b->eng) {
      const int rc = flush_samples(h);
      if (rc) return rc;
    }
  }
  // direct launches of [from, to) for every engine, as in fdtd_engine_step_range
  auto direct = [&](int from, int to) -> int {
    for (fdtd_engine* h : b->eng) {
      for (int t = from; t < to; ++t) {
        if (h->pending == 0) h->pending_base = t;
        int rc = launch_step(h, t, h->pending);
        if (rc) return rc;
        if (h->n_samples > 0 && ++h->pending == h->M) {
          rc = flush_samples(h);
          if (rc) return rc;
        }
      }
    }
    return 0;
  };
  int n = n0;
  // complete a pending partial block first, so graph blocks start with no samples pending
  const int lead = b->eng[0]->pending > 0 ? std::min(n1 - n0, b->M - b->eng[0]->pending) : 0;
  if (lead > 0) {
    const int rc = direct(n, n + lead);
    if (rc) return rc;
    n += lead;
  }
  const int N = static_cast<int>(b->eng.size());
  bool empty = true;
  for (fdtd_engine* h : b->eng) empty = empty && h->pending == 0;
  while (empty && n + b->M <= n1) {
    if (!b->exec) {
      const int rc = batch_capture(b);
      if (rc) return rc;
    }
    set_bases_kernel<<<(N + 127) / 128, 128, 0, b->stream>>>(b->d_bases, N, n);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
    ++b->graph_launches;
    n += b->M;
    for (fdtd_engine* h : b->eng) h->pending_base = n;
  }
  {
    // tail steps (fewer than a block) run as direct launches
    const int rc = direct(n, n1);
    if (rc) return rc;
  }
  // as fdtd_engine_step_range: the DFT of every step of the range lands inside it
  for (fdtd_engine* h : b->eng) {
    const int rc = flush_samples(h);
    if (rc) return rc;
  }
  CUDA_TRY(cudaEventRecord(b->ev1, b->stream));
  CUDA_TRY(cudaEventSynchronize(b->ev1));
  CUDA_TRY(cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1));
  for (fdtd_engine* h : b->eng) {
    const int rc = check_status(h);
    if (rc) return rc;
  }
  return 0;
}

int fdtd_batch_last_ms(fdtd_batch* b, float* ms) {
  if (!b || !ms) return fail(FDTD_ERR_INVALID_ARG, "bad arguments");
  *ms = b->last_ms;
  return 0;
}

int fdtd_batch_info(fdtd_batch* b, int* n_engines, int* block_steps, int64_t* graph_launches) {
  if (!b) return fail(FDTD_ERR_INVALID_ARG, "null batch");
  if (n_engines) *n_engines = static_cast<int>(b->eng.size());
  if (block_steps) *block_steps = b->M;
  if (graph_launches) *graph_launches = b->graph_launches;
  return 0;
}


// ---------------------------------------------------------------------------
// Bloch pairs: a Bloch-periodic scene carries a complex field.  Its real and
// imaginary parts are two engines (same grid, coefficients and monitors; each
// holds the sources of its part); they evolve independently except on the
// Bloch faces, where the wrap kernel couples them through the phase e^{ikL}.
// ---------------------------------------------------------------------------
}  // extern "C"

struct fdtd_bloch {
  fdtd_engine* re = nullptr;
  fdtd_engine* im = nullptr;
  float pc[3] = {1, 1, 1}, ps[3] = {0, 0, 0};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.0f;
};

extern "C" {

int fdtd_bloch_create(fdtd_engine* re, fdtd_engine* im, const float* phase_cos, const float* phase_sin,
                      fdtd_bloch** out) {
  if (!re || !im || re == im || !phase_cos || !phase_sin || !out) return fail(FDTD_ERR_INVALID_ARG, "bad Bloch pair arguments");
  *out = nullptr;
  if (!re->finalized || !im->finalized) return fail(FDTD_ERR_STATE, "both engines must be finalized");
  if (re->in_pair || im->in_pair) return fail(FDTD_ERR_STATE, "an engine is already in a Bloch pair");
  if (!re->wrap) return fail(FDTD_ERR_INVALID_ARG, "the engines have no periodic or Bloch face");
  if (re->nl_general >= 0 || im->nl_general >= 0)
    return fail(FDTD_ERR_UNSUPPORTED, "nonlinear media on Bloch (complex) fields");
  const fdtd_grid_desc &a = re->desc, &b = im->desc;
  bool same = a.nx == b.nx && a.ny == b.ny && a.nz == b.nz && a.dt == b.dt && re->stream == im->stream && re->M == im->M &&
              re->storage == im->storage;
  for (int f = 0; f < 6; ++f) same = same && a.boundary[f] == b.boundary[f];
  for (int x = 0; x < 3; ++x) same = same && a.pml_lo[x] == b.pml_lo[x] && a.pml_hi[x] == b.pml_hi[x];
  if (!same) return fail(FDTD_ERR_INVALID_ARG, "the two channels need the same grid, boundaries, stream and sample block");
  if (re->variant > 3 || im->variant > 3) return fail(FDTD_ERR_UNSUPPORTED, "Bloch pairs run launch variants 1-3");
  fdtd_bloch* p = new fdtd_bloch();
  p->re = re;
  p->im = im;
  for (int x = 0; x < 3; ++x) {
    const bool bl = x < 2 && a.boundary[2 * x] == FDTD_BND_BLOCH;
    p->pc[x] = bl ? phase_cos[x] : 1.0f;
    p->ps[x] = bl ? phase_sin[x] : 0.0f;
  }
  cudaError_t err = cudaEventCreate(&p->ev0);
  if (err == cudaSuccess) err = cudaEventCreate(&p->ev1);
  if (err != cudaSuccess) {
    const int rc = cuda_fail(err, "Bloch pair events");
    fdtd_bloch_destroy(p);
    return rc;
  }
  re->in_pair = im->in_pair = true;
  *out = p;
  return 0;
}

int fdtd_bloch_destroy(fdtd_bloch* p) {
  if (!p) return 0;
  if (p->re) p->re->in_pair = false;
  if (p->im) p->im->in_pair = false;
  if (p->ev0) cudaEventDestroy(p->ev0);
  if (p->ev1) cudaEventDestroy(p->ev1);
  delete p;
  return 0;
}

int fdtd_bloch_step_range(fdtd_bloch* p, int n0, int n1) {
  NvtxRange nvtx_range("fdtd_bloch_step_range");
  if (!p) return fail(FDTD_ERR_INVALID_ARG, "null Bloch pair");
  if (n1 < n0 || n0 < 0) return fail(FDTD_ERR_INVALID_ARG, "bad step range");
  fdtd_engine* hs[2] = {p->re, p->im};
  for (fdtd_engine* h : hs) {
    for (const auto& t : h->terms)
      if (t.signal && n1 > t.aux_len) return fail(FDTD_ERR_INVALID_ARG, "source signal table shorter than the range");
    for (const auto& l : h->lines)
      if (n1 > l.n_steps) return fail(FDTD_ERR_INVALID_ARG, "incident line history shorter than the range");
    if (h->n_samples > 0 && h->n_freq > 0 && n1 > h->dft_steps)
      return fail(FDTD_ERR_INVALID_ARG, "DFT weight table shorter than the range");
  }
  const cudaStream_t st = p->re->stream;
  CUDA_TRY(cudaEventRecord(p->ev0, st));
  for (int n = n0; n < n1; ++n) {
    for (fdtd_engine* h : hs) {
      if (h->pending == 0) h->pending_base = n;
      if (h->pending_base + h->pending != n) {
        const int rc = flush_samples(h);
        if (rc) return rc;
        h->pending_base = n;
      }
      const int rc = launch_step(h, n, -1);  // step kernel only: the pair runs the wrap kernel
      if (rc) return rc;
    }
    StepParams pr, pim;
    fill_params(p->re, pr);
    fill_params(p->im, pim);
    WrapFields fr, fi;
    for (int c = 0; c < 3; ++c) {
      fr.eold[c] = p->re->E[1 - p->re->cur][c];
      fr.enew[c] = p->re->E[p->re->cur][c];
      fr.hnew[c] = p->re->H[p->re->cur][c];
      fi.eold[c] = p->im->E[1 - p->im->cur][c];
      fi.enew[c] = p->im->E[p->im->cur][c];
      fi.hnew[c] = p->im->H[p->im->cur][c];
    }
    const int err = launch_wrap_fixup(pr, &pim, fr, &fi, p->pc, p->ps, n, st, p->re->storage);
    if (err != 0) return cuda_fail(static_cast<cudaError_t>(err), "wrap_fixup_kernel launch");
    for (fdtd_engine* h : hs) {
      int rc = launch_gather(h, h->n_samples > 0 ? h->pending : -1);
      if (rc) return rc;
      if (h->n_samples > 0 && ++h->pending == h->M) {
        rc = flush_samples(h);
        if (rc) return rc;
      }
    }
  }
  // the DFT of every step of the range lands inside the range
  for (fdtd_engine* h : hs) {
    const int rc = flush_samples(h);
    if (rc) return rc;
  }
  CUDA_TRY(cudaEventRecord(p->ev1, st));
  CUDA_TRY(cudaEventSynchronize(p->ev1));
  CUDA_TRY(cudaEventElapsedTime(&p->last_ms, p->ev0, p->ev1));
  for (fdtd_engine* h : hs) {
    const int rc = check_status(h);
    if (rc) return rc;
  }
  return 0;
}

int fdtd_bloch_last_ms(fdtd_bloch* p, float* ms) {
  if (!p || !ms) return fail(FDTD_ERR_INVALID_ARG, "bad arguments");
  *ms = p->last_ms;
  return 0;
}

}  // extern "C"
