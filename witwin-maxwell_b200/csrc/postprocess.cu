// Consumers of the DFT planes on the GPU: the plane-wave (diffraction order)
// projection of a periodic plane's spectrum and the near-to-far-field radiation
// integral of equivalent surface currents.
//
// Diffraction (witwin/maxwell/postprocess/diffraction.py:84-196): for the order
// grid (m, n) with kx_m = ka + m Ga, ky_n = kb + n Gb, the amplitude of each
// field component is the mean over the plane of F(a, b) exp(-i (kx a + ky b)).
// The phase factors separate, so the projection runs as two passes:
//   S[n][a][c] = sum_b F_c(a, b) e^{-i ky_n b}        (one thread per (n, a, c))
//   A[m][n][c] = sum_a S[n][a][c] e^{-i kx_m a} / (Na Nb)   (one per (m, n, c))
// Sums and phases in FP64 (the plane holds up to ~10^6 samples).
//
// Near-to-far field (witwin/maxwell/postprocess/nfft.py:100-137): for each
// direction s the radiation vectors N = sum_p J_w(p) e^{-i k s.r_p} and
// L = sum_p M_w(p) e^{-i k s.r_p}, then
//   E = P (eta s x (s x N) + s x L),  H = P ((1/eta) s x (s x L) - s x N),
//   P = -i k e^{i k R} / (4 pi R),  power density = Re(E x H*) . s / 2.
// One thread per direction; the CTA stages tiles of points and weighted currents
// in shared memory (every thread reads every point), FP32 phases and FP64 sums.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "../../include/fdtd_b200.h"
#include "common.cuh"

namespace fdtdb200 {

namespace {

constexpr int kPpThreads = 256;
constexpr int kNfftTile = 256;

// S[n][a][c] (interleaved complex, FP64): sum over b.
__global__ void diffraction_rows_kernel(int na, int nb, const float* __restrict__ field, const float* __restrict__ cb,
                                        int n_n, const double* __restrict__ ky, double2* __restrict__ s) {
  const int64_t total = static_cast<int64_t>(n_n) * na * 3;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(t % 3);
    const int a = static_cast<int>((t / 3) % na);
    const int n = static_cast<int>(t / (3 * static_cast<int64_t>(na)));
    const double k = ky[n];
    double re = 0.0, im = 0.0;
    for (int b = 0; b < nb; ++b) {
      const int64_t x = ((static_cast<int64_t>(a) * nb + b) * 3 + c) * 2;
      const double fr = field[x], fi = field[x + 1];
      double sn, cs;
      sincos(-k * static_cast<double>(cb[b]), &sn, &cs);
      re += fr * cs - fi * sn;
      im += fr * sn + fi * cs;
    }
    s[t] = make_double2(re, im);
  }
}

// A[m][n][c] (interleaved complex, FP32 out): sum over a of S, scaled by 1 / (Na Nb).
__global__ void diffraction_orders_kernel(int na, int n_m, const double* __restrict__ kx, int n_n,
                                          const float* __restrict__ ca, const double2* __restrict__ s, double scale,
                                          float* __restrict__ out) {
  const int64_t total = static_cast<int64_t>(n_m) * n_n * 3;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(t % 3);
    const int n = static_cast<int>((t / 3) % n_n);
    const int m = static_cast<int>(t / (3 * static_cast<int64_t>(n_n)));
    const double k = kx[m];
    double re = 0.0, im = 0.0;
    for (int a = 0; a < na; ++a) {
      const double2 v = s[(static_cast<int64_t>(n) * na + a) * 3 + c];
      double sn, cs;
      sincos(-k * static_cast<double>(ca[a]), &sn, &cs);
      re += v.x * cs - v.y * sn;
      im += v.x * sn + v.y * cs;
    }
    out[2 * t] = static_cast<float>(re * scale);
    out[2 * t + 1] = static_cast<float>(im * scale);
  }
}

struct C3 {
  double r[3], i[3];
};

__device__ __forceinline__ C3 cross_real_complex(const double s[3], const C3& v) {
  C3 o;
  o.r[0] = s[1] * v.r[2] - s[2] * v.r[1];
  o.i[0] = s[1] * v.i[2] - s[2] * v.i[1];
  o.r[1] = s[2] * v.r[0] - s[0] * v.r[2];
  o.i[1] = s[2] * v.i[0] - s[0] * v.i[2];
  o.r[2] = s[0] * v.r[1] - s[1] * v.r[0];
  o.i[2] = s[0] * v.i[1] - s[1] * v.i[0];
  return o;
}

__global__ void __launch_bounds__(kPpThreads) nfft_kernel(int n_points, const float* __restrict__ points,
                                                           const float* __restrict__ jw, const float* __restrict__ mw,
                                                           int n_dirs, const float* __restrict__ dirs,
                                                           const float* __restrict__ radius, double k, double eta,
                                                           float* __restrict__ e_out, float* __restrict__ h_out,
                                                           float* __restrict__ power) {
  __shared__ float sp[kNfftTile][3];
  __shared__ float sj[kNfftTile][6];
  __shared__ float sm[kNfftTile][6];
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = d < n_dirs;
  double s[3] = {0.0, 0.0, 0.0};
  if (active) {
#pragma unroll
    for (int c = 0; c < 3; ++c) s[c] = dirs[3 * d + c];
  }
  const float kf = static_cast<float>(k);
  const float sx = static_cast<float>(s[0]), sy = static_cast<float>(s[1]), sz = static_cast<float>(s[2]);
  C3 N{}, L{};
  for (int p0 = 0; p0 < n_points; p0 += kNfftTile) {
    const int cnt = min(kNfftTile, n_points - p0);
    __syncthreads();
    for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
      for (int c = 0; c < 3; ++c) sp[q][c] = points[3 * (p0 + q) + c];
      for (int c = 0; c < 6; ++c) {
        sj[q][c] = jw[6 * (p0 + q) + c];
        sm[q][c] = mw[6 * (p0 + q) + c];
      }
    }
    __syncthreads();
    if (!active) continue;
    for (int q = 0; q < cnt; ++q) {
      // phase -k s.r in FP32 (|k r| stays within a few hundred radians on a monitor box)
      const float ph = -kf * (sx * sp[q][0] + sy * sp[q][1] + sz * sp[q][2]);
      float sn, cs;
      sincosf(ph, &sn, &cs);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float jr = sj[q][2 * c], ji = sj[q][2 * c + 1];
        const float mr = sm[q][2 * c], mi = sm[q][2 * c + 1];
        N.r[c] += static_cast<double>(jr * cs - ji * sn);
        N.i[c] += static_cast<double>(jr * sn + ji * cs);
        L.r[c] += static_cast<double>(mr * cs - mi * sn);
        L.i[c] += static_cast<double>(mr * sn + mi * cs);
      }
    }
  }
  if (!active) return;
  const C3 sN = cross_real_complex(s, N), sL = cross_real_complex(s, L);
  const C3 ssN = cross_real_complex(s, sN), ssL = cross_real_complex(s, sL);
  // P = -i k e^{i k R} / (4 pi R)
  const double R = radius[d];
  double sn, cs;
  sincos(k * R, &sn, &cs);
  const double amp = k / (4.0 * 3.141592653589793 * R);
  const double pr = amp * sn, pi = -amp * cs;  // -i (cos + i sin) = sin - i cos
  C3 E, H;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double er = eta * ssN.r[c] + sL.r[c], ei = eta * ssN.i[c] + sL.i[c];
    const double hr = ssL.r[c] / eta - sN.r[c], hi = ssL.i[c] / eta - sN.i[c];
    E.r[c] = pr * er - pi * ei;
    E.i[c] = pr * ei + pi * er;
    H.r[c] = pr * hr - pi * hi;
    H.i[c] = pr * hi + pi * hr;
    e_out[6 * d + 2 * c] = static_cast<float>(E.r[c]);
    e_out[6 * d + 2 * c + 1] = static_cast<float>(E.i[c]);
    h_out[6 * d + 2 * c] = static_cast<float>(H.r[c]);
    h_out[6 * d + 2 * c + 1] = static_cast<float>(H.i[c]);
  }
  // Re(E x conj(H)) . s / 2
  double pw = 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int a = (c + 1) % 3, b = (c + 2) % 3;
    const double re = (E.r[a] * H.r[b] + E.i[a] * H.i[b]) - (E.r[b] * H.r[a] + E.i[b] * H.i[a]);
    pw += 0.5 * re * s[c];
  }
  power[d] = static_cast<float>(pw);
}

int pp_fail(const char* msg) {
  set_last_error(msg);
  return FDTD_ERR_INVALID_ARG;
}

int pp_check(const char* what) {
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    set_last_error(std::string(what) + ": " + cudaGetErrorString(err));
    return FDTD_ERR_CUDA;
  }
  return 0;
}

unsigned pp_blocks(int64_t n) {
  int64_t b = (n + kPpThreads - 1) / kPpThreads;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return static_cast<unsigned>(b);
}

}  // namespace

}  // namespace fdtdb200

using namespace fdtdb200;

extern "C" int fdtd_pp_diffraction(int na, int nb, const float* coords_a, const float* coords_b, const float* field,
                                   int n_m, const double* kx, int n_n, const double* ky, double* scratch,
                                   float* amplitudes, void* stream) {
  if (na <= 0 || nb <= 0 || n_m <= 0 || n_n <= 0 || !coords_a || !coords_b || !field || !kx || !ky || !scratch ||
      !amplitudes)
    return pp_fail("diffraction: bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double2* s = reinterpret_cast<double2*>(scratch);
  diffraction_rows_kernel<<<pp_blocks(static_cast<int64_t>(n_n) * na * 3), kPpThreads, 0, st>>>(
      na, nb, field, coords_b, n_n, ky, s);
  diffraction_orders_kernel<<<pp_blocks(static_cast<int64_t>(n_m) * n_n * 3), kPpThreads, 0, st>>>(
      na, n_m, kx, n_n, coords_a, s, 1.0 / (static_cast<double>(na) * nb), amplitudes);
  return pp_check("diffraction");
}

extern "C" int fdtd_pp_nfft(int n_points, const float* points, const float* j_weighted, const float* m_weighted,
                            int n_dirs, const float* directions, const float* radius, double k, double eta,
                            float* e_out, float* h_out, float* power, void* stream) {
  if (n_points <= 0 || n_dirs <= 0 || !points || !j_weighted || !m_weighted || !directions || !radius || !e_out ||
      !h_out || !power || !(k > 0.0) || !(eta > 0.0))
    return pp_fail("nfft: bad arguments");
  const unsigned blocks = static_cast<unsigned>((n_dirs + kPpThreads - 1) / kPpThreads);
  nfft_kernel<<<blocks, kPpThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      n_points, points, j_weighted, m_weighted, n_dirs, directions, radius, k, eta, e_out, h_out, power);
  return pp_check("nfft");
}
