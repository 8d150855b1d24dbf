/*
 * CPU oracle for the FDTD time-stepping hot path (test infrastructure only).
 *
 * This file restates, in plain C, the arithmetic of the reference's per-op
 * FDTD kernels so that the CUDA product can be checked against an independent
 * CPU implementation.  It is compiled twice: with -DREAL=double (the FP64
 * accuracy oracle) and with -DREAL=float (the FP32 restatement used as the CPU
 * baseline).  Only tests, smoke() and the benchmark's CPU-baseline leg load it;
 * nothing in the product path links or calls it.
 *
 * Volume functions take an [i_begin, i_end) plane range (or an element range)
 * so that a caller can split the work across host threads.
 *
 * Every function cites the reference source it restates (paths are relative to
 * the witwin-maxwell project root).  Layout: C-contiguous [X][Y][Z] arrays,
 * z fastest (witwin/maxwell/fdtd/cuda/kernels/common.cuh:61-63).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#ifndef REAL
#define REAL double
#endif
typedef REAL real;

#define OFF(i, j, k, ny, nz) ((((int64_t)(i)) * (ny) + (j)) * (int64_t)(nz) + (k))

enum { BND_NONE = 0, BND_PML = 1, BND_PERIODIC = 2, BND_BLOCH = 3, BND_PEC = 4, BND_PMC = 5 };

int oracle_real_size(void) { return (int)sizeof(real); }

/* ------------------------------------------------------------------------- */
/* Magnetic update (witwin/maxwell/fdtd/cuda/kernels/magnetic.cu:20-212;      */
/* tests/fdtd/cuda/torch_reference.py:269-580).                               */
/*                                                                            */
/* comp 0 = Hx: a-axis y (second = Ez), b-axis z (first = Ey), curl = a - b   */
/* comp 1 = Hy: a-axis x (second = Ez), b-axis z (first = Ex), curl = b - a   */
/* comp 2 = Hz: a-axis x (second = Ey), b-axis y (first = Ex), curl = a - b   */
/* mode 0: standard; 1: dense CPML psi; 2: slab-compressed CPML psi.          */
/* Forward differences: second has +1 extent along a, first +1 along b.       */
/* ------------------------------------------------------------------------- */
static int comp_axis_a(int comp) { return comp == 0 ? 1 : 0; }
static int comp_axis_b(int comp) { return comp == 2 ? 1 : 2; }

static int compact_local(int coord, int low, int hstart, int hlen) {
  /* witwin/maxwell/fdtd/cuda/kernels/common.cuh:65-78 */
  if (coord < low) return coord;
  if (coord >= hstart && coord < hstart + hlen) return low + coord - hstart;
  return -1;
}

static int64_t compact_offset(int axis, int i, int j, int k, int ny, int nz, int local, int clen) {
  /* witwin/maxwell/fdtd/cuda/kernels/common.cuh:80-96 */
  if (axis == 0) return OFF(local, j, k, ny, nz);
  if (axis == 1) return OFF(i, local, k, clen, nz);
  return OFF(i, j, local, ny, clen);
}

static real psi_step(real *psi, const real *b, const real *c, int mode, int axis, int i, int j, int k,
                     int ny, int nz, int coord, int low, int hstart, int hlen, real deriv, int write) {
  int64_t off;
  if (mode == 1) {
    off = OFF(i, j, k, ny, nz);
  } else {
    int local = compact_local(coord, low, hstart, hlen);
    if (local < 0) return (real)0;
    off = compact_offset(axis, i, j, k, ny, nz, local, low + hlen);
  }
  real v = b[coord] * psi[off] + c[coord] * deriv;
  if (write) psi[off] = v;
  return v;
}

void oracle_h_update(int i_begin, int i_end, int comp, int mode, int nx, int ny, int nz, real *field, const real *first,
                     const real *second, const real *decay, const real *curl, const real *inv_a,
                     const real *inv_b, real *psi_a, real *psi_b, const real *ika, const real *ba,
                     const real *ca, const real *ikb, const real *bb, const real *cb, int a_low,
                     int a_hstart, int a_hlen, int b_low, int b_hstart, int b_hlen) {
  const int A = comp_axis_a(comp), B = comp_axis_b(comp);
  /* shapes of the sources */
  const int sy2 = ny + (A == 1), sz2 = nz + (A == 2); /* second: +1 along A */
  const int sy1 = ny + (B == 1), sz1 = nz + (B == 2); /* first: +1 along B */
  for (int i = i_begin; i < i_end && i < nx; ++i) {
    for (int j = 0; j < ny; ++j) {
      for (int k = 0; k < nz; ++k) {
        const int64_t lin = OFF(i, j, k, ny, nz);
        const int ca_ = A == 0 ? i : (A == 1 ? j : k);
        const int cb_ = B == 0 ? i : (B == 1 ? j : k);
        const int64_t s0 = OFF(i, j, k, sy2, sz2);
        const int64_t s1 = OFF(i + (A == 0), j + (A == 1), k + (A == 2), sy2, sz2);
        const int64_t f0 = OFF(i, j, k, sy1, sz1);
        const int64_t f1 = OFF(i + (B == 0), j + (B == 1), k + (B == 2), sy1, sz1);
        const real da = (second[s1] - second[s0]) * inv_a[ca_];
        const real db = (first[f1] - first[f0]) * inv_b[cb_];
        real ea = da, eb = db;
        if (mode != 0) {
          const real pa = psi_step(psi_a, ba, ca, mode, A, i, j, k, ny, nz, ca_, a_low, a_hstart, a_hlen, da, 1);
          const real pb = psi_step(psi_b, bb, cb, mode, B, i, j, k, ny, nz, cb_, b_low, b_hstart, b_hlen, db, 1);
          ea = da * ika[ca_] + pa;
          eb = db * ikb[cb_] + pb;
        }
        const real c = comp == 1 ? (eb - ea) : (ea - eb);
        field[lin] = field[lin] * decay[lin] - curl[lin] * c;
      }
    }
  }
}

/* ------------------------------------------------------------------------- */
/* Electric update with boundary-mode-aware backward differences               */
/* (witwin/maxwell/fdtd/cuda/kernels/electric.cu:18-119, 242-311, 462-553,     */
/* 647-941; tests/fdtd/cuda/torch_reference.py:152-230, 581-960, 1102-1275).  */
/*                                                                            */
/* comp 0 = Ex: a-axis y (second = Hz), b-axis z (first = Hy), curl = a - b   */
/* comp 1 = Ey: a-axis x (second = Hz), b-axis z (first = Hx), curl = b - a   */
/* comp 2 = Ez: a-axis x (second = Hy), b-axis y (first = Hx), curl = a - b   */
/* Sources have extent size-1 along the difference axis.                      */
/* ------------------------------------------------------------------------- */
static real bdiff(const real *src, int axis, int i, int j, int k, int tsize, int sy, int sz, int low_mode,
                  int high_mode, const real *inv) {
  const int coord = axis == 0 ? i : (axis == 1 ? j : k);
  const int ssize = tsize - 1;
  const real iv = inv[coord];
  if (coord == 0 || coord + 1 == tsize) {
    const int64_t lo = axis == 0 ? OFF(0, j, k, sy, sz) : (axis == 1 ? OFF(i, 0, k, sy, sz) : OFF(i, j, 0, sy, sz));
    const int64_t hi = axis == 0 ? OFF(ssize - 1, j, k, sy, sz)
                                 : (axis == 1 ? OFF(i, ssize - 1, k, sy, sz) : OFF(i, j, ssize - 1, sy, sz));
    if (coord == 0) {
      if (low_mode == BND_PERIODIC) return (src[lo] - src[hi]) * iv;
      if (low_mode == BND_PMC) return (real)2 * src[lo] * iv;
      return (real)0;
    }
    if (high_mode == BND_PERIODIC) return (src[lo] - src[hi]) * iv;
    if (high_mode == BND_PMC) return (real)(-2) * src[hi] * iv;
    return (real)0;
  }
  const int64_t cur = OFF(i, j, k, sy, sz);
  const int64_t prv = axis == 0 ? OFF(i - 1, j, k, sy, sz) : (axis == 1 ? OFF(i, j - 1, k, sy, sz) : OFF(i, j, k - 1, sy, sz));
  return (src[cur] - src[prv]) * iv;
}

static int is_pec(int coord, int size, int lo, int hi) {
  return (coord == 0 && lo == BND_PEC) || (coord + 1 == size && hi == BND_PEC);
}
static int is_inactive(int coord, int size, int lo, int hi) {
  const int l = coord == 0 && (lo == BND_NONE || lo == BND_PML);
  const int h = coord + 1 == size && (hi == BND_NONE || hi == BND_PML);
  return l || h;
}

void oracle_e_update(int i_begin, int i_end, int comp, int mode, int nx, int ny, int nz, real *field, const real *first,
                     const real *second, const real *decay, const real *curl, const real *inv_a,
                     const real *inv_b, int a_lo, int a_hi, int b_lo, int b_hi, real *psi_a, real *psi_b,
                     const real *ika, const real *ba, const real *ca, const real *ikb, const real *bb,
                     const real *cb, int a_low, int a_hstart, int a_hlen, int b_low, int b_hstart, int b_hlen) {
  const int A = comp_axis_a(comp), B = comp_axis_b(comp);
  const int sy2 = ny - (A == 1), sz2 = nz - (A == 2); /* second: -1 along A */
  const int sy1 = ny - (B == 1), sz1 = nz - (B == 2); /* first: -1 along B */
  const int size_a = A == 0 ? nx : (A == 1 ? ny : nz);
  const int size_b = B == 0 ? nx : (B == 1 ? ny : nz);
  for (int i = i_begin; i < i_end && i < nx; ++i) {
    for (int j = 0; j < ny; ++j) {
      for (int k = 0; k < nz; ++k) {
        const int64_t lin = OFF(i, j, k, ny, nz);
        const int ca_ = A == 0 ? i : (A == 1 ? j : k);
        const int cb_ = B == 0 ? i : (B == 1 ? j : k);
        if (is_pec(ca_, size_a, a_lo, a_hi) || is_pec(cb_, size_b, b_lo, b_hi)) {
          field[lin] = (real)0;
          continue;
        }
        if (is_inactive(ca_, size_a, a_lo, a_hi) || is_inactive(cb_, size_b, b_lo, b_hi)) continue;
        const real da = bdiff(second, A, i, j, k, size_a, sy2, sz2, a_lo, a_hi, inv_a);
        const real db = bdiff(first, B, i, j, k, size_b, sy1, sz1, b_lo, b_hi, inv_b);
        real ea = da, eb = db;
        if (mode != 0) {
          const real pa = psi_step(psi_a, ba, ca, mode, A, i, j, k, ny, nz, ca_, a_low, a_hstart, a_hlen, da, 1);
          const real pb = psi_step(psi_b, bb, cb, mode, B, i, j, k, ny, nz, cb_, b_low, b_hstart, b_hlen, db, 1);
          ea = da * ika[ca_] + pa;
          eb = db * ikb[cb_] + pb;
        }
        const real c = comp == 1 ? (eb - ea) : (ea - eb);
        field[lin] = field[lin] * decay[lin] + curl[lin] * c;
      }
    }
  }
}

/* ------------------------------------------------------------------------- */
/* ADE polarisation currents over elements [x0, n) (witwin/maxwell/fdtd/cuda/kernels/dispersive.cu:  */
/* 18-83; templates witwin/maxwell/fdtd/runtime/materials.py:530-589).         */
/* ------------------------------------------------------------------------- */
void oracle_debye(int64_t x0, int64_t n, const real *e, const real *drive, real decay, real dt, real *p, real *j) {
  for (int64_t x = x0; x < n; ++x) {
    const real prev = p[x];
    const real next = decay * prev + drive[x] * e[x];
    p[x] = next;
    j[x] = (next - prev) / dt;
  }
}

void oracle_drude(int64_t x0, int64_t n, const real *e, const real *drive, real decay, real *j) {
  for (int64_t x = x0; x < n; ++x) j[x] = decay * j[x] + drive[x] * e[x];
}

void oracle_lorentz(int64_t x0, int64_t n, const real *e, const real *drive, real decay, real restoring, real dt, real *p,
                    real *j) {
  for (int64_t x = x0; x < n; ++x) {
    const real nj = decay * j[x] - restoring * p[x] + drive[x] * e[x];
    j[x] = nj;
    p[x] = p[x] + dt * nj;
  }
}

void oracle_apply_polarization(int64_t x0, int64_t n, const real *j, const real *inv_eps, real dt, real *e) {
  for (int64_t x = x0; x < n; ++x) e[x] -= dt * j[x] * inv_eps[x];
}

/* ------------------------------------------------------------------------- */
/* Soft source patch add (witwin/maxwell/fdtd/cuda/kernels/sources.cu:135-154; */
/* out-of-range cells are skipped, torch_reference.py:1450-1483).              */
/* ------------------------------------------------------------------------- */
void oracle_add_patch(int fx, int fy, int fz, real *field, int px, int py, int pz, const real *patch, int oi,
                      int oj, int ok, real signal) {
  for (int i = 0; i < px; ++i)
    for (int j = 0; j < py; ++j)
      for (int k = 0; k < pz; ++k) {
        const int gi = oi + i, gj = oj + j, gk = ok + k;
        if (gi < 0 || gj < 0 || gk < 0 || gi >= fx || gj >= fy || gk >= fz) continue;
        field[OFF(gi, gj, gk, fy, fz)] += signal * patch[OFF(i, j, k, py, pz)];
      }
}

/* TFSF scaled line patch: value = coeff * incident[sample_index[axis coord]] * scale
 * (witwin/maxwell/fdtd/cuda/kernels/sources.cu:485-545; torch_reference.py:1738-1756). */
void oracle_add_line_patch(int fx, int fy, int fz, real *field, int px, int py, int pz, const real *coeff,
                           const real *incident, const int64_t *sample_idx, int axis, int oi, int oj, int ok,
                           real scale) {
  for (int i = 0; i < px; ++i)
    for (int j = 0; j < py; ++j)
      for (int k = 0; k < pz; ++k) {
        const int gi = oi + i, gj = oj + j, gk = ok + k;
        if (gi < 0 || gj < 0 || gk < 0 || gi >= fx || gj >= fy || gk >= fz) continue;
        const int a = axis == 0 ? i : (axis == 1 ? j : k);
        field[OFF(gi, gj, gk, fy, fz)] += coeff[OFF(i, j, k, py, pz)] * incident[sample_idx[a]] * scale;
      }
}

/* ------------------------------------------------------------------------- */
/* 1-D auxiliary incident grid (witwin/maxwell/fdtd/cuda/kernels/sources.cu:   */
/* 803-839; torch_reference.py:1944-1961).                                     */
/* ------------------------------------------------------------------------- */
void oracle_aux_magnetic(int ne, real *h, const real *e, const real *hdecay, const real *hcurl) {
  for (int x = 0; x < ne - 1; ++x) h[x] = hdecay[x] * h[x] - hcurl[x] * (e[x + 1] - e[x]);
}

void oracle_aux_electric(int ne, real *e, const real *h, const real *edecay, const real *ecurl, int src_index,
                         real src_value) {
  for (int x = 1; x < ne - 1; ++x) {
    if (x == src_index) continue;
    e[x] = edecay[x] * e[x] - ecurl[x] * (h[x] - h[x - 1]);
  }
  /* the source cell first, then the last cell pinned to zero: the reference's
     kernel checks the last cell before the source cell (sources.cu:829-835) */
  if (src_index >= 0 && src_index < ne) e[src_index] = src_value;
  if (ne > 0) e[ne - 1] = (real)0;
}

/* ------------------------------------------------------------------------- */
/* Running DFT accumulation (witwin/maxwell/fdtd/cuda/kernels/observers.cu:    */
/* 7-78, spectral.cu:9-146; torch_reference.py:1964-2016).                     */
/* ------------------------------------------------------------------------- */
void oracle_point_observers(int fy, int fz, const real *field, int npts, const int *pi, const int *pj,
                            const int *pk, real *re, real *im, real wcos, real wsin) {
  for (int p = 0; p < npts; ++p) {
    const real v = field[OFF(pi[p], pj[p], pk[p], fy, fz)];
    re[p] += v * wcos;
    im[p] += v * wsin;
  }
}

void oracle_plane_observer(int fx, int fy, int fz, const real *field, int axis, int index, real *re, real *im,
                           real wcos, real wsin) {
  if (axis == 0) {
    for (int j = 0; j < fy; ++j)
      for (int k = 0; k < fz; ++k) {
        const real v = field[OFF(index, j, k, fy, fz)];
        re[j * fz + k] += v * wcos;
        im[j * fz + k] += v * wsin;
      }
  } else if (axis == 1) {
    for (int i = 0; i < fx; ++i)
      for (int k = 0; k < fz; ++k) {
        const real v = field[OFF(i, index, k, fy, fz)];
        re[i * fz + k] += v * wcos;
        im[i * fz + k] += v * wsin;
      }
  } else {
    for (int i = 0; i < fx; ++i)
      for (int j = 0; j < fy; ++j) {
        const real v = field[OFF(i, j, index, fy, fz)];
        re[i * fy + j] += v * wcos;
        im[i * fy + j] += v * wsin;
      }
  }
}

void oracle_dft_volume(int64_t x0, int64_t x1, int64_t n, int nf, const real *field, real *re, real *im, const real *wcos,
                       const real *wsin) {
  for (int64_t x = x0; x < x1 && x < n; ++x) {
    const real v = field[x];
    for (int f = 0; f < nf; ++f) {
      re[(int64_t)f * n + x] += v * wcos[f];
      im[(int64_t)f * n + x] += v * wsin[f];
    }
  }
}

/* ------------------------------------------------------------------------- */
/* PEC face clamp (witwin/maxwell/fdtd/cuda/kernels/boundary.cu:69-168).       */
/* ------------------------------------------------------------------------- */
void oracle_clamp_face(int fx, int fy, int fz, real *field, int axis, int side) {
  const int n[3] = {fx, fy, fz};
  const int idx = side == 0 ? 0 : n[axis] - 1;
  for (int i = 0; i < fx; ++i)
    for (int j = 0; j < fy; ++j)
      for (int k = 0; k < fz; ++k) {
        const int c = axis == 0 ? i : (axis == 1 ? j : k);
        if (c == idx) field[OFF(i, j, k, fy, fz)] = (real)0;
      }
}
