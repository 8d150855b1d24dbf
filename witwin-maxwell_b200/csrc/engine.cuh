// Internal data structures of the fused FDTD step engine.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "common.cuh"

namespace fdtdb200 {

// A dense patch over an axis-aligned box of one field component that is added
// to that component every step.  The added value is coeff[cell] * s, where s is
// either signal[n] (a soft source whose waveform the host evaluated in FP64) or
// aux_hist[n * aux_len + sample_index[coord along sample_axis]] (a TFSF face
// correction that reads the 1-D incident line).
struct InjectionTerm {
  int comp;  // 0..2 = Ex..Ez (applied in the E phase), 3..5 = Hx..Hz (H phase)
  int i0, i1, j0, j1, k0, k1;
  const float* coeff;     // [i1-i0][j1-j0][k1-k0]
  const float* signal;    // per-step scalar table, or nullptr
  const float* aux_hist;  // per-step incident line history, or nullptr
  const int* sample_index;
  int aux_len;
  int sample_axis;
  float scale;
};

// One Debye/Drude/Lorentz pole acting on one E component over a box.
struct PoleTerm {
  int comp;  // 0..2
  int kind;  // 0 Debye, 1 Drude, 2 Lorentz
  int i0, i1, j0, j1, k0, k1;
  // z range of the stored arrays: [kk0, kk0 + nkk) with kk0 = k0 rounded down
  // and kk0 + nkk = k1 rounded up to multiples of four; the padding cells have
  // zero drive and zero 1/eps, so their state stays zero.
  int kk0, nkk;
  float decay, restoring, dt, inv_dt;
  const float* drive;    // [i1-i0][j1-j0][nkk]
  const float* inv_eps;  // same layout (1/eps of the component, absolute)
  float* pol;            // same layout: polarisation (Debye, Lorentz)
  float* cur;            // same layout: current
};

// One monitor region in flush order: slots [base, base + count) of component
// comp (0..5) over the box starting at (i0, j0, k0) with nj x nk cells per plane.
struct RegionFlush {
  int64_t base;
  int64_t count;
  int is_h;
  int comp;
  int i0, j0, k0, nj, nk;
};

// A box of one component whose values are written into the per-step sample
// ring buffer that feeds the batched monitor DFT.
struct SampleRegion {
  int comp;  // 0..5
  int i0, i1, j0, j1, k0, k1;
  int64_t base;  // first sample slot of the region
};

// Per-axis CSR index of thin boxes: an item is listed along the axis where it
// is thinnest (x: per plane i, y: per row j, z: per cell k), so a lane visits
// only items that can contain its plane, row or z cell.
struct BoxIndex {
  const int* ptr[3];
  const int* ids[3];
};

struct StepParams {
  int NX, NY, NZ, P, SZ;  // node counts, padded z pitch, z-slab row length
  int TY, CX, Q, ROWS;    // tile rows, planes per chunk, float4 per row, thread rows (TY + 2)
  int pf_dist;            // L2 prefetch distance of the x march in planes (0: none)
  const float* Ein[3];
  float* Eout[3];
  const float* Hin[3];
  float* Hout[3];
  const float* ecurl[3];
  const float* edecay[3];
  float ecurl_u[3], edecay_u[3];
  const float* hcurl[3];
  const float* hdecay[3];
  float hcurl_u[3], hdecay_u[3];
  const float* inv_e[3];
  const float* inv_h[3];
  float inv_e_u[3], inv_h_u[3];  // uniform-grid values (used when every entry of an axis is equal)
  int uniform_grid;              // every axis has constant spacing (inv_*_u hold the values)
  const float* eb[3];
  const float* ec[3];
  const float* eik[3];
  const float* hb[3];
  const float* hc[3];
  const float* hik[3];
  int slab_lo[3], slab_hi[3];
  // z-slab psi rows hold the low slab at [0, zlo4) and the high slab cells
  // k >= zhs4 at zlo4 + k - zhs4 (both segment starts multiples of four, so a
  // vector lane group maps to contiguous aligned storage); row length SZ.
  int zlo4, zhs4;
  float* psiE[3][2];
  const float* psiHin[3][2];
  float* psiHout[3][2];
  int bnd[6];
  int cpml;
  // injection / ADE / sampling
  const InjectionTerm* terms;
  BoxIndex term_index[2];  // [0] E-phase terms, [1] H-phase terms
  int n_terms[2];
  const PoleTerm* poles;
  const int* pole_plane_ptr;  // [NX + 1] CSR over planes
  const int* pole_plane_ids;
  int n_poles;
  const SampleRegion* regions;
  BoxIndex region_index[2];  // [0] E regions, [1] H regions
  int n_regions[2];
  float* samples;  // [M][n_samples]
  int64_t n_samples;
  int sample_block;  // M
  // Per-plane activity bits (kPlane* flags): which x-indexed lists hold items
  // for plane i.  Lets a warp skip every lookup on planes that have none.
  const unsigned* plane_bits;
  // Per-warp feature class (kClass* bits) of each warp task, indexed
  // [(chunk * kblocks + kblock) * NY + j]; built by launch_classify for the
  // current chunk length.
  const unsigned char* warp_class;
  // Field storage: kStoreF32, kStoreF16 or kStoreBF16 (E, H arrays hold that
  // type; ADE pole state is BF16 with BF16 fields, FP32 otherwise).  A stored field
  // value x of component c (0..2 Ex..Ez, 3..5 Hx..Hz) means x * fscale[c];
  // finv[c] = 1 / fscale[c].  Scales are powers of two, so the FP32 path and the
  // round trip through storage lose nothing beyond the storage rounding.
  int storage;
  float fscale[6], finv[6];
  // When set, the step index of a launch is *step_base + n (graph-captured
  // step blocks whose base step is written before each replay); else n.
  const int* step_base;
  // Device status word: a kernel whose bounded wait ran out stores
  // FDTD_ERR_TIMEOUT here (read back by the host after stepping).
  int* status;
  // Polling rounds of a bounded pipeline wait before it gives up and reports
  // FDTD_ERR_TIMEOUT (fdtd_engine_set_wait_limit; the default is 1 << 20).
  int wait_limit;
  // Warp kernel only: run just the CTAs (8 rows, one z block, one x chunk)
  // in which some warp task has the CPML class; the row-tile kernel runs the
  // others (launch variant 10 on scenes with CPML).
  int shell_only;
  // PMC faces, bit f for face f (x_lo, x_hi, y_lo, y_hi, z_lo, z_hi): the
  // tangential E on such a face is updated with the difference across it
  // doubled (the mirrored H outside is minus the H inside, electric.cu:18-119).
  int pmc;
  // 1: tangential E on PEC faces is zeroed after the source terms and the ADE
  // correction (the reference enforces PEC faces last in scenes without TFSF,
  // witwin/maxwell/fdtd/runtime/stepping.py:2316-2318); with TFSF the
  // corrections and sources added after the update stay (0).
  int pec_clamp;
  // Bounding box [nl_lo, nl_hi) (node indices) of the cells whose E
  // coefficients an instantaneous nonlinearity rewrites before every step:
  // warp tasks whose footprint meets it read the coefficient arrays whatever
  // the values at classification time (empty: nl_lo[0] >= nl_hi[0]).
  int nl_lo[3], nl_hi[3];
  // Warp kernels: the launch grid covers row blocks, z blocks and x chunks
  // starting at (rb0, kb0, ch0) of the full task grid, whose z-block count is
  // n_kb (the class table's layout); 0, 0, 0 and gridDim.y for a full launch.
  int rb0, kb0, ch0, n_kb;
};

// A warp task needs the CPML code (some cell of its footprint lies in a slab)
// or the coefficient arrays (some coefficient of its footprint differs from
// the component's background value).
constexpr unsigned kClassCpml = 1u;
constexpr unsigned kClassCoef = 2u;

// Fill p.warp_class (out) for chunk length p.CX: one warp per task.
int launch_classify(const StepParams& p, int n_kblocks, int n_chunks, unsigned char* out, cudaStream_t stream);

// Wrap faces (periodic / Bloch axes): the new-E output, old-E and new-H
// inputs of one field channel after its step kernel, for the wrap kernel
// (bloch.cu) that updates the E cells the step kernel defers.
struct WrapFields {
  const float* eold[3];
  float* enew[3];
  const float* hnew[3];
};
int64_t wrap_cell_count(const StepParams& p);
// Pole table of the ADE pass (ade_pass.cu), passed in the kernel parameters.
constexpr int kAdeMaxPoles = 32;
constexpr int kAdeCellsPerLane = 4;  // a tile is 32 * kAdeCellsPerLane z cells of one row
struct AdePole {
  int comp, kind;
  int i0, j0, nj;  // box origin and row count (j1 - j0)
  int k0, k1;      // cells of the box along z
  int kk0, nkk;    // stored z range (PoleTerm)
  float decay, restoring, dt, inv_dt;
  const float* drive;
  const float* inv_eps;
  float* pol;
  float* cur;
};
struct AdeParams {
  const float* Ein[3];
  float* Eout[3];
  int NY, P;
  // PEC faces (bit f for face f) whose tangential E stays zero after the pass
  // (StepParams::pec_clamp), and the grid extents the face test needs
  int pec_faces, NX, NZ;
  // Scenes with an instantaneous nonlinearity subtract J times the E curl
  // coefficient of this step (dt 1) instead of dt J / eps
  // (witwin/maxwell/fdtd/runtime/materials.py:751-773); nullptr otherwise.
  const float* nl_curl[3];
  AdePole poles[kAdeMaxPoles];
};
// ADE pass after the step kernel: tiles are int4 {i * NY + j, k0, k1, pole
// mask}, one warp each.
int launch_ade_pass(const AdeParams& a, const int* tiles, int n_tiles, cudaStream_t stream);
// pim / fi: the imaginary channel of a Bloch pair, or nullptr (real periodic).
// storage: kStoreF32 or kStoreBF16 (the stored field type of both channels).
int launch_wrap_fixup(const StepParams& pr, const StepParams* pim, const WrapFields& fr, const WrapFields* fi,
                      const float* phase_cos, const float* phase_sin, int n, cudaStream_t stream, int storage);

constexpr int kStoreF32 = 0;
constexpr int kStoreF16 = 1;
constexpr int kStoreBF16 = 2;

constexpr unsigned kPlaneHTerms = 1u;
constexpr unsigned kPlaneETerms = 2u;
constexpr unsigned kPlaneHRegions = 4u;
constexpr unsigned kPlaneERegions = 8u;
constexpr unsigned kPlanePoles = 16u;

}  // namespace fdtdb200
