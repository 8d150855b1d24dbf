/*
 * fdtd_b200.h -- C ABI of the B200 FDTD time-stepping library (libfdtd_b200.so).
 *
 * Two groups of entry points:
 *
 *  1. The fused step engine (fdtd_engine_*): binds the compiled solver-scene
 *     tensors of one simulation, packs them into its internal padded layout and
 *     advances whole step ranges with one fused kernel per time step.  It
 *     replaces the per-step kernel sequence of the reference's step driver,
 *     witwin/maxwell/fdtd/runtime/stepping.py:1740-1815 (_field_update_block)
 *     and :2289-2345 (the solve loop), and the host-side running-DFT loop of
 *     witwin/maxwell/fdtd/observers.py:577-659.
 *
 *  2. Per-op entry points (fdtd_op_*) with the semantics of the reference's
 *     torch ops witwin_maxwell_fdtd_cuda::<name>, schemas at
 *     witwin/maxwell/fdtd/cuda/extension.cpp:2059-2196, so that the reference's
 *     NativeFDTDModule (witwin/maxwell/fdtd/cuda/backend.py:89-115) can be
 *     re-pointed op by op.
 *
 * Conventions: every array argument is a device pointer to float32 data in
 * C-contiguous [X][Y][Z] order (z fastest) unless stated otherwise; shapes are
 * passed as plain ints; `stream` is a cudaStream_t (NULL = legacy default).
 * Every function returns 0 on success or a negative status:
 */
#ifndef FDTD_B200_H
#define FDTD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FDTD_OK 0
#define FDTD_ERR_INVALID_ARG (-1)
#define FDTD_ERR_CUDA (-2)
#define FDTD_ERR_UNSUPPORTED (-3)
#define FDTD_ERR_STATE (-4)
#define FDTD_ERR_TIMEOUT (-5)

/* Boundary codes, witwin/maxwell/fdtd/boundary/common.py:5-10. */
#define FDTD_BND_NONE 0
#define FDTD_BND_PML 1
#define FDTD_BND_PERIODIC 2
#define FDTD_BND_BLOCH 3
#define FDTD_BND_PEC 4
#define FDTD_BND_PMC 5

/* Last error message of the calling thread (engine-independent). */
const char* fdtd_last_error(void);
/* Library version string. */
const char* fdtd_version(void);

/* ------------------------------------------------------------------------ */
/* 1. Fused step engine                                                       */
/* ------------------------------------------------------------------------ */
typedef struct fdtd_engine fdtd_engine;

typedef struct {
  int nx, ny, nz;       /* node counts per axis, CPML cells included (scene.py:1260-1281) */
  double dt;            /* time step (fdtd/solver.py:145-159) */
  int boundary[6];      /* x_lo, x_hi, y_lo, y_hi, z_lo, z_hi boundary codes */
  int pml_lo[3];        /* CPML slab length on the low face of each axis (0 = none) */
  int pml_hi[3];        /* CPML slab length on the high face of each axis */
  int sample_block;     /* monitor samples buffered between DFT flushes (0 = 32) */
  int tile_rows;        /* y rows per CTA (0 = default) */
  int chunk_planes;     /* x planes per CTA (0 = default) */
} fdtd_grid_desc;

/* Create an engine on the current CUDA device.  Replaces FDTD.init_field,
 * witwin/maxwell/fdtd/runtime/stepping.py:1624-1654 (field allocation). */
int fdtd_engine_create(const fdtd_grid_desc* desc, void* stream, fdtd_engine** out);
int fdtd_engine_destroy(fdtd_engine* h);

/* Field storage of the engine's state: FDTD_STORE_F32 (default, exact FP32
 * path), FDTD_STORE_F16 or FDTD_STORE_BF16 (E and H stored in 16 bits, all
 * arithmetic in FP32; ADE pole state FP32 with FP16 fields, BF16 with BF16
 * fields).  A stored value x of
 * component c (0..2 Ex..Ez, 3..5 Hx..Hz) represents x * scales[c]; scales
 * must be powers of two, or NULL: FP16 then estimates them at finalize from the
 * source tables and the TFSF incident line (peak mapped to [32, 64)), BF16
 * uses 1.  No counterpart in the reference (its fields are FP32 only,
 * stepping.py:1625-1630).  Call right after fdtd_engine_create (the field
 * buffers are re-allocated and zeroed).  Reduced storage runs launch variant 2
 * only, and the adjoint needs FP32.  Engines with periodic or Bloch faces take
 * FP32 or BF16 (FDTD_ERR_UNSUPPORTED for FP16); both engines of a Bloch pair
 * need the same kind.  FP16 values above 65504 * scale overflow
 * to infinity: give explicit scales when the sources do not bound the field. */
#define FDTD_STORE_F32 0
#define FDTD_STORE_F16 1
#define FDTD_STORE_BF16 2
int fdtd_engine_set_storage(fdtd_engine* h, int kind, const float* scales);
int fdtd_engine_get_storage(fdtd_engine* h, int* kind, float* scales);

/* Per-axis inverse spacings: inv_e has N entries (dual), inv_h N-1 (primal),
 * witwin/maxwell/fdtd/runtime/initialization.py:131-139. */
int fdtd_engine_set_spacing(fdtd_engine* h, int axis, const float* inv_e, const float* inv_h);

/* CPML (b, c, 1/kappa) profiles of one axis, witwin/maxwell/fdtd/boundary/cpml.py:114-210
 * and :398-402: *_e have N entries, *_h have N-1. */
int fdtd_engine_set_cpml(fdtd_engine* h, int axis, const float* b_e, const float* c_e, const float* ik_e,
                         const float* b_h, const float* c_h, const float* ik_h);

/* Update coefficients of component comp (0..2 = Ex..Ez, 3..5 = Hx..Hz) in the
 * reference's Yee shape, or NULL with the uniform scalar value
 * (witwin/maxwell/fdtd/runtime/materials.py:942-1008, :1550-1574). */
int fdtd_engine_set_coefficients(fdtd_engine* h, int comp, const float* decay, float decay_uniform,
                                 const float* curl, float curl_uniform);

/* Copy a field component between the reference Yee-shaped tensor and the
 * engine's current state (witwin/maxwell/fdtd/runtime/stepping.py:1625-1630). */
int fdtd_engine_pack_field(fdtd_engine* h, int comp, const float* src);
int fdtd_engine_unpack_field(fdtd_engine* h, int comp, float* dst);

/* Copy a CPML psi array in the reference's slab-compressed layout
 * (witwin/maxwell/fdtd/boundary/cpml.py:218-333); which = 0 for the a-axis
 * array, 1 for the b-axis array of component comp (e.g. Hx: psi_hx_y, psi_hx_z). */
int fdtd_engine_pack_psi(fdtd_engine* h, int comp, int which, const float* src);
int fdtd_engine_unpack_psi(fdtd_engine* h, int comp, int which, float* dst);

/* One Debye (kind 0), Drude (1) or Lorentz (2) pole on E component comp over
 * the box [i0,i1)x[j0,j1)x[k0,k1); drive and inv_eps are box-dense
 * (witwin/maxwell/fdtd/runtime/materials.py:530-589, dispersive.cu:18-83).
 * Returns the pole id in *pole_id. */
int fdtd_engine_add_pole(fdtd_engine* h, int comp, int kind, const int* box, const float* drive,
                         const float* inv_eps, float decay, float restoring, int* pole_id);
int fdtd_engine_pole_state(fdtd_engine* h, int pole_id, float* pol_out, float* cur_out);
/* Overwrite a pole's state (box-dense, either pointer may be NULL); FP32 or FP16 field storage. */
int fdtd_engine_set_pole_state(fdtd_engine* h, int pole_id, const float* pol, const float* cur);

/* Instantaneous nonlinear cells of E component comp (0..2): before every step
 * the engine recomposes their E coefficients from E^n
 * (witwin/maxwell/fdtd/runtime/materials.py:1664-1770; kernels
 * dispersive.cu:267-400; replaces updateKerrElectricField{Ex,Ey,Ez}Curl3D and
 * updateNonlinearElectricCoefficients3D before update_electric_fields,
 * stepping.py:1794-1796).  cells: n_cells x (i, j, k) Yee indices of comp;
 * params: n_cells x 6 floats (eps_lin, decay, sigma_static, chi2, chi3,
 * tpa_sigma), with decay the static decay in the Kerr form (general = 0:
 * curl = dt / eps_eff * decay) and the external decay in the general form
 * (general = 1: decay and curl rewritten).  Host or device pointers.  Pass only
 * cells with a nonzero chi2, chi3 or tpa channel, and set the component's
 * coefficient arrays (curl; curl and decay in the general form) to the
 * formula's values with those channels zero.  Poles in such a scene subtract
 * J times this step's curl coefficient (materials.py:751-773).  Not with
 * reduced storage, Bloch fields or the adjoint. */
int fdtd_engine_set_nonlinear(fdtd_engine* h, int comp, int n_cells, const int* cells, const float* params,
                              int general, float eps0);

/* Full (off-diagonal) anisotropy of E component comp (0..2) over box (Yee
 * indices): after the step kernel the engine adds
 *   E_c += (coeff_a <curlH_a> + coeff_b <curlH_b>) / 4
 * (witwin/maxwell/fdtd/cuda/kernels/aniso.cu:26-580, applied right after the
 * E update, runtime/stepping.py:1808-1811), a < b the two other axes,
 * <curlH_d> the sum of curl(H)_d over the four d-edges around the cell and
 * coeff = dt inv_cd / eps0 from the per-edge inverse permittivity tensor
 * (runtime/materials.py:1421-1440); coeff_a / coeff_b are box-dense (host or
 * device).  The base curl coefficient of the component carries the inverse
 * tensor's diagonal.  One box per component; the box stays a cell clear of the
 * CPML slabs; not with periodic / Bloch faces, poles, nonlinear media,
 * reduced storage or the adjoint. */
int fdtd_engine_set_full_aniso(fdtd_engine* h, int comp, const int* box, const float* coeff_a, const float* coeff_b);

/* Soft source patch: comp gets coeff[cell] * signal[n] added at step n
 * (witwin/maxwell/fdtd/cuda/kernels/sources.cu:135-154; the signal table
 * holds the host-evaluated waveform, excitation/temporal.py:408-491). */
int fdtd_engine_add_patch(fdtd_engine* h, int comp, const int* box, const float* coeff, const float* signal,
                          int n_signal, float scale);
/* Time-shifted patch (sources.cu:173-221, excitation/temporal.py:232-251; the
 * pulsed soft GaussianBeam of injection.py:920-949): comp gets
 * scale[cell] * w(n * dt + t_offset - delay[cell]) at step n, w of kind 0 (CW,
 * amplitude cos(2 pi frequency t + phase)) or 1 (Gaussian pulse,
 * amplitude exp(-(tau 2 pi fwidth)^2 / 2) cos(2 pi frequency tau + phase),
 * tau = t - wdelay).  scale and delay (seconds) are box-dense; the engine
 * evaluates the waveform per cell on the GPU before every step; n_steps bounds
 * the steps it may run.  At most 8 per engine. */
int fdtd_engine_add_shifted_patch(fdtd_engine* h, int comp, const int* box, const float* scale, const float* delay,
                                  double t_offset, int kind, double frequency, double fwidth, double amplitude,
                                  double phase, double wdelay, int n_steps);

/* 1-D incident line for TFSF (witwin/maxwell/fdtd/excitation/spatial.py:311-469):
 * the engine precomputes its whole history for n_steps steps.  Coefficient
 * vectors: e_decay/e_curl have n_e entries, h_decay/h_curl n_e-1; source
 * holds the FP32 source value for each step.  Returns the line id. */
int fdtd_engine_add_aux_line(fdtd_engine* h, int n_e, const float* e_decay, const float* e_curl,
                             const float* h_decay, const float* h_curl, int source_index,
                             const float* source, int n_steps, int* line_id);
/* TFSF face correction: comp gets coeff[cell] * line[sample_index[coord]] * scale,
 * sampling the line's E history (sample_kind 0) or H history (1)
 * (witwin/maxwell/fdtd/cuda/kernels/sources.cu:485-545, excitation/tfsf_apply.py:136-264). */
int fdtd_engine_add_line_patch(fdtd_engine* h, int comp, const int* box, const float* coeff, int line_id,
                               int sample_kind, const int* sample_index, int sample_axis, float scale);

/* Monitor sample region of component comp over box; *base receives the first
 * slot of the region in the DFT accumulator vector. */
int fdtd_engine_add_sample_region(fdtd_engine* h, int comp, const int* box, int64_t* base);

/* Running DFT of all sample regions (witwin/maxwell/fdtd/observers.py:577-659,
 * spectral.py:165-232): omega (host, rad/s, n_freq entries) and the host
 * window weight per step (n_steps entries, FP64).  Phases are reduced in FP64
 * on the GPU; H regions carry the -omega*dt/2 retard (spectral.py:197-220). */
int fdtd_engine_set_dft(fdtd_engine* h, int n_freq, const double* omega, int n_steps, const double* window);
/* The same with one window per frequency: window holds n_steps x n_freq FP64
 * weights, [step][frequency] (the per-frequency spectral start steps of
 * witwin/maxwell/fdtd/runtime/spectral.py:250-298: CW runs start each
 * frequency's Hanning / ramp window after its own transient). */
int fdtd_engine_set_dft_windows(fdtd_engine* h, int n_freq, const double* omega, int n_steps, const double* window);
/* Read the accumulated DFT: re/im device arrays of n_freq * n_samples floats,
 * [freq][slot] order, unscaled (scale 2/sum(window) is applied by the caller). */
int fdtd_engine_read_dft(fdtd_engine* h, float* re, float* im);

/* Freeze the scene description and build device tables.  Must precede stepping. */
int fdtd_engine_finalize(fdtd_engine* h);
/* Advance steps [n0, n1).  One fused kernel per step, a DFT flush every
 * sample_block steps and at the end of the range. */
int fdtd_engine_step_range(fdtd_engine* h, int n0, int n1);
/* Flush buffered monitor samples into the DFT accumulators now. */
int fdtd_engine_flush(fdtd_engine* h);
/* on = 0: fdtd_engine_step_range no longer flushes at the end of every range
 * (only every sample_block steps); call fdtd_engine_flush before reading the
 * spectra.  For callers that advance one step per call (the x-slab halo
 * exchange). */
int fdtd_engine_set_range_flush(fdtd_engine* h, int on);
/* One x plane i of component comp's current state in the component's Yee
 * shape [ny_c][nz_c], to (get) or from (set) a device or host buffer, on the
 * engine's stream; FP32 storage.  The x-slab decomposition moves its halo
 * planes with them (witwin/maxwell/fdtd/distributed/nccl_transport.py:14-24,
 * one plane per face per step). */
int fdtd_engine_get_plane(fdtd_engine* h, int comp, int i, float* dst);
int fdtd_engine_set_plane(fdtd_engine* h, int comp, int i, const float* src);

/* Checkpoints of the full time-stepping state (fields, psi, ADE state),
 * witwin/maxwell/fdtd/checkpoint.py:365-568. */
int fdtd_engine_checkpoint_save(fdtd_engine* h, int slot);
/* Allocate checkpoint slots [0, n_slots) now (one allocation per slot), so
 * that later saves allocate nothing. */
int fdtd_engine_checkpoint_reserve(fdtd_engine* h, int n_slots);
int fdtd_engine_checkpoint_load(fdtd_engine* h, int slot);

/* Tile shape selection: time the candidate (tile_rows, chunk_planes) pairs on
 * the bound scene (state is saved and restored) and keep the fastest. */
int fdtd_engine_autotune(fdtd_engine* h, int* tile_rows, int* chunk_planes);
/* Launch configuration of the fused step kernel.  Variants 1-3: the scalar
 * warp kernel (one z cell per lane) with a register budget of about 100 (1),
 * 64 (2: four 256-thread CTAs per SM) or 85 (3) per thread; 4: the same warp
 * decomposition fed by TMA plane tiles; 5-9: the z-vectorised warp kernel (5:
 * four cells per lane, 6: two cells per lane, direct loads; 7 / 8: two cells
 * per lane fed by a 4- / 3-plane cp.async ring; 9: four cells per lane, 3-plane
 * ring); 10: the row-tile kernel (a TMA-fed ring of plane tiles, eight row
 * warps and a halo warp per CTA sharing y-neighbour rows through shared
 * memory; with CPML in the scene the CTAs that meet a slab run in the warp
 * kernel of variant 2 after it; poles run in the ADE pass, and variant 2 runs
 * in its place where that pass cannot take them).  Default: 10 for FP32
 * engines without CPML, periodic or Bloch faces, 2 otherwise; reduced storage
 * runs 2 only.
 * chunk_planes is the number of x planes each warp marches through (0 picks
 * the variant's default).  tile_rows is accepted for compatibility and
 * ignored. */
int fdtd_engine_set_launch(fdtd_engine* h, int variant, int tile_rows, int chunk_planes);
int fdtd_engine_get_launch(fdtd_engine* h, int* variant, int* tile_rows, int* chunk_planes);
/* Where the Debye / Drude / Lorentz poles advance: on (1, the default) in a
 * separate streaming pass after the step kernel, over the cells the pole boxes
 * cover, in the reference's order (E update, TFSF and source terms, then the
 * dispersive correction: witwin/maxwell/fdtd/runtime/stepping.py:2290-2316);
 * off (0) inside the fused step kernel.  The pass is used with FP32 storage,
 * launch variants 1-3 and no periodic / Bloch face; elsewhere the poles stay
 * in the step kernel.  The two orders agree to FP32 rounding. */
int fdtd_engine_set_ade_pass(fdtd_engine* h, int on);
/* L2 prefetch distance of the scalar step kernels (variants 1-3; default 2):
 * warps whose footprint has no CPML and no coefficient-array cell prefetch
 * their row of the E/H fields `planes` x planes (0..16; 0 disables) ahead of
 * their march.  Results do not depend on it. */
int fdtd_engine_set_prefetch(fdtd_engine* h, int planes);
/* Failure detection: polling rounds (default 1 << 20) a bounded pipeline wait
 * inside a step kernel makes before it gives up, records FDTD_ERR_TIMEOUT in
 * the device status word and returns; the next step_range then returns
 * FDTD_ERR_TIMEOUT.  The TMA variant (4) waits on its mbarrier ring this way;
 * its producer still waits for every copy it issued before the block exits
 * (that drain has its own fixed bound).  0 makes every pipeline wait run out
 * at once, which is how the timeout path is tested.  No counterpart in the
 * reference (its kernels have no device-side waits). */
int fdtd_engine_set_wait_limit(fdtd_engine* h, int rounds);
/* Launch configuration and launch count bookkeeping. */
int fdtd_engine_info(fdtd_engine* h, int* tile_rows, int* chunk_planes, int* grid_x, int* grid_y,
                     int* block, int64_t* launches);
/* Average device time of one fused step kernel over `reps` back-to-back
 * launches at step index n (CUDA events on the engine stream).  The launches
 * advance the field state like steps do but record no monitor samples. */
int fdtd_engine_time_kernel(fdtd_engine* h, int n, int reps, float* ms);
/* Device time of the last step_range in milliseconds (CUDA events). */
int fdtd_engine_last_ms(fdtd_engine* h, float* ms);

/* Batched scenes: independent engines (finalized, created on `stream`, with
 * one common even sample block M) stepped together.  Each block of M steps of
 * every engine is captured once into a CUDA graph in which every engine runs
 * on its own stream forked from `stream`, so the small scenes of a design
 * batch fill the GPU together; the graph is replayed for every block (the
 * block's base step is written to each engine's device-side base before the
 * replay) and the remaining steps run as direct launches.  Results equal the
 * engines stepped one by one.  No counterpart in the reference, which steps
 * one scene per Simulation (witwin/maxwell/fdtd/runtime/stepping.py:2289-2345).
 * While a batch exists its engines are stepped only through it. */
typedef struct fdtd_batch fdtd_batch;
int fdtd_batch_create(fdtd_engine* const* engines, int n, void* stream, fdtd_batch** out);
int fdtd_batch_destroy(fdtd_batch* b);
/* Launch-shape autotune per size class (node counts rounded to 32): the first
 * engine of each class runs fdtd_engine_autotune, the others take its pick. */
int fdtd_batch_autotune(fdtd_batch* b);
int fdtd_batch_step_range(fdtd_batch* b, int n0, int n1);
int fdtd_batch_last_ms(fdtd_batch* b, float* ms);
int fdtd_batch_info(fdtd_batch* b, int* n_engines, int* block_steps, int64_t* graph_launches);

/* Periodic and Bloch-periodic faces (x and y axes, both faces of an axis
 * alike, no CPML on that axis).  The step kernel defers the E cells whose
 * backward difference wraps around the grid; a wrap kernel updates them once
 * the whole new H is in memory, reading the far face with the phase e^{-ikL} /
 * e^{+ikL} (witwin/maxwell/fdtd/cuda/kernels/electric.cu:124-168, 356-453,
 * 1164-1229).  A periodic engine steps with fdtd_engine_step_range.  A Bloch
 * field is complex: create two engines on the same scene (the real and the
 * imaginary part, each with the sources of its part) and step them as one pair;
 * phase_cos / phase_sin hold cos(k L) and sin(k L) per axis (x, y, z; entries of
 * axes without Bloch faces are ignored).  Periodic and Bloch engines run launch
 * variants 1-3 with FP32 storage, and have no adjoint. */
typedef struct fdtd_bloch fdtd_bloch;
int fdtd_bloch_create(fdtd_engine* re, fdtd_engine* im, const float* phase_cos, const float* phase_sin,
                      fdtd_bloch** out);
int fdtd_bloch_destroy(fdtd_bloch* p);
int fdtd_bloch_step_range(fdtd_bloch* p, int n0, int n1);
int fdtd_bloch_last_ms(fdtd_bloch* p, float* ms);

/* Reverse-time adjoint: the exact discrete transpose of the fused step (H and
 * E updates, CPML psi, E edge modes), monitor seeds and dL/deps of design
 * boxes.  Replaces the reference's native reverse runners
 * (witwin/maxwell/fdtd/adjoint/native.py:48-725, kernels/adjoint.cu:295-411 and
 * 1224-1690) and its segment replay (adjoint/core.py:3527-3565).
 *
 * fdtd_engine_adjoint_init: allocate and zero the adjoint state.
 * design_boxes holds 6 ints per E component ([i0,i1,j0,j1,k0,k1] in that
 * component's Yee index space; an empty box means none) or is NULL.  Boxes
 * must stay clear of CPML slabs and domain edges; they may cover ADE cells
 * (the design variable is then eps_inf).  max_segment is the longest replay
 * (steps).
 * Dispersive (ADE) media carry adjoint pole state through the exact transpose
 * of the Debye / Drude / Lorentz recursions (the reference's dispersive reverse
 * runner, witwin/maxwell/fdtd/adjoint/native.py:2104). */
int fdtd_engine_adjoint_init(fdtd_engine* h, const int* design_boxes, int max_segment);
/* Monitor gradients dL/d(unscaled DFT accumulator), [n_freq][n_samples]
 * (host or device pointers); NULL clears the seeds. */
int fdtd_engine_adjoint_set_seed(fdtd_engine* h, const float* g_re, const float* g_im);
/* Forward replay of steps [n0, n1) from the current state (restore a
 * checkpoint first) without monitor sampling, recording the design-box E
 * history E^{n0} .. E^{n1}. */
int fdtd_engine_replay_range(fdtd_engine* h, int n0, int n1);
/* fdtd_engine_step_range with monitor sampling that also records the
 * design-box E history E^{n0} .. E^{n1} (n1 - n0 <= max_segment), so that the
 * reverse pass over [n0, n1) needs no replay: the whole history stays in HBM. */
int fdtd_engine_step_range_recorded(fdtd_engine* h, int n0, int n1);
/* Reverse steps n1-1 down to n0; with design boxes the last replay must cover
 * [n0, n1). */
int fdtd_engine_adjoint_range(fdtd_engine* h, int n1, int n0);
/* The whole reverse pass of an n_steps forward run that saved checkpoint slot s
 * at step s * stride (fdtd_engine_checkpoint_save before stepping segment s;
 * stride <= max_segment): for each segment from the last to the first, replay
 * it from its checkpoint (recording the design-box E history) and run its
 * reverse steps.  The reverse of segment s runs on a second stream while the
 * engine stream replays segment s - 1 (double-buffered histories), so the two
 * latency-bound passes overlap; the call returns when both are done.  The
 * result equals fdtd_engine_replay_range + fdtd_engine_adjoint_range per
 * segment (the reference's segment replay, witwin/maxwell/fdtd/adjoint/
 * core.py:3527-3565, with its checkpoints, checkpoint.py:365-568). */
int fdtd_engine_backward_replay(fdtd_engine* h, int n_steps, int stride);
/* Region replay (on by default): inside fdtd_engine_backward_replay, step t
 * of a T-step segment updates only the warp tasks over the design boxes grown
 * by T - t + 2 cells (the domain of dependence of the recorded design-box E:
 * one cell per step), with the scalar warp kernels; the history, and so the
 * gradient, is the full replay's bit for bit.  Applies to FP32 engines without
 * periodic / Bloch faces on launch variants 1-3 or 10; 0 replays whole steps. */
int fdtd_engine_set_replay_region(fdtd_engine* h, int on);
/* Accumulated dL/deps (absolute permittivity) of the design box of E
 * component comp (0..2), box-dense [i][j][k]. */
int fdtd_engine_adjoint_grad(fdtd_engine* h, int comp, float* out);
/* Adjoint state in the reference's shapes: kind 0 = field component comp
 * (0..5, which ignored), kind 1 = CPML psi (comp 0..5, which 0/1 as
 * fdtd_engine_pack_psi), kind 2 = ADE pole state (comp = pole id, which 0 = the
 * adjoint of P, 1 = the adjoint of J; box-dense). */
int fdtd_engine_adjoint_pack(fdtd_engine* h, int kind, int comp, int which, const float* src);
int fdtd_engine_adjoint_unpack(fdtd_engine* h, int kind, int comp, int which, float* dst);

/* ------------------------------------------------------------------------ */
/* 2. Per-op entry points (reference op semantics)                           */
/* ------------------------------------------------------------------------ */

/* Magnetic update of component comp (0 Hx, 1 Hy, 2 Hz) over an (nx, ny, nz)
 * H array; mode 0 = standard (update_magnetic_h*_standard), 1 = dense CPML
 * (update_magnetic_h*_cpml), 2 = slab-compressed CPML
 * (update_magnetic_h*_cpml_compressed); witwin/maxwell/fdtd/cuda/kernels/magnetic.cu:20-212.
 * first/second are the b-axis / a-axis E sources (Hx: Ey, Ez; Hy: Ex, Ez; Hz: Ex, Ey).
 * decay/curl may be NULL to use the uniform scalars. slab = {a_low, a_high_start,
 * a_high_len, b_low, b_high_start, b_high_len}. */
int fdtd_op_update_magnetic(int comp, int mode, int nx, int ny, int nz, float* field, const float* first,
                            const float* second, const float* decay, const float* curl, float decay_u,
                            float curl_u, const float* inv_a, const float* inv_b, float* psi_a, float* psi_b,
                            const float* ika, const float* ba, const float* ca, const float* ikb,
                            const float* bb, const float* cb, const int* slab, void* stream);

/* Complex E update on Bloch faces (electric.cu:356-453, update_electric_e*_bloch;
 * z_standard = 1: Ex / Ey with Bloch y / x and a standard z difference with
 * boundary modes z_low_mode / z_high_mode, electric.cu:1164-1528,
 * update_electric_e{x,y}_bloch_{y,x}_standard_z).  (nx, ny, nz) is the E
 * component's shape; first/second as in fdtd_op_update_electric (Ex: Hy, Hz;
 * Ey: Hx, Hz; Ez: Hx, Hy), each as real and imaginary arrays; phases a / b and
 * inv_a / inv_b in the reference's order (Ex: y, z; Ey: x, z; Ez: x, y); decay
 * and curl are E-shaped arrays. */
int fdtd_op_update_electric_bloch(int comp, int z_standard, int nx, int ny, int nz, float* e_re, float* e_im,
                                  const float* first_re, const float* first_im, const float* second_re,
                                  const float* second_im, const float* decay, const float* curl, float phase_cos_a,
                                  float phase_sin_a, float phase_cos_b, float phase_sin_b, const float* inv_a,
                                  const float* inv_b, int z_low_mode, int z_high_mode, void* stream);
/* z-CPML correction of Ex (comp 0, its H is Hy, t axis y) or Ey (comp 1, Hx,
 * t axis x) over a region of fshape at offset in the full grid (the per-axis
 * CPML corrections of the Bloch-x/y + CPML-z scenes, electric.cu:1164-1528,
 * apply_electric_e{x,y}_cpml_z_correction): field, curl and psi are
 * region-shaped, h has the full shape hshape, inv_kappa / b / c / inv_dz are
 * full-length z profiles; full_size_t / full_size_z are the full E extents
 * along t and z. */
int fdtd_op_apply_cpml_z_correction(int comp, float* field, const int* fshape, const float* h, const int* hshape,
                                    const float* curl, float* psi, const float* inv_kappa, const float* b,
                                    const float* c, const float* inv_dz, const int* offset, int low_mode,
                                    int high_mode, int full_size_t, int full_size_z, void* stream);
/* Face projection of a periodic field along axis (projection.cu:43-60,
 * project_periodic_boundary) and of a Bloch field with phase e^{ikL}
 * (projection.cu:62-125, project_bloch_boundary). */
int fdtd_op_project_periodic(float* field, const int* fshape, int axis, void* stream);
int fdtd_op_project_bloch(float* field_re, float* field_im, const int* fshape, int axis, float phase_cos,
                          float phase_sin, void* stream);

/* Electric update of component comp (0 Ex, 1 Ey, 2 Ez) with boundary-mode-aware
 * backward differences; modes = {a_low, a_high, b_low, b_high} boundary codes;
 * witwin/maxwell/fdtd/cuda/kernels/electric.cu:242-941 (update_electric_e*_{standard,cpml,cpml_compressed}).
 * first/second: Ex: Hy, Hz; Ey: Hx, Hz; Ez: Hx, Hy. */
int fdtd_op_update_electric(int comp, int mode, int nx, int ny, int nz, float* field, const float* first,
                            const float* second, const float* decay, const float* curl, float decay_u,
                            float curl_u, const float* inv_a, const float* inv_b, const int* modes,
                            float* psi_a, float* psi_b, const float* ika, const float* ba, const float* ca,
                            const float* ikb, const float* bb, const float* cb, const int* slab, void* stream);

/* ADE ops, witwin/maxwell/fdtd/cuda/kernels/dispersive.cu:18-83
 * (update_debye_current, update_drude_current, update_lorentz_current, apply_polarization_current). */
int fdtd_op_update_debye(int64_t n, const float* e, const float* drive, float decay, float dt, float* pol,
                         float* cur, void* stream);
int fdtd_op_update_drude(int64_t n, const float* e, const float* drive, float decay, float* cur, void* stream);
int fdtd_op_update_lorentz(int64_t n, const float* e, const float* drive, float decay, float restoring,
                           float dt, float* pol, float* cur, void* stream);
int fdtd_op_apply_polarization(int64_t n, const float* cur, const float* inv_eps, float dt, float* e,
                               void* stream);

/* Instantaneous nonlinear E coefficients of component comp (0..2) over its
 * whole Yee array (update_kerr_e{x,y,z}_curl and update_nonlinear_coefficients,
 * extension.cpp:2109-2112; kernels dispersive.cu:165-400).  shapes: the
 * Ex, Ey, Ez array shapes (9 ints); eps, decay / external_decay, sigma, chi2,
 * chi3, tpa and the outputs have comp's shape.  E is collocated onto comp's
 * edge (4-point averages, clamped indices); eps_eff is floored at 1e-12 eps0.
 * Kerr: curl = dt / (eps + eps0 chi3 |E|^2) * decay.  General:
 * eps_eff = eps + eps0 (chi2 E_comp + chi3 |E|^2), sigma = max(sigma + tpa |E|^2, 0),
 * half = sigma dt / (2 eps_eff), decay = ext (1 - half) / (1 + half),
 * curl = ext dt / eps_eff / (1 + half). */
/* Off-diagonal anisotropic coupling of E component comp (update_electric_e{x,y,z}_full_aniso,
 * extension.cpp:2113-2115; kernels/aniso.cu:26-580): e has comp's Yee shape on a grid of nx x ny x nz nodes;
 * coeff_a / coeff_b (comp's shape) weight the two other curl(H) components, lower axis first;
 * inv_d* are the per-node inverse spacings; periodic axes wrap the stencils. */
int fdtd_op_update_electric_full_aniso(int comp, int nx, int ny, int nz, float* e, const float* hx, const float* hy,
                                       const float* hz, const float* coeff_a, const float* coeff_b,
                                       const float* inv_dx, const float* inv_dy, const float* inv_dz, int periodic_x,
                                       int periodic_y, int periodic_z, void* stream);
int fdtd_op_update_kerr_curl(int comp, const int* shapes, const float* ex, const float* ey, const float* ez,
                             const float* eps, const float* decay, const float* chi3, float dt, float eps0,
                             float* curl, void* stream);
int fdtd_op_update_nonlinear_coefficients(int comp, const int* shapes, const float* ex, const float* ey,
                                          const float* ez, const float* eps, const float* external_decay,
                                          const float* sigma, const float* chi2, const float* chi3, const float* tpa,
                                          float dt, float eps0, float* decay, float* curl, void* stream);

/* add_source_patch (sources.cu:135-154): field[off + idx] += signal * patch[idx],
 * cells outside the field are skipped.  fshape/pshape/offset are int[3]. */
int fdtd_op_add_source_patch(float* field, const int* fshape, const float* patch, const int* pshape,
                             const int* offset, float signal, void* stream);
/* addCwPhasedSourcePatch3D (sources.cu:156-171, launched by excitation/
 * temporal.py:133-144): value = signal_cos * patch_cos + signal_sin * patch_sin. */
int fdtd_op_add_cw_patch(float* field, const int* fshape, const float* patch_cos, const float* patch_sin,
                         const int* pshape, const int* offset, float signal_cos, float signal_sin, void* stream);
/* addTimeShiftedSourcePatch3D (sources.cu:173-221, excitation/temporal.py:232-251):
 * value = patch * w(time - delay[idx]), w of kind 0 (CW, amplitude
 * cos(2 pi frequency t + phase)), 1 (Gaussian pulse of width fwidth centred at
 * wdelay) or 2 (Ricker centred at wdelay), waveforms.py:83-107; with causal_gate
 * a cell adds nothing while time < activation[idx] (activation may be NULL
 * without the gate). */
int fdtd_op_add_shifted_patch(float* field, const int* fshape, const float* patch, const float* delay,
                              const float* activation, int causal_gate, const int* pshape, const int* offset, int kind,
                              float time, float frequency, float fwidth, float amplitude, float phase, float wdelay,
                              void* stream);
/* add_scaled_line_source_patch (sources.cu:485-545): value = coeff * incident[sample_idx[a]] * scale. */
int fdtd_op_add_line_patch(float* field, const int* fshape, const float* coeff, const int* pshape,
                           const int* offset, const float* incident, const int64_t* sample_idx, int axis,
                           float scale, void* stream);
/* Auxiliary 1-D grid (sources.cu:803-839). */
int fdtd_op_aux_magnetic(int n_e, float* h, const float* e, const float* h_decay, const float* h_curl,
                         void* stream);
/* The last cell (n_e - 1) is pinned to zero before the source cell is
 * considered; a negative source_index injects nothing. */
int fdtd_op_aux_electric(int n_e, float* e, const float* h, const float* e_decay, const float* e_curl,
                         int source_index, float source_value, void* stream);

/* Whole incident-line history in one call, allocating no device memory.  No
 * counterpart in the reference: it is a variant of the history kernel behind
 * fdtd_engine_add_aux_line whose running line state lives in a fixed device
 * array instead of allocated scratch.
 *
 * For callers that cannot allocate: a process whose free device memory is all
 * reserved by its own caching pool (cudaMalloc would fail or make the pool
 * release cached blocks), and a caller on a latency-critical stream, where
 * cudaFree's device-wide synchronisation would stall every other stream.
 *
 * Every pointer is device memory owned by the caller: the coefficient arrays
 * (e_decay, e_curl: n_e; h_decay, h_curl: n_e - 1), source (n_steps values for
 * the source cell), and the outputs e_hist and h_hist (n_steps x n_e, row n =
 * the line before E/after H of step n; the last entry of each H row is zero).
 * Same recurrence as fdtd_op_aux_magnetic followed by fdtd_op_aux_electric,
 * stepped n_steps times from a zero line.  A negative source_index injects
 * nothing; a source on the last cell (n_e - 1) is overridden by that cell's
 * zero, as in the reference's update_auxiliary_electric_kernel.
 *
 * Limit: n_e <= FDTD_AUX_STATIC_MAX_CELLS; larger lines return
 * FDTD_ERR_INVALID_ARG.  The line state starts at zero on every call (the
 * kernel clears it); nothing else needs clearing.  Every call looks up the
 * array's device address on the current device (no allocation); the first call
 * on a device may load the module, so make one call per device, with that
 * device current, before any stream capture.
 * The array is shared by every call on a device: calls that can overlap
 * (different streams, or unordered host threads) race on it and both results
 * are undefined, so order them on one stream. */
#define FDTD_AUX_STATIC_MAX_CELLS 16384
int fdtd_op_aux_line_history_static(int n_e, const float* e_decay, const float* e_curl, const float* h_decay,
                                    const float* h_curl, int source_index, const float* source, int n_steps,
                                    float* e_hist, float* h_hist, void* stream);
/* Observers (observers.cu:7-78) and the batched full-field DFT (spectral.cu:9-146). */
int fdtd_op_point_observers(const float* field, const int* fshape, int n_points, const int* pi, const int* pj,
                            const int* pk, float* re, float* im, float wcos, float wsin, void* stream);
int fdtd_op_plane_observer(const float* field, const int* fshape, int axis, int index, float* re, float* im,
                           float wcos, float wsin, void* stream);
int fdtd_op_dft_volume(int64_t n, int n_freq, const float* field, float* re, float* im, const float* wcos,
                       const float* wsin, void* stream);
/* PEC face clamp (boundary.cu:69-168). */
int fdtd_op_clamp_face(float* field, const int* fshape, int axis, int side, void* stream);

/* ------------------------------------------------------------------------ */
/* 3. Consumers of the DFT planes                                            */
/* ------------------------------------------------------------------------ */
/* Diffraction-order projection of one frequency's plane spectrum
 * (witwin/maxwell/postprocess/diffraction.py:84-196): field holds the
 * co-located complex components [na][nb][3] (interleaved re, im; float32) of E
 * or of H on the plane's tangential coordinates coords_a [na], coords_b [nb];
 * for the order grid kx[n_m] x ky[n_n] (FP64) it writes
 * amplitudes[m][n][3] (interleaved complex) = the mean over the plane of
 * F exp(-i (kx a + ky b)).  scratch: 2 * n_n * na * 3 doubles of device memory. */
int fdtd_pp_diffraction(int na, int nb, const float* coords_a, const float* coords_b, const float* field, int n_m,
                        const double* kx, int n_n, const double* ky, double* scratch, float* amplitudes,
                        void* stream);
/* Near-to-far-field transform (witwin/maxwell/postprocess/nfft.py:100-137):
 * points [P][3] (metres), quadrature-weighted surface currents j_weighted /
 * m_weighted [P][3] (interleaved complex), unit directions [D][3] and radii
 * [D]; lossless background wavenumber k and impedance eta.  Writes the far E
 * and H [D][3] (interleaved complex) and the radial power density [D]. */
int fdtd_pp_nfft(int n_points, const float* points, const float* j_weighted, const float* m_weighted, int n_dirs,
                 const float* directions, const float* radius, double k, double eta, float* e_out, float* h_out,
                 float* power, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FDTD_B200_H */
