/*
 * rfxb200 -- C ABI of the B200 FDTD time-stepping library.
 *
 * The reference (bk-squared/rfx 1.6.7) is pure Python/JAX and has no plugin or
 * FFI API of its own.  Its seam for this path is the pure-Python function
 *   rfx.simulation.run(grid, materials, n_steps, *, boundary, cpml_axes,
 *                      pec_axes, sources, probes, dft_planes, pec_mask,
 *                      checkpoint, checkpoint_segments, ...)   rfx/simulation.py:1686
 * and its graded-mesh twin
 *   rfx.nonuniform.run_nonuniform(...)                          rfx/nonuniform.py:1589
 * whose bodies run one jax.lax.scan over the step function built by
 *   make_core_step                                              rfx/simulation.py:1227
 *   _build_nu_scan                                              rfx/nonuniform.py:998
 * Each entry point below names the piece of that seam it replaces.
 *
 * Conventions
 *  - All functions return 0 on success or a negative RFXB_E_* code; the
 *    message of the last failure on the calling thread is rfxb_last_error().
 *    Nothing raises inside a kernel; device-side status is read back.
 *  - Array arguments named *_dev are device pointers, *_host host pointers.
 *    Field and material arrays use the reference layout: (nx, ny, nz)
 *    C-order float32, z fastest.
 *  - A plan owns its internal state (padded double-buffered fields, CPML
 *    psi, update coefficients, Kahan DFT compensation, checkpoints).  The
 *    caller owns everything it passes in: materials, source tables, probe
 *    outputs, DFT accumulators, adjoint tables, gradient buffers.
 *  - Work is stream-ordered on the cudaStream_t given (0 = legacy default).
 *    A plan must not be used from two threads at once.
 */
#ifndef RFXB200_H
#define RFXB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RFXB_OK 0
#define RFXB_E_INVALID (-1)   /* bad descriptor or argument */
#define RFXB_E_SHAPE (-2)     /* inconsistent sizes */
#define RFXB_E_NOMEM (-3)     /* device allocation failed */
#define RFXB_E_LAUNCH (-4)    /* kernel launch or CUDA runtime failure */
#define RFXB_E_STATE (-5)     /* call out of order (e.g. adjoint before forward) */
#define RFXB_E_TIMEOUT (-6)   /* a bounded wait inside a kernel ran out (device status word) */
#define RFXB_E_WORK (-7)      /* a persistent kernel met an invalid work item (device status word) */

#define RFXB_AXIS_X 1u
#define RFXB_AXIS_Y 2u
#define RFXB_AXIS_Z 4u

/* field component codes (ex ey ez hx hy hz) */
#define RFXB_EX 0
#define RFXB_EY 1
#define RFXB_EZ 2
#define RFXB_HX 3
#define RFXB_HY 4
#define RFXB_HZ 5
/* probe flag: sample before soft-source injection (lumped-port V/I,
 * rfx/simulation.py:1449-1500) */
#define RFXB_PROBE_PRESOURCE 16

typedef struct RfxbPlan RfxbPlan;
typedef struct RfxbBatch RfxbBatch;

/* One running-DFT plane (rfx/probes/probes.py:379-449). */
typedef struct {
  int axis;        /* normal axis 0/1/2 */
  int index;       /* plane index along the axis */
  int component;   /* RFXB_EX..RFXB_HZ */
  int n_freqs;
} RfxbDftDesc;

/* One Poynting-flux monitor (rfx/probes/probes.py:476-580, accumulated as in
 * rfx/simulation.py:1590-1642): the two tangential E components on plane
 * `index` of the normal axis and the two tangential H components averaged
 * over planes index-1 and index (index 0: plane 0 twice), on the region
 * [lo1, hi1) x [lo2, hi2) of the plane's tangential axes (x-normal: y, z;
 * y-normal: x, z; z-normal: x, y). */
typedef struct {
  int axis, index;
  int lo1, hi1, lo2, hi2;
  int n_freqs;
} RfxbFluxDesc;

/* The near-to-far-field Huygens box (rfx/farfield.py:32-79 NTFFBox): six
 * faces at i_lo, i_hi (x), j_lo, j_hi (y) and k_lo, k_hi (z), each covering
 * the half-open ranges [lo, hi) of its two tangential axes.  Accumulated as
 * rfx/farfield.py:208-313 accumulate_ntff does, once per step after the E
 * update and source injection. */
typedef struct {
  int i_lo, i_hi, j_lo, j_hi, k_lo, k_hi;
  int n_freqs;
} RfxbNtffDesc;

/* Static description of one simulation (grid, boundaries, monitors).
 * Replaces the trace-time setup of _build_step_setup (rfx/simulation.py:626)
 * and _build_nu_scan (rfx/nonuniform.py:998). */
typedef struct {
  int nx, ny, nz;
  double dt;
  /* inverse spacing tables, length nx / ny / nz (host).  E-update tables
   * ("inv_d_e") and H-update tables ("inv_d_h") as built by
   * rfx/nonuniform.py:187-224; for a uniform grid every entry is 1/dx. */
  const float* inv_xe_host; const float* inv_xh_host;
  const float* inv_ye_host; const float* inv_yh_host;
  const float* inv_ze_host; const float* inv_zh_host;
  /* CPML (rfx/boundaries/cpml.py:346-478): layers per face (0 = none), the
   * axes that absorb, and per face (x_lo, x_hi, y_lo, y_hi, z_lo, z_hi) the
   * float32 b, c, kappa profiles of length cpml_layers with the hi faces
   * pre-flipped, plus each face's boundary cell size. */
  int cpml_layers;
  unsigned cpml_axes;
  const float* cpml_b_host;      /* [6][cpml_layers] */
  const float* cpml_c_host;      /* [6][cpml_layers] */
  const float* cpml_kappa_host;  /* [6][cpml_layers] */
  double cpml_cell[6];
  /* PEC faces applied after every E update (rfx/boundaries/pec.py:13-47) */
  unsigned pec_axes;
  /* soft sources: n_src x (i, j, k, component) (rfx/simulation.py:44-54) */
  int n_src;
  const int32_t* src_cells_host;
  /* point probes: n_probe x (i, j, k, component | flags) (rfx/simulation.py:75-80) */
  int n_probe;
  const int32_t* probe_cells_host;
  /* running-DFT planes */
  int n_dft;
  const RfxbDftDesc* dft_host;
  /* gradient region [i0,i1) x [j0,j1) x [k0,k1) whose forward history the
   * adjoint needs; i0 >= i1 means none */
  int grad_box[6];
  /* Poynting-flux monitors */
  int n_flux;
  const RfxbFluxDesc* flux_host;
  /* NTFF Huygens box, NULL for none */
  const RfxbNtffDesc* ntff_host;
} RfxbDesc;

/* Per-call device buffers of the forward path. */
typedef struct {
  const float* src_wave_dev;   /* [n_total_steps][n_src], row = global step */
  float* probe_out_dev;        /* [n_total_steps][n_probe], may be NULL */
  void* const* dft_acc_dev;    /* n_dft complex64 arrays (n_freqs, n1, n2), accumulated */
  const void* const* dft_phase_dev; /* n_dft float2 arrays [n_total_steps][n_freqs]: (cos, sin)*dt */
  /* n_flux complex128 accumulators [4][n_freqs][n1][n2] (E1, E2, H1, H2),
   * accumulated, and n_flux complex128 kernels [n_total_steps][2][n_freqs]:
   * the E and H phase factors times dt and the window weight of each step */
  void* const* flux_acc_dev;
  const void* const* flux_kernel_dev;
  /* NTFF box: complex64 running sums and Kahan residuals, each the six faces
   * x_lo, x_hi, y_lo, y_hi, z_lo, z_hi back to back, face f an array
   * (n_freqs, n1, n2, 4) of the tangential components (x faces: ey ez hy hz;
   * y faces: ex ez hx hz; z faces: ex ey hx hy), and the complex64 phase
   * table [n_total_steps][2][n_freqs] (E factor, H factor, both times dt).
   * All three NULL: no accumulation. */
  void* ntff_acc_dev;
  void* ntff_cmp_dev;
  const void* ntff_phase_dev;
} RfxbStepIO;

/* Per-call device buffers of the adjoint path. */
typedef struct {
  const float* g_dev;          /* dJ/d(probe samples) [n_total_steps][n_probe] */
  double* grad_dev;            /* dJ/d eps_r over grad_box, accumulated (C order) */
  const float* dca_dev;        /* d ca / d eps_r over grad_box */
  const float* dcb_dev;        /* d cb / d eps_r over grad_box */
  float* src_adj_dev;          /* dJ/d(source table) [n_total_steps][n_src], may be NULL */
  /* DFT-plane objectives (the transpose of the running DFT,
   * rfx/simulation.py:1574-1588): per DFT plane of the plan a complex64
   * cotangent (n_freqs, n1, n2) = dJ/dRe(acc) + i dJ/dIm(acc), or NULL, and
   * the phase table the forward accumulated with ([n_total_steps][n_freqs]
   * (cos, sin) * dt).  Both arrays NULL: no DFT-plane cotangents. */
  const void* const* dft_cot_dev;
  const void* const* dft_phase_dev;
  /* NTFF-box objectives (the transpose of rfx/farfield.py:208-313): a
   * complex64 cotangent laid out like the running sums of RfxbStepIO
   * (faces x_lo .. z_hi, each (n_freqs, n1, n2, 4)) and the phase table the
   * forward used ([n_total_steps][2][n_freqs]).  NULL: none. */
  const void* ntff_cot_dev;
  const void* ntff_phase_dev;
  /* Flux-monitor objectives (the transpose of rfx/simulation.py:1590-1642):
   * per monitor a complex128 cotangent laid out like its accumulator
   * ([4][n_freqs][n1][n2]) or NULL, and the kernel table the forward used.
   * Both arrays NULL: none. */
  const void* const* flux_cot_dev;
  const void* const* flux_kernel_dev;
} RfxbAdjointIO;

int rfxb_version(void);
const char* rfxb_last_error(void);

/* Create / destroy a plan.  Replaces the trace-time setup named above.
 * A plan lives on the device current at its creation; destroy waits for the
 * current device before freeing, so call it with that device current. */
int rfxb_plan_create(const RfxbDesc* desc, RfxbPlan** out);
void rfxb_plan_destroy(RfxbPlan* plan);

/* Materials -> per-cell update coefficients (ca, cb of rfx/core/yee.py:387-393,
 * ce of rfx/boundaries/cpml.py:536, ch of cpml.py:818), computed on device in
 * float32.  mu_r_dev may be NULL (mu_r = 1).  edge_mask_dev (uint8, bits
 * 1/2/4 = ex/ey/ez zeroed after each E update, the output of
 * tangential_edge_masks at rfx/boundaries/pec.py:90-176) may be NULL. */
int rfxb_plan_set_materials(RfxbPlan* plan, const float* eps_r_dev, const float* sigma_dev,
                            const float* mu_r_dev, const uint8_t* edge_mask_dev, void* stream);

/* Zero fields, psi, DFT compensation and the step parity (init_state +
 * init_cpml, rfx/core/yee.py:42-58, rfx/boundaries/cpml.py:346). */
int rfxb_plan_reset(RfxbPlan* plan, void* stream);
/* Copy fields between caller arrays (reference layout) and the plan state.
 * fields_dev: 6 pointers ex ey ez hx hy hz. */
int rfxb_plan_load_fields(RfxbPlan* plan, const float* const* fields_dev, void* stream);
int rfxb_plan_store_fields(RfxbPlan* plan, float* const* fields_dev, void* stream);

/* Advance n_steps steps starting at global step step0 (the scan of
 * rfx/simulation.py:1969-1977 / rfx/nonuniform.py:1796 over the body of
 * rfx/simulation.py:1255-1685 / rfx/nonuniform.py:1256-1568).  The uniform
 * or graded lane is selected by the spacing tables; the DFT sample time is
 * encoded in the caller's phase table. */
int rfxb_plan_advance(RfxbPlan* plan, const RfxbStepIO* io, int step0, int n_steps, void* stream);

/* load_fields + advance + store_fields in one call: the shape of an XLA
 * custom call that aliases the fields in and out. */
int rfxb_forward(RfxbPlan* plan, const RfxbStepIO* io, float* const* fields_dev,
                 int step0, int n_steps, void* stream);

/* Forward history of the gradient region for steps [step0, step0+n_steps):
 * the plan keeps E^n and curl H^{n+1/2} there, for the adjoint.  Must be
 * called before the advance that produces those steps. */
int rfxb_plan_record_history(RfxbPlan* plan, int step0, int n_steps);

/* Checkpoints of the full state (fields, psi, parity) in plan-owned HBM:
 * the storage of checkpoint-every-K with segment recompute, replacing
 * jax.checkpoint segments (rfx/simulation.py:2011-2058,
 * rfx/nonuniform.py:1755-1794). */
int rfxb_plan_checkpoint_reserve(RfxbPlan* plan, int n_slots);
int rfxb_plan_checkpoint_save(RfxbPlan* plan, int slot, void* stream);
int rfxb_plan_checkpoint_load(RfxbPlan* plan, int slot, void* stream);

/* Resumable state of a plan as one byte blob (restart of long runs and
 * sweeps).  rfx's save_state (rfx/checkpoint.py:33-62) writes the six fields
 * and the step to HDF5; a resumed CPML run also needs its psi, and a resumed
 * DFT its Kahan residuals, so the blob holds a header (magic "RFXBST01",
 * shape, CPML layers and axes, section sizes) followed by the current
 * fields, psi and DFT residuals in the plan's own layout.  dst / src may be
 * device or host memory; save_state is asynchronous on `stream`,
 * restore_state reads the header synchronously and rejects a blob of another
 * shape or CPML set-up with RFXB_E_SHAPE. */
long long rfxb_plan_state_bytes(const RfxbPlan* plan);
int rfxb_plan_save_state(RfxbPlan* plan, void* dst, void* stream);
int rfxb_plan_restore_state(RfxbPlan* plan, const void* src, void* stream);

/* Reverse-time adjoint: the transpose of the forward step, replacing
 * jax.grad through the scan.  adjoint_begin zeroes the adjoint state and
 * injects the probe cotangent of the last step n_total-1; adjoint_advance
 * runs the reverse steps step_hi-1 down to step_hi-n_steps, whose history
 * must have been recorded. */
int rfxb_plan_adjoint_begin(RfxbPlan* plan, const RfxbAdjointIO* aio, int n_total, void* stream);
int rfxb_plan_adjoint_advance(RfxbPlan* plan, const RfxbAdjointIO* aio, int step_hi, int n_steps,
                              void* stream);

/* Batched sweep: many plans (uneven grid sizes) advanced together, one
 * launch per step for all of them, the step loop captured in a CUDA graph.
 * Replaces a Python loop of independent run()/forward() calls, the only
 * batching the reference offers for uneven grids (rfx/vmap_sweep.py:871
 * batches equal grids only). */
int rfxb_batch_create(RfxbPlan* const* plans, int n_plans, RfxbBatch** out);
/* Like rfxb_plan_destroy: call with the plans' device current. */
void rfxb_batch_destroy(RfxbBatch* batch);
int rfxb_batch_advance(RfxbBatch* batch, const RfxbStepIO* ios, int step0, int n_steps, void* stream);
int rfxb_batch_record_history(RfxbBatch* batch, int step0, int n_steps);
int rfxb_batch_adjoint_begin(RfxbBatch* batch, const RfxbAdjointIO* aios, int n_total, void* stream);
int rfxb_batch_adjoint_advance(RfxbBatch* batch, const RfxbAdjointIO* aios, int step_hi, int n_steps,
                               void* stream);

/* Synchronise the stream and read the device status word of the plan's (or
 * batch's) launches: RFXB_E_TIMEOUT if a bounded pipeline wait inside a step
 * kernel ran out (the kernel then left without hanging the GPU). */
int rfxb_plan_device_status(RfxbPlan* plan, void* stream);
int rfxb_batch_device_status(RfxbBatch* batch, void* stream);

/* Forward steps without any device allocation.  No counterpart in the
 * reference: rfx leaves memory to JAX, so it never needs this.  It is for
 * callers that cannot call cudaMalloc -- a host program whose own allocator
 * owns all device memory, or one that cannot afford the device-wide
 * synchronisation an allocation may bring mid-loop -- and therefore cannot
 * create a plan.  One call loads the caller's fields (reference layout),
 * computes the coefficients from eps_r_dev / sigma_dev (mu_r = 1, no edge
 * mask), starts from zero CPML psi, runs n_steps steps of the fused step
 * kernel with sources and probes from io, and writes the fields back.  All
 * internal state lives in one fixed 64 MiB device array inside the library:
 * grids whose state does not fit (about 0.8 M cells) get RFXB_E_NOMEM, and DFT
 * planes or gradient regions get RFXB_E_INVALID (use a plan for those).  The
 * first call on a device sets it up (the array's address, the kernel's
 * shared-memory limit); make that first call before any stream capture.  Each
 * call uploads small host tables from memory that lives only during the call,
 * so a call on a capturing stream is refused with RFXB_E_INVALID; no call may
 * follow a cudaDeviceReset of the device.  Calls share the array: each clears
 * what must start at zero, and two calls whose GPU work overlaps race on it.
 * Negative counts and null source / probe tables with a positive count are
 * refused with RFXB_E_INVALID. */
int rfxb_forward_noalloc(const RfxbDesc* desc, const float* eps_r_dev, const float* sigma_dev,
                         float* const* fields_dev, const RfxbStepIO* io, int step0, int n_steps, void* stream);

/* Sum of E^2 + H^2 over the cells box[0] <= i < box[1], box[2] <= j < box[3],
 * box[4] <= k < box[5] of the plan's current state, written (float64,
 * overwritten) to *energy_dev in stream order: the interior-energy check of
 * run_until_decay (rfx/simulation.py:2493-2505). */
int rfxb_plan_box_energy(RfxbPlan* plan, const int* box, double* energy_dev, void* stream);
/* The same sum with every cell weighted by wx[i] * wy[j] * wz[k] (device
 * float64 tables of length nx, ny, nz): the graded lane's interior-energy
 * check, weighted by the primal cell volume dx[i] dy[j] dz[k]
 * (rfx/nonuniform.py:2143-2156). */
int rfxb_plan_box_energy_weighted(RfxbPlan* plan, const int* box, const double* wx_dev, const double* wy_dev,
                                  const double* wz_dev, double* energy_dev, void* stream);

/* Net outgoing co-located Poynting flux through the faces of the box
 * (faces at i = box[0] and i = box[1], j = box[2] and box[3], k = box[4] and
 * box[5], each over the half-open ranges of its tangential axes): on an x
 * face Ey Hz - Ez Hy, on a y face Ez Hx - Ex Hz, on a z face Ex Hy - Ey Hx,
 * with sign + on the high face and - on the low one, summed in float64 and
 * written (overwritten) to *flux_dev in stream order: the radiated-flux stop
 * of run_until_decay (rfx/simulation.py:2513-2540). */
int rfxb_plan_box_flux(RfxbPlan* plan, const int* box, double* flux_dev, void* stream);

/* Bytes of device memory a plan holds (state, coefficients, psi, history,
 * checkpoints, and the intermediate state of two-step passes once used). */
int64_t rfxb_plan_device_bytes(const RfxbPlan* plan);

/* Which forward step kernel the launches of a plan (or batch) use: 0 the
 * generic one (cp.async staging, CPML psi read from global memory), 1 TMA
 * staging without CPML, 2 TMA staging with the CPML psi staged by TMA one
 * plane ahead; -1 for a null handle.  A diagnostic of this implementation,
 * no counterpart in the reference. */
int rfxb_plan_forward_variant(const RfxbPlan* plan);
int rfxb_batch_forward_variant(const RfxbBatch* batch);

/* Which reverse step kernel the adjoint launches of a plan (or batch) use:
 * 0 cp.async staging, 1 TMA staging with CPML psi read from global memory,
 * 2 TMA staging with the adjoint psi and ce staged by TMA one plane ahead,
 * 3 TMA staging without any CPML (groups without CPML); with 1 or 2, tiles
 * whose reverse step touches no slab run on 3 beside it, and with 2 the
 * CPML work of tiles that reach no y slab runs on variant 4 (variant 2
 * without the y-slab terms, four CTAs per SM) on a third stream.  -1 before
 * the first adjoint advance or for a null handle.  A diagnostic of this
 * implementation, no counterpart in the reference. */
int rfxb_plan_adjoint_variant(const RfxbPlan* plan);
int rfxb_batch_adjoint_variant(const RfxbBatch* batch);

/* Step-kernel launches per forward time step (*fwd: 1, or 2 with the split
 * into CPML and plain tiles; with two-step passes, fwd_depth 2, the launches
 * of one pass of two steps: the two-step tiles plus two launches of each
 * one-step list) and per reverse time step (*rev: 1, 2 with the
 * split, 3 when variant 4 takes the CPML work without a y slab; -1 before
 * the first adjoint advance), not counting DFT / flux / NTFF epilogue
 * kernels.  A diagnostic of this implementation. */
int rfxb_plan_step_launches(const RfxbPlan* plan, int* fwd, int* rev);
int rfxb_batch_step_launches(const RfxbBatch* batch, int* fwd, int* rev);

/* Launch configuration of a plan's (or batch's) step launches: the choices
 * the autotuner (rfx_b200/autotune.py) searches.  Every setting computes the
 * same steps; they differ in how the tiles are split among kernel variants
 * and streams and in which launch a captured graph hands to the SMs first.
 *   fwd_split  1: forward tiles split, the CPML-free variant 1 beside the
 *                 staged-psi variant 2 on two streams; 0: one launch
 *   fwd_order  with the split, 0: plain-tile launch first, 1: CPML-tile
 *                 launch first
 *   adj_lite   1: reverse CPML work of tiles that reach no y slab on
 *                 variant 4 (third stream); 0: on variant 2
 *   adj_order  order of the reverse launches, a permutation of (variant 4,
 *                 variant 2, variant 3) by index: 0 (4,2,3), 1 (4,3,2),
 *                 2 (2,4,3), 3 (2,3,4), 4 (3,4,2), 5 (3,2,4); without
 *                 variant 4 only the relative order of 2 and 3 counts
 *   fwd_persist  0: the launches above; k >= 1: one persistent launch per
 *                 step over both forward lists (as many CTAs as are resident,
 *                 each pulling items from device queues), k-1 CTAs per SM
 *                 taking CPML-free items first, the others CPML items first
 *   adj_persist  0: the launches above; 1: one persistent launch per reverse
 *                 step over the three reverse lists, one CTA per SM taking
 *                 each list first
 *   l2_promo   L2 promotion of the plans' TMA boxes: 0 none, 1 64 B,
 *                 2 128 B, 3 256 B (how much of a partly covered line a halo
 *                 miss fetches; the plans' maps are re-encoded)
 *   fwd_depth  time steps per forward pass over HBM: 1 (0 means 1), or 2
 *                 where the group has tiles for it: temporal blocking, the
 *                 CPML-free interior tiles away from sources, probes and the
 *                 gradient region advance two steps per pass on the two-step
 *                 kernel while the rest runs one launch per step through an
 *                 intermediate field buffer (allocated on first use, 24 bytes
 *                 per cell); an odd remaining step runs alone, and every
 *                 step does while a plan has per-cell mu_r.  Excludes
 *                 fwd_persist > 0.  Results equal depth 1
 *                 bit for bit (rfxb_*_step_launches then counts the
 *                 launches of one pass of two steps).
 * rfxb_*_launch_config writes the current setting to *current and the
 * largest value each field accepts on this plan/batch to *limits (0 where a
 * choice does not exist, e.g. fwd_split on a group without staged-psi CPML).
 * rfxb_*_set_launch_config checks each field against those limits
 * (RFXB_E_INVALID otherwise), synchronises the device and drops the cached
 * step graphs.  A tuning interface of this implementation; the reference
 * has no counterpart (XLA schedules its scan body itself). */
typedef struct RfxbLaunchConfig {
  int32_t fwd_split;
  int32_t fwd_order;
  int32_t adj_lite;
  int32_t adj_order;
  int32_t fwd_persist;
  int32_t adj_persist;
  int32_t l2_promo;
  int32_t fwd_depth;
} RfxbLaunchConfig;

int rfxb_plan_launch_config(const RfxbPlan* plan, RfxbLaunchConfig* current, RfxbLaunchConfig* limits);
int rfxb_plan_set_launch_config(RfxbPlan* plan, const RfxbLaunchConfig* config);
int rfxb_batch_launch_config(const RfxbBatch* batch, RfxbLaunchConfig* current, RfxbLaunchConfig* limits);
int rfxb_batch_set_launch_config(RfxbBatch* batch, const RfxbLaunchConfig* config);

/* Test hooks of the persistent step kernels (no counterpart in the
 * reference).  debug_fault: from the next launch on, the CTA with block
 * index `cta` (-1: none) does not load plane xa of its first work item, and
 * every pipeline wait gives up after `wait_limit` polls, so that CTA's wait
 * runs out and rfxb_*_device_status reports RFXB_E_TIMEOUT (no box is left
 * in flight: the CTA drains the others before leaving).  debug_poison
 * replaces entry `index` of a work list (0/1 forward CPML/CPML-free, 2/3/4
 * reverse y-slab/other CPML/CPML-free) with an empty x range, which the
 * persistent kernels skip and report as RFXB_E_WORK.  Both leave the batch's
 * state invalid: only the status check is meaningful afterwards. */
int rfxb_batch_debug_fault(RfxbBatch* batch, int cta, int wait_limit);
int rfxb_batch_debug_poison(RfxbBatch* batch, int list, int index);

/* Host only, no device needed: the work list (x ranges of (TY x 32) tiles)
 * that a batch of plans with these shapes launches for one step, for tests
 * of the tiling.  dims: 5 ints per plan (nx, ny, nz, CPML layers, CPML axes
 * bits x=1 y=2 z=4); resident: the CTA capacity the lists are balanced for.
 * which: 0 every tile on one kernel; 1 / 2 forward CPML-free / staged-psi
 * tiles; 3 / 4 reverse CPML-free / CPML tiles; 5 / 6 the reverse CPML tiles
 * split into those that reach a y slab (variant 2) and the rest (variant 4);
 * 7 / 8 / 9 a two-step pass's two-step tiles / one-step CPML-free work /
 * one-step CPML work (for 7 the plan index carries, from bit 16 on, where the
 * item also stores its intermediate state: 1 every plane, 2 its first plane,
 * 4 its last plane).
 * out: 5 ints per item (plan, y0, z0, xa, xb), *n_out the item count (with
 * out == NULL only the count).  A diagnostic of this implementation. */
int rfxb_debug_work_lists(int n_plans, const int32_t* dims, int32_t resident, int32_t which, int32_t* out,
                          int32_t cap, int32_t* n_out);

#ifdef __cplusplus
}
#endif

#endif /* RFXB200_H */
