/*
 * bmc_b200.h -- C ABI of the B200 (sm_100a) Bloch-McConnell simulator and Levenberg-Marquardt fitter.
 *
 * Plain C: pointers, sizes and status codes; no C++ or torch types cross this boundary.
 * Every pointer named `d_*` is DEVICE memory owned by the caller; `h_*` is host memory.
 * Every call is asynchronous on the given CUDA stream (`stream` is a cudaStream_t, NULL = legacy
 * default stream) and returns a status; `bmc_last_error` gives the message of the last failure
 * on the calling thread. Exceptions never cross the ABI.
 *
 * Data layout (the reference's, BMC-JAX simulation/params.py:18-49 and simulation/events.py:20-32):
 *   params   d_params[n_fields][n_voxels], float64, rows in SimParams order with every CEST field
 *            expanded into n_cest rows:
 *              water_r1, water_r2, water_f, cest_k[n_cest], cest_f[n_cest], cest_dw[n_cest],
 *              cest_r1[n_cest], cest_r2[n_cest], mt_k, mt_f, mt_dw, mt_r1, mt_r2,
 *              mt_lineshape (0 none, 1 Lorentzian, 2 super-Lorentzian, as a float), b0, gamma,
 *              b0_inhom, rel_b1.            n_fields = 13 + 5 n_cest   (BMC_N_FIELDS)
 *   events   six arrays [n_offsets][n_events] (row-major by offset): type int32 (0 DELAY,
 *            1 RF_PULSE, 2 GRADIENT, 3 ADC, 4 SPOILER), dt [s], rf_amp [Hz], rf_phase [rad],
 *            rf_freq [Hz] float64, adc_idx int32 (carried, not used by the solver).
 *   state    N = 3 (1 + n_cest) + 1 entries: water x, CEST x..., water y, CEST y..., water z,
 *            CEST z..., MT z (simulation/matrix.py:224-234). d_m0[n_voxels][N].
 *   output   Z[n_voxels][n_offsets] = state[mz_loc] after the last event of every offset, or
 *            the whole state [n_voxels][n_offsets][N] when mz_loc < 0.
 */
#ifndef BMC_B200_H
#define BMC_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BMC_ABI_VERSION 4
#define BMC_MAX_CEST 5             /* water + up to five CEST pools + MT: N <= 19 */
#define BMC_MAX_TANGENTS 8
#define BMC_N_FIELDS(n_cest) (13 + 5 * (n_cest))

typedef enum {
    BMC_OK = 0,
    BMC_ERR_INVALID = 1,           /* a size, pointer or option is out of range */
    BMC_ERR_CUDA = 2,              /* a CUDA runtime call failed */
    BMC_ERR_UNSUPPORTED = 3,       /* e.g. n_cest above BMC_MAX_CEST */
    BMC_ERR_NUMERIC = 4,           /* reserved; see "Numerical failures" below */
} bmc_status;

/* Numerical failures. The calls are asynchronous, so a failure found while the kernels run cannot be
 * returned as a status: a chain whose generator has a non-finite norm, or that would need more
 * squarings than the cap of 200, carries NaN to its outputs (Z, tangents, fitted values), as the
 * reference's NaN propagates. Callers test the outputs with isfinite. */

/* precision of the propagation arithmetic. BMC_F64: float64, except that in the forward model without
 * tangents the Taylor terms below 1e-6 of the state (by the series bound) are formed in float32 and
 * added to the float64 state once per sub-step, at most ~2e-13 of the state per event. Tangents, the
 * dense path for long events and the LM arithmetic are float64 throughout. BMC_F32: float32 Taylor
 * propagation, float64 dense path (about 1e-4 in Z over thousands of pulse samples, the level of the
 * reference's own float32 path). BMC_MIXED: the state and the first Taylor term of every sub-step in
 * float64 (more leading terms where their bound exceeds three times the state), every later term formed
 * in float32, and a truncation tolerance of 1e-8 per sub-step: the state itself is never rounded to
 * float32 (measured: ~4e-10 in Z over the 4,023-event benchmark train). Forward model only; float64
 * dense path. */
#define BMC_F64 0
#define BMC_F32 1
#define BMC_MIXED 2

/* special tangent seeds (bmc_tangents.field_row) */
#define BMC_SEED_NONE (-1)         /* only d_dm0 drives this tangent */
#define BMC_SEED_SPREAD_SIGMA (-2) /* derivative with respect to the B0-spread width sigma [Hz] */

typedef struct {
    int32_t n_voxels;
    int32_t n_offsets;
    int32_t n_events;
    int32_t n_cest;                /* 0 .. BMC_MAX_CEST */
    int32_t mz_loc;                /* state index returned as Z; < 0 returns the full state */
    int32_t reset_after_adc;       /* 1: the state returns to M0 after every ADC (reference default) */
    int32_t precision;             /* BMC_F64, BMC_F32 or BMC_MIXED */
    int32_t reserved;
} bmc_problem;

typedef struct {
    const int32_t* d_type;
    const double* d_dt;
    const double* d_rf_amp;
    const double* d_rf_phase;
    const double* d_rf_freq;
    const int32_t* d_adc_idx;      /* may be NULL */
} bmc_events;

/* B0 spread inside a voxel (simulation/spread.py:38-106): Z is the weighted mean over n_nodes
 * isochromats, node j at b0_inhom + sigma u_j / (gamma b0 / 2 pi). NULL spread = one isochromat. */
typedef struct {
    int32_t n_nodes;               /* <= 64 */
    const double* h_u;             /* [n_nodes] offsets in units of sigma */
    const double* h_w;             /* [n_nodes] weights, summing to 1 */
    const double* d_sigma_hz;      /* [n_voxels] width per voxel [Hz] */
} bmc_spread;

/* Forward-mode tangents: tangent p seeds d(field_row[p]) = d_seed[p][voxel] (per voxel) and
 * dM0 = d_dm0[p][voxel][N] (NULL = 0). BMC_SEED_SPREAD_SIGMA seeds d(sigma) instead of a field. */
typedef struct {
    int32_t n_tangents;            /* 1 .. BMC_MAX_TANGENTS */
    int32_t field_row[BMC_MAX_TANGENTS];
    const double* d_seed;          /* [n_tangents][n_voxels] */
    const double* d_dm0;           /* [n_tangents][n_voxels][N] or NULL */
} bmc_tangents;

/* Free parameters of a Levenberg-Marquardt fit (fitting/params.py:38-112, fitting/joint.py:99-138).
 * Slot p writes x_phys = x_scaled * scale[p] into params row field_row[p] as
 *   mode 0 "value": field = x_phys;  1 "factor": field = base * x_phys;  2 "add": field = base + x_phys
 * or, for field_row == BMC_SLOT_M_START, scales the start state (mode 0: initial_state(params) * x,
 * rebuilt from the current pools; mode 1: d_m0 * x), or for BMC_SLOT_SPREAD_SIGMA sets the spread
 * width. Where d_free[v][p] == 0 the slot is held at its carried value and its step is exactly zero. */
#define BMC_SLOT_M_START (-3)
#define BMC_SLOT_SPREAD_SIGMA (-2)
typedef struct {
    int32_t n_params;              /* 1 .. BMC_MAX_TANGENTS */
    int32_t n_iter;
    double lam0;
    int32_t field_row[BMC_MAX_TANGENTS];
    int32_t mode[BMC_MAX_TANGENTS];
    double scale[BMC_MAX_TANGENTS];
    double lo[BMC_MAX_TANGENTS];   /* bounds, scaled units */
    double hi[BMC_MAX_TANGENTS];
    const double* d_free;          /* [n_voxels][n_params] 1/0, or NULL = all free */
    int32_t n_points_skip;         /* leading simulated offsets left out of the residual (skip_first) */
    int32_t reserved;
} bmc_fit_spec;

/* Library identity. */
int32_t bmc_abi_version(void);
const char* bmc_version(void);

/* Message of the last non-OK status on this thread (copied, NUL-terminated). Returns its length. */
size_t bmc_last_error(char* buf, size_t buf_len);

/* Free the cached device workspaces of every device (call with no work in flight). */
bmc_status bmc_release(void);

/*
 * Forward model. Replaces simulation/simulate.py:134-148 (simulate_spectrum, vmapped over offsets),
 * simulation/voxels.py:89-129 (simulate_voxels), simulation/spread.py:77-106
 * (simulate_spectrum_spread, with `spread`) and fitting/experiment.py:58-61 (Experiment.simulate).
 * d_out: [n_voxels][n_offsets] (mz_loc >= 0) or [n_voxels][n_offsets][N].
 */
bmc_status bmc_simulate(const bmc_problem* prob, const double* d_params, const bmc_events* ev,
                        const double* d_m0, const bmc_spread* spread, double* d_out, void* stream);

/*
 * Forward model, keeping the state after every event (the reference's return_full_trajectory=True,
 * simulation/simulate.py:80-132): d_traj[n_voxels][n_offsets][n_events][N], float64 propagation.
 */
bmc_status bmc_simulate_trajectory(const bmc_problem* prob, const double* d_params, const bmc_events* ev,
                                   const double* d_m0, double* d_traj, void* stream);

/*
 * Forward model and its forward-mode tangents: Z and dZ along each seeded direction.
 * Replaces the jax.jacfwd of the model in fitting/lm.py:39, fitting/joint.py:300,317 and
 * design/crlb.py:57. d_z: [n_voxels][n_offsets]; d_jz: [n_tangents][n_voxels][n_offsets]
 * (state index prob->mz_loc, which must be >= 0).
 *
 * Two kernels compute the same derivatives. Forward mode carries every tangent through every event as
 * a dual number (one launch per tangent; two per launch for at most one CEST pool). Where each row's
 * state evolves in a single event -- an RF block or a delay; no spoiler or gradient; no readout that
 * resets the state before the row ends: the CW Z-spectra and B1 ladders -- and two or more tangents are
 * asked for, one launch computes the Frechet derivative of that event's exponential in the readout's
 * direction, and every tangent follows from it (reverse mode through the exponential). The results agree
 * to rounding (~1e-12 relative). bmc_lm_fit chooses the same way. An uneven plan (bmc_uneven_create)
 * decides once when it is built: where every row's evolving events are one block of at most two events
 * repeated at most 64 times (or at most two events once), its tangents and its primal passes both go
 * through the block kernel (no read-back, so also inside a captured graph). Choosing reads one flag back from
 * the device (a stream synchronisation), so a stream being captured into a CUDA graph keeps forward
 * mode. bmc_set_tangent_mode(BMC_TANGENTS_FORWARD) makes forward mode the only one (process-wide);
 * BMC_TANGENTS_AUTO (the default) restores the choice.
 */
#define BMC_TANGENTS_AUTO 0
#define BMC_TANGENTS_FORWARD 1
bmc_status bmc_set_tangent_mode(int32_t mode);
bmc_status bmc_simulate_jvp(const bmc_problem* prob, const double* d_params, const bmc_events* ev,
                            const double* d_m0, const bmc_spread* spread, const bmc_tangents* tan,
                            double* d_z, double* d_jz, void* stream);

/*
 * Second-order tangents for protocol design. Replaces the derivative of the Cramer-Rao bound with
 * respect to the design that design/optimize.py:43-113 takes by automatic differentiation through
 * jax.jacfwd of the model (design/crlb.py:57): Z and its tangents as bmc_simulate_jvp computes them,
 * plus the derivative of both along one direction of the inputs -- d_params_dir [n_fields][n_voxels]
 * and d_m0_dir [n_voxels][N] (either NULL = 0), and ev_dir (NULL = 0), whose d_dt, d_rf_amp,
 * d_rf_phase and d_rf_freq are the per-unit change of the table's fields ([n_offsets][n_events] like
 * ev; NULL fields = 0; d_type and d_adc_idx are not read). d_dz: [n_voxels][n_offsets];
 * d_djz: [n_tangents][n_voxels][n_offsets]. Exact derivatives of the computed approximation: every
 * scalar of the chain carries its design derivative, every state entry its tangents (forward mode over
 * forward mode); long events take a dense scaling and squaring per chain. float64, mz_loc >= 0, no
 * spread, tangents of params fields only (no d_dm0). One launch per tangent; meant for the small
 * problems of a design (truths x protocol rows), not for bulk simulation.
 */
bmc_status bmc_simulate_design_jvp(const bmc_problem* prob, const double* d_params, const bmc_events* ev,
                                   const double* d_m0, const double* d_params_dir, const bmc_events* ev_dir,
                                   const double* d_m0_dir, const bmc_tangents* tan, double* d_z, double* d_jz,
                                   double* d_dz, double* d_djz, void* stream);

/*
 * Bounded Levenberg-Marquardt of every voxel, all iterations on the device.
 * Replaces fitting/lm.py:20-67 as driven by fitting/independent.py:51-129 (fit_batch, vmapped over
 * voxels) and the uncoupled branch of fitting/joint.py:359-374 (per-sample damping, `free` holds).
 * d_z_meas: [n_voxels][n_offsets - n_points_skip]; d_x0: [n_voxels][n_params] scaled units.
 * d_x_out: [n_voxels][n_params] scaled. d_cost_traj: [n_voxels][n_iter] or NULL (the cost after each
 * step, fitting/lm.py:61). d_x_traj: [n_voxels][n_iter][n_params] or NULL.
 * The float64 normal equations are solved by Gaussian elimination with partial pivoting.
 */
bmc_status bmc_lm_fit(const bmc_problem* prob, const double* d_params, const bmc_events* ev,
                      const double* d_m0, const bmc_spread* spread, const bmc_fit_spec* spec,
                      const double* d_z_meas, const double* d_x0, double* d_x_out,
                      double* d_cost_traj, double* d_x_traj, void* stream);

/*
 * Per-sample normal-equation blocks for a coupled joint fit (fitting/joint.py:149-162, 344-348):
 * for every voxel v, H_v = J_v^T J_v, g_v = J_v^T r_v and c_v = r_v^T r_v, from the residual
 * d_r[n_voxels][n_points] and the tangents d_jz[n_tangents][n_voxels][n_points].
 * d_H: [n_voxels][n_tangents][n_tangents], d_g: [n_voxels][n_tangents], d_c: [n_voxels].
 */
bmc_status bmc_normal_blocks(int32_t n_voxels, int32_t n_points, int32_t n_tangents,
                             const double* d_r, const double* d_jz, double* d_H, double* d_g,
                             double* d_c, void* stream);

/*
 * bmc_simulate without any device allocation. No counterpart in the reference: an addition for
 * callers that cannot let a library call cudaMalloc -- a handler inside JAX/XLA (JAX reserves most of
 * the GPU's memory for its own allocator), code under another framework's fixed memory budget, or a
 * latency-bound pipeline (cudaMalloc/cudaFree synchronise the device). Same arguments and results as
 * bmc_simulate (bit-identical Z: every chain chooses its own Taylor degree and float32 switch point, so
 * the order the chains run in does not matter). Its only scratch, the preprocessed event records and a
 * status word, lives in one static device array of 32 MiB per GPU that loads the library, held until
 * exit, so n_offsets x n_events may be at most 699,045 records in float64 (1,048,568 in float32);
 * larger tables are rejected with BMC_ERR_INVALID and a message. The CUDA driver reserves the array
 * when it loads the library's device code on a device, which under CUDA's default lazy loading is the
 * first bmc_* call there: a caller whose framework reserves most of the GPU up front (JAX's
 * preallocation) makes one call, e.g. a bmc_simulate_noalloc of a tiny problem, on every device before
 * that reservation, or runs with CUDA_MODULE_LOADING=EAGER. The first call on a device also takes the
 * array's device address and uploads the Taylor tables (issue it before any stream capture). Every call
 * reuses the same array and overwrites the previous call's records: calls that overlap on the GPU
 * (other streams, other host threads) race and must be serialised by the caller. Numerical failures
 * show as NaN in d_out, as for bmc_simulate; the status word is not reported.
 */
bmc_status bmc_simulate_noalloc(const bmc_problem* prob, const double* d_params, const bmc_events* ev,
                                const double* d_m0, const bmc_spread* spread, double* d_out, void* stream);

/*
 * Uneven batches: voxels of one pool count with their own event tables (different offsets, pulse
 * trains) in one launch. BMC-JAX expresses one event table per Experiment (fitting/experiment.py:43-46,
 * fitting/joint.py:255), so an uneven batch is there one call per shape class; these entry points run
 * the class mix at once and give every voxel the result its own class's call gives.
 *   bmc_uneven_create: tables t = 0..n_tables-1 of h_n_offsets[t] x h_n_events[t] events, their six
 *     arrays concatenated in table order in `ev` (device); h_voxel_table[v] names voxel v's table.
 *     Builds the chain map (canonical order: voxel-major, then table row) and the tables' records on the
 *     device (allocates; synchronises the device once). *n_chains = total rows; h_chain_start (host,
 *     n_voxels + 1 entries, may be NULL) receives the first chain of every voxel.
 *   bmc_uneven_simulate: d_params [13 + 5 n_cest][n_voxels], d_m0 [n_voxels][N], an optional B0 spread
 *     (as for bmc_simulate, sigma per voxel); d_z [n_chains] = state mz_loc after each chain's last
 *     event; with tangents (field rows -1..n_fields-1, and BMC_SEED_SPREAD_SIGMA with a spread),
 *     d_jz [n_tangents][n_chains]. d_active [n_voxels] (device, may be NULL = all): voxels with 0 are
 *     skipped and their outputs left as they were (a fit re-launches only what moved, with no host
 *     synchronisation). Replaces simulation/simulate.py:134-148 + voxels.py:89-129 + spread.py:77-106 per
 *     shape class, and the jacfwd of fitting/joint.py:300,317.
 */
typedef struct {
    int32_t n_tables;
    const int32_t* h_n_offsets;    /* host [n_tables] */
    const int32_t* h_n_events;     /* host [n_tables] */
    bmc_events ev;                 /* device: the tables' arrays, concatenated */
} bmc_table_set;

bmc_status bmc_uneven_create(int32_t n_cest, int32_t n_voxels, const int32_t* h_voxel_table,
                             const bmc_table_set* tables, int32_t mz_loc, int32_t reset_after_adc, void** plan,
                             int64_t* n_chains, int64_t* h_chain_start);
bmc_status bmc_uneven_simulate(const void* plan, const double* d_params, const double* d_m0,
                               const bmc_spread* spread, const bmc_tangents* tangents, const int32_t* d_active,
                               double* d_z, double* d_jz, void* stream);
bmc_status bmc_uneven_destroy(void* plan);
/* The norm ||X|| = dt ||A|| above which an event of this plan's chains is exponentiated densely (one lane
 * group per chain, scaling and squaring) rather than by the truncated Taylor action (one lane per chain);
 * 0 restores the library's default (100). A tuning knob with no counterpart in the reference: both
 * paths meet the same tolerance, only their speed differs (bmc_b200.autotune measures it per plan). */
bmc_status bmc_uneven_set_dense_switch(void* plan, double norm);
/* *out = 1 when this plan's passes take the block kernel in the current tangent mode (every row one
 * repeated block of at most two events, BMC_TANGENTS_AUTO): its events are then all exponentiated
 * densely and the threshold above is not consulted; 0 otherwise. Host only, no device work. */
bmc_status bmc_uneven_uses_block_kernel(const void* plan, int32_t* out);

/*
 * The damped joint step with one value shared by every sample (fitting/joint.py:149-162's
 * (H + lam (diag H + 1e-9 I)) d = -g, solved through the Schur complement of the shared column).
 *   bmc_normal_segments: per voxel v, over its chains d_chain_start[v] .. d_chain_start[v+1]-1:
 *     d_H [n_voxels][P][P] = J J^T, d_g [n_voxels][P] = J r, d_c [n_voxels] = r^T r, with
 *     d_jz [P][n_chains] and d_r [n_chains]; P <= 9.
 *   The damping is `lam`, or *d_lam when d_lam (device, one double) is not NULL: a loop that keeps lambda
 *   on the device then needs no host synchronisation.
 *   bmc_schur_step: P = n_local + n_shared (the shared column last, n_shared 0 or 1, n_local <= 8);
 *     d_free [n_voxels][n_local] (1 free, 0 held; NULL = all free) -> d_dx_local [n_voxels][n_local],
 *     d_dx_shared [1]. d_work holds (2 n_local + 4) n_voxels + 4 doubles. The shared sums are taken in
 *     a fixed order (deterministic).
 *   bmc_schur_eliminate + bmc_schur_back: the same step in two halves, for voxels sharded over several
 *     GPUs. eliminate writes the per-voxel elimination into d_work ((2 n_local + 4) n_voxels doubles) and
 *     this shard's four Schur sums into d_sums [4]; the caller adds d_sums over every shard (e.g. one
 *     4-double all-reduce) and passes the total to back, which forms the shared step and each voxel's.
 */
bmc_status bmc_normal_segments(int32_t n_voxels, int32_t n_params, int64_t n_chains, const int64_t* d_chain_start,
                               const double* d_jz, const double* d_r, double* d_H, double* d_g, double* d_c,
                               void* stream);
bmc_status bmc_schur_step(int32_t n_voxels, int32_t n_local, int32_t n_shared, const double* d_H, const double* d_g,
                          const double* d_free, double lam, const double* d_lam, double* d_dx_local,
                          double* d_dx_shared, double* d_work, void* stream);
bmc_status bmc_schur_eliminate(int32_t n_voxels, int32_t n_local, int32_t n_shared, const double* d_H,
                               const double* d_g, const double* d_free, double lam, const double* d_lam,
                               double* d_work, double* d_sums, void* stream);
bmc_status bmc_schur_back(int32_t n_voxels, int32_t n_local, int32_t n_shared, const double* d_sums, double lam,
                          const double* d_lam, const double* d_work, double* d_dx_local, double* d_dx_shared,
                          void* stream);

/*
 * Learned warm start: a multilayer perceptron that maps a measured saturation ladder to normalised
 * starting values for bmc_lm_fit, trained and evaluated with tcgen05 tensor-core GEMMs (bf16 inputs,
 * fp32 accumulation). BMC-JAX has no learned component; these entry points are the
 * bmc_mlp_{forward,backward,adam_step} of the build's boundary (starting values for
 * fitting/independent.py:51-129, whose plain x0 stays the fallback).
 *
 * Network: x (n_in) -> n_hidden_layers x [affine, GELU (erf form)] of width n_hidden -> affine ->
 * y (n_out). Every dimension is padded: in_pad = n_in rounded up to 64, out_pad = n_out rounded up
 * to 64; n_hidden must be a multiple of 128 (<= 1024), n_out <= 128, 1..8 hidden layers.
 * Parameters (d_params, float32, the master copy; also d_grad, d_m, d_v): for each layer l in order
 * (hidden layers, then the output layer) W_l [out_l][in_l] row-major, then b_l [out_l], with
 * in_0 = in_pad, in_l = n_hidden, out_l = n_hidden, out_L = out_pad; padded rows and columns must be
 * zero (they then stay zero). The shadow (bf16, `shadow_bytes`) holds W_l and W_l^T per layer, as the
 * tensor cores read them; bmc_mlp_sync rebuilds it from d_params and bmc_mlp_adam_step keeps it current.
 * The work buffer (256-byte aligned, `work_bytes` for a batch size) holds the activations a backward
 * pass needs; its first int32 is a status word: bit 0 is set when a GEMM gave up waiting for its
 * tensor-core operations (about two seconds), and the caller clears it.
 * Inputs x [batch][n_in] float32 are normalised as (x - d_in_shift[i]) * d_in_scale[i] (either may
 * be NULL); outputs d_y [batch][n_out] float32 (may be NULL). Loss: mean over batch and outputs of
 * (y - target)^2, added to *d_loss (may be NULL); gradients overwrite d_grad.
 */
typedef struct {
    int32_t n_in;
    int32_t n_hidden;
    int32_t n_hidden_layers;
    int32_t n_out;
} bmc_mlp_shape;

bmc_status bmc_mlp_sizes(const bmc_mlp_shape* shape, int64_t batch, int64_t* n_params, int64_t* shadow_bytes,
                         int64_t* work_bytes);
bmc_status bmc_mlp_sync(const bmc_mlp_shape* shape, const float* d_params, void* d_shadow, void* stream);
bmc_status bmc_mlp_forward(const bmc_mlp_shape* shape, const float* d_params, const void* d_shadow,
                           const float* d_x, const float* d_in_shift, const float* d_in_scale, int64_t batch,
                           float* d_y, void* d_work, int32_t keep_for_backward, void* stream);
bmc_status bmc_mlp_backward(const bmc_mlp_shape* shape, const void* d_shadow, const float* d_target, int64_t batch,
                            void* d_work, float* d_grad, float* d_loss, void* stream);
bmc_status bmc_mlp_adam_step(const bmc_mlp_shape* shape, float* d_params, const float* d_grad, float* d_m,
                             float* d_v, void* d_shadow, int32_t step, float lr, float beta1, float beta2, float eps,
                             void* stream);
/* bmc_mlp_adam_step with the step count on the device: step *d_step + 1, then *d_step is advanced, so
 * that a training step captured into a CUDA graph can be replayed. */
bmc_status bmc_mlp_adam_step_dev(const bmc_mlp_shape* shape, float* d_params, const float* d_grad, float* d_m,
                                 float* d_v, void* d_shadow, int32_t* d_step, float lr, float beta1, float beta2,
                                 float eps, void* stream);

/*
 * Diagnostics (no counterpart in the reference: measurement support for the benchmark).
 * bmc_simulate_counted: bmc_simulate that also adds the work it executed to d_work[5] (device,
 *   zeroed by the caller): [0] Taylor sub-step terms each chain needed (one sparse operator product
 *   each), [1] dense-path Horner column products, [2] dense-path squarings, [3] Taylor terms executed
 *   (a warp runs to the largest need among its chains), [4] of the terms in [0], those formed in float32.
 * bmc_simulate_jvp_counted: bmc_simulate_jvp that adds the same five counts to d_work[5], summed over
 *   its launches: in forward mode one per tangent (two per launch for at most one CEST pool), each
 *   carrying the primal and its tangents through the same steps as dual numbers; in the adjoint kernel
 *   one launch whose [1] counts the Horner column products of the pair (exp, Frechet derivative) and
 *   [2] its squarings.
 * bmc_probe_fma_peak: launches `blocks` x 256 threads of 8 independent FMA chains x `iters`
 *   (float64 or float32) and returns the FLOPs one launch executes, to time against.
 */
bmc_status bmc_simulate_counted(const bmc_problem* prob, const double* d_params, const bmc_events* ev,
                                const double* d_m0, const bmc_spread* spread, double* d_out,
                                unsigned long long* d_work, void* stream);
bmc_status bmc_simulate_jvp_counted(const bmc_problem* prob, const double* d_params, const bmc_events* ev,
                                    const double* d_m0, const bmc_spread* spread, const bmc_tangents* tan,
                                    double* d_z, double* d_jz, unsigned long long* d_work, void* stream);
bmc_status bmc_probe_fma_peak(int32_t precision, int32_t blocks, int32_t iters, double* flops_per_launch,
                              void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BMC_B200_H */
