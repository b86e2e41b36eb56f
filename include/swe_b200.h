/* swe_b200.h -- C ABI of the B200 (sm_100a) shallow-water finite-volume step.
 *
 * Drop-in boundary for the hot path of arsanjeevk/gpu-hybrid-flood-forecasting.
 * Each entry point replaces one function of the reference (paths inside the
 * reference project):
 *
 *   swe_domain_create   NumpyShallowWaterSolver.__init__ / ShallowWaterSolver.__init__
 *                       src/hybrid_flood/numpy_solver/shallow_water_2d.py:333-365,
 *                       src/hybrid_flood/jax_solver/shallow_water_2d.py:213-253
 *                       (plus boundary codes, jax_solver/boundary_conditions.py:9-26)
 *   swe_step            finite_volume_step(state, params, dt, time_s)
 *                       numpy_solver/shallow_water_2d.py:277-327, jax_solver/numerics.py:312-369
 *   swe_max_inverse_dt  the reduction inside compute_cfl_dt
 *                       numpy_solver/shallow_water_2d.py:269-273, jax_solver/numerics.py:299-304
 *   swe_cfl_dt          compute_cfl_dt(state, params)
 *                       numpy_solver/shallow_water_2d.py:267-274, jax_solver/numerics.py:297-309
 *   swe_rainfall_rate   rainfall_rate(params, time_s)
 *                       numpy_solver/shallow_water_2d.py:254-264, jax_solver/numerics.py:286-294
 *   swe_run             NumpyShallowWaterSolver.run / ShallowWaterSolver.run / integrate_to_outputs
 *                       numpy_solver/shallow_water_2d.py:382-424,
 *                       jax_solver/shallow_water_2d.py:278-306, jax_solver/numerics.py:372-434
 *   swe_advance         the fixed-count step loop of jax_solver/benchmarking.py:46-57,
 *                       with CFL-limited dt as in the run loop
 *
 * Conventions
 *   - Fields are float32, row-major [rows][cols]: row index = y (northward),
 *     column = x (eastward).  `pitch` is the row stride in ELEMENTS (>= cols).
 *   - State and output buffers are caller-owned DEVICE pointers.  Static fields
 *     passed to swe_domain_create may be host or device pointers (see
 *     `fields_on_host`); the domain keeps its own packed device copy.
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).  All work is
 *     enqueued on it; entry points that return a host value synchronise it.
 *   - Every entry point returns an int status (SWE_OK = 0).  swe_last_error()
 *     gives the message of the last failure on the calling thread.
 *   - A domain handle may be used by one host thread at a time.
 */
#ifndef SWE_B200_H
#define SWE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SWE_OK 0
#define SWE_ERR_INVALID 1   /* bad argument: the reference raises ValueError */
#define SWE_ERR_CUDA 2      /* CUDA runtime error */
#define SWE_ERR_MAX_STEPS 3 /* max_steps ran out: the reference raises RuntimeError */
#define SWE_ERR_NONFINITE 4 /* NaN/Inf reached the CFL reduction */
#define SWE_ERR_NO_DEVICE 5 /* no usable sm_100 device */

#define SWE_REFLECTIVE 0 /* jax_solver/boundary_conditions.py:9 */
#define SWE_OPEN 1       /* jax_solver/boundary_conditions.py:10 (zero-gradient copy) */

#define SWE_ARITH_EXACT 0 /* every operation rounded as the reference NumPy solver */
#define SWE_ARITH_FAST 1  /* FMA + hardware approximations, tolerance-checked */

typedef struct swe_domain *swe_domain_t;

typedef struct {
    int32_t rows, cols;
    double dx, dy;             /* cell size (m); the reference uses dx = dy = resolution_m */
    double gravity;            /* m s^-2, reference default 9.81 */
    double cfl;                /* reference default 0.45 */
    double dry_tolerance;      /* m, reference default 1e-4 */
    double max_dt;             /* s, reference default 10 */
    double default_rainfall;   /* m/s outside the hyetograph record */
    int32_t boundary[4];       /* left, right, bottom, top: SWE_REFLECTIVE / SWE_OPEN */
    int32_t n_rain;            /* hyetograph length (>= 1) */
    const float *rain_times;   /* HOST, n_rain times (s), increasing */
    const float *rain_rates;   /* HOST, n_rain rates (m/s) */
    const float *bed;          /* rows*cols, contiguous */
    const float *manning_n;    /* rows*cols */
    const uint8_t *domain_mask;/* rows*cols, nonzero = active */
    const float *rainfall_multiplier; /* rows*cols, or NULL = domain_mask as 0/1 */
    int32_t fields_on_host;    /* 1: bed/manning_n/domain_mask/multiplier are host pointers */
    int32_t arithmetic;        /* SWE_ARITH_EXACT or SWE_ARITH_FAST */
} swe_domain_desc;

typedef struct {
    double final_time_s;   /* NumpyResult.final_time_s */
    int32_t outputs_written;
    int32_t steps_used;
    int32_t status;        /* SWE_OK, SWE_ERR_MAX_STEPS or SWE_ERR_NONFINITE */
    int32_t reserved;
    /* FP64 mass ledger (m^3): volume0, volume, rain_in, outflow, clip_gain, mask_loss.
     * volume - (volume0 + rain_in - outflow + clip_gain - mask_loss) is the closing error. */
    double ledger[6];
} swe_run_result;

/* Create a domain: validates the descriptor, packs bed and n^2 (with the mask)
 * into pitched device planes, uploads the hyetograph.  Allocates device memory. */
int swe_domain_create(const swe_domain_desc *desc, swe_domain_t *out);
int swe_domain_destroy(swe_domain_t d);

/* One step: out = finite_volume_step(in, params, dt, time_s).  `dt` and
 * `time_s` are float64 as in the reference; the kernel rounds dt, dt*rate and
 * dt*gravity to float32 where the reference does.  Outputs must not alias inputs. */
int swe_step(swe_domain_t d, const float *h, const float *hu, const float *hv, int64_t pitch_in,
             float *h_out, float *hu_out, float *hv_out, int64_t pitch_out, double dt,
             double time_s, void *stream);

/* Largest (|u|+c)/dx + (|v|+c)/dy over active cells (float32, as the reference). */
int swe_max_inverse_dt(swe_domain_t d, const float *h, const float *hu, const float *hv,
                       int64_t pitch, float *max_inverse_dt_out, void *stream);

/* compute_cfl_dt: min(cfl / max_inverse_dt, max_dt), or max_dt if the maximum is 0. */
int swe_cfl_dt(swe_domain_t d, const float *h, const float *hu, const float *hv, int64_t pitch,
               double *dt_out, void *stream);

/* rainfall_rate: np.interp of the hyetograph at time_s (float64). */
int swe_rainfall_rate(swe_domain_t d, double time_s, double *rate_out);

/* Adaptive run to fixed output times (the reference run loop: dt = min(cfl_dt,
 * target - t), an output is recorded when t >= target - 1e-7).  The clock is
 * float64 and lives on the device; the host only polls completion.
 *   output_times: HOST float32[n_out], output_times[0] == 0, strictly increasing
 *   out_*: DEVICE float32[n_out][rows][cols] (slot 0 receives the initial state)
 * Returns SWE_ERR_MAX_STEPS (result filled) when max_steps was insufficient. */
int swe_run(swe_domain_t d, const float *h0, const float *hu0, const float *hv0,
            int64_t pitch_in, const float *output_times, int32_t n_out, int32_t max_steps,
            float *out_h, float *out_hu, float *out_hv, swe_run_result *result, void *stream);

/* swe_run with the initial state and the outputs in HOST memory: the state is
 * copied in, and each output is copied back to out_* (HOST float32
 * [n_out][rows][cols]) as soon as the run has recorded it, on a second stream
 * while the later steps run.  Page-locked (pinned) host buffers let the copies
 * overlap the steps; pageable ones work but serialise them.  Same results,
 * validation and status codes as swe_run. */
int swe_run_host(swe_domain_t d, const float *h0, const float *hu0, const float *hv0, int64_t pitch_in,
                 const float *output_times, int32_t n_out, int32_t max_steps, float *out_h, float *out_hu,
                 float *out_hv, swe_run_result *result, void *stream);

/* Advance (h, hu, hv) in place by exactly n_steps CFL-limited steps starting at
 * time start_s; the state, final time and ledger are returned in `result`. */
int swe_advance(swe_domain_t d, float *h, float *hu, float *hv, int64_t pitch, int32_t n_steps,
                double start_s, swe_run_result *result, void *stream);

/* Device-resident stepping: the reference's step loop
 * (`state = finite_volume_step(state, params, compute_cfl_dt(state), t)`,
 * numpy_solver/shallow_water_2d.py:402-412) with the state kept in the
 * domain's own buffers between calls, so that a caller can advance in pieces
 * without copying the state in and out each time.
 *   swe_resident_load   copies (h, hu, hv) in and starts the float64 clock at
 *                       start_s (the initial CFL reduction is enqueued);
 *   swe_resident_steps  enqueues n_steps CFL-limited steps and returns without
 *                       waiting (as CUDA graphs of up to 32 steps, captured on
 *                       first use);
 *   swe_resident_prepare captures, without running anything, the graphs that
 *                       a call of n_steps steps uses, from either ping-pong
 *                       buffer (it may follow other steps), so that the
 *                       later swe_resident_steps only launches;
 *   swe_resident_store  copies the current state out and reports the clock,
 *                       the steps taken since the load and the FP64 ledger
 *                       (it synchronises the stream).
 * Any other run on the domain (swe_run, swe_advance, swe_advance_to, an
 * ensemble or strip advance) ends the resident state. */
int swe_resident_load(swe_domain_t d, const float *h, const float *hu, const float *hv, int64_t pitch,
                      double start_s, void *stream);
int swe_resident_steps(swe_domain_t d, int32_t n_steps, void *stream);
int swe_resident_prepare(swe_domain_t d, int32_t n_steps);
int swe_resident_store(swe_domain_t d, float *h, float *hu, float *hv, int64_t pitch,
                       swe_run_result *result, void *stream);

/* Number of kernel launches the last swe_run/swe_advance on this domain enqueued. */
int64_t swe_last_launch_count(swe_domain_t d);

/* Enable (1) or disable (0) CUDA-event timing of the step kernels that
 * swe_run/swe_advance enqueue (events on the caller's stream around the first
 * and the last step launch). */
int swe_set_timing(swe_domain_t d, int32_t enable);

/* Milliseconds between the start of the first and the end of the last step
 * kernel of the last timed swe_run/swe_advance, and the step launches between. */
int swe_last_step_time(swe_domain_t d, double *ms, int64_t *step_launches);

/* Scale every rain rate of the hyetograph by `scale` (>= 0; 1 restores it).
 * The differentiable rollout treats this scale as a parameter. */
int swe_domain_set_rain_scale(swe_domain_t d, double scale);

/* Replace the Manning n field (rows*cols contiguous, host or device); the
 * domain mask is kept. */
int swe_domain_set_manning(swe_domain_t d, const float *manning_n, int32_t on_host, void *stream);

/* Reverse mode of one step (no counterpart in the reference, which never
 * differentiates its solver): given lam = dL/dU_{k+1} and the state U_k that
 * was stepped with (dt, time_s), write lam_out = dL/dU_k and ADD dL/d(n^2)
 * into grad_n2 (rows*cols, device) and dL/d(rain scale) into *grad_rain_scale
 * (one device double).  dt is held fixed (stop-gradient).  lam_out may alias lam. */
int swe_adjoint_step(swe_domain_t d, const float *h, const float *hu, const float *hv, int64_t pitch,
                     const float *lam_h, const float *lam_hu, const float *lam_hv, int64_t lam_pitch,
                     float *lam_h_out, float *lam_hu_out, float *lam_hv_out, int64_t out_pitch,
                     float *grad_n2, double *grad_rain_scale, double dt, double time_s, void *stream);

/* Fixed-dt (or logged-dt) rollout with gauge observations: the forward of the
 * differentiable rollout (no counterpart in the reference).  (h, hu, hv)
 * advance IN PLACE by n_steps steps from t0: of dt each, or of dts[k] (host
 * float64 [n_steps], e.g. the log of an adaptive advance_to) when dts is
 * non-NULL; the clock is accumulated in float64 as in the run loop.  Every
 * obs_every steps the depths at the n_gauges flat cell indices (device int64,
 * row-major numbering) go to obs (device float32 [n_steps/obs_every][n_gauges]).
 * If ckpt is non-NULL the states at steps 0, ckpt_every, 2*ckpt_every, ...
 * below n_steps are stored there as [k][3][rows][cols]. */
int swe_rollout_forward(swe_domain_t d, float *h, float *hu, float *hv, int64_t pitch, int32_t n_steps,
                        double dt, double t0, const double *dts, const int64_t *gauge_index, int32_t n_gauges,
                        int32_t obs_every, float *obs, float *ckpt, int32_t ckpt_every, void *stream);

/* Reverse of swe_rollout_forward (same dt / dts): from its checkpoints and
 * dL/dobs (device, the layout of obs), writes dL/dU_0 to (lam_h, lam_hu,
 * lam_hv), and ADDS dL/d(n^2) into grad_n2 and dL/d(rain scale) into
 * *grad_rain_scale.  lam_in = 1: the lam planes hold dL/dU_{n_steps} on entry
 * (a loss on the final state); 0: they start at zero.  Each segment of
 * ckpt_every steps is recomputed from its checkpoint and reversed step by
 * step; seg (device, ckpt_every*3*rows*cols floats) and a second buffer of the
 * domain's hold two segments, so that the next segment is recomputed on a
 * stream of the domain's own while the current one is reversed on `stream`.
 * That stream waits for `stream`'s earlier work and `stream` waits for it
 * before the call's last work: callers see only `stream`. */
int swe_rollout_backward(swe_domain_t d, const float *ckpt, int32_t ckpt_every, int32_t n_steps,
                         double dt, double t0, const double *dts, const int64_t *gauge_index,
                         int32_t n_gauges, int32_t obs_every, const float *grad_obs, float *lam_h,
                         float *lam_hu, float *lam_hv, int64_t lam_pitch, int32_t lam_in, float *grad_n2,
                         double *grad_rain_scale, float *seg, void *stream);

/* Advance (h, hu, hv) IN PLACE from t_start to t_target with CFL-limited
 * steps (dt = min(cfl_dt, t_target - t)), at most max_steps of them: the
 * physics of one correction interval, advance_physics_to_time
 * (hybrid/coupled_forecast.py:123-161), with a float64 clock.
 * dt_log (device float64 [max_steps], or NULL) receives every step's dt, for
 * replaying the interval (swe_rollout_forward/backward with dts).
 * SWE_ERR_MAX_STEPS when the target was not reached within 1e-7 s. */
int swe_advance_to(swe_domain_t d, float *h, float *hu, float *hv, int64_t pitch, double t_start,
                   double t_target, int32_t max_steps, double *dt_log, swe_run_result *result, void *stream);

#define SWE_FEATURES_REFERENCE6 0 /* (h,u,v) standardised, rain/scale, terrain, roughness */
#define SWE_FEATURES_STATE5 1     /* (h, hu, hv, bed, rain mm/h), each standardised */

/* Network input features of a state, channels-last [rows][cols][C] in
 * float32 or bfloat16 (network_features, hybrid/coupled_forecast.py:53-79).
 * mean/stddev: host float[3] (REFERENCE6: h, u, v) or float[5] (STATE5);
 * rain_feature is the value of the rain channel (REFERENCE6: rate in mm/h
 * over the rain scale; STATE5: rate in mm/h, standardised here);
 * terrain/roughness: device rows*cols float32 (REFERENCE6 only, may be NULL). */
int swe_network_features(swe_domain_t d, const float *h, const float *hu, const float *hv, int64_t pitch,
                         int32_t layout, const float *mean, const float *stddev, float rain_feature,
                         const float *terrain, const float *roughness, void *out, int32_t out_bf16,
                         void *stream);

/* Output fields of a state in the common forecast schema (conserved_to_xarray,
 * src/hybrid_flood/structured_io.py:160-209): depth, x_velocity and y_velocity
 * (momentum / depth where depth > dry_tolerance, else 0) and velocity (their
 * hypot), each NaN off the domain mask.  Outputs are four device float32 planes
 * of pitch out_pitch; values equal the reference's NumPy arrays bit for bit. */
int swe_output_fields(swe_domain_t d, const float *h, const float *hu, const float *hv, int64_t pitch,
                      float *depth, float *x_velocity, float *y_velocity, float *speed, int64_t out_pitch,
                      void *stream);

/* In place y = act(y + bias[channel]) over a channels-last tensor of n elements
 * with `channels` innermost (the bias and ReLU of a convolution of the residual
 * U-Net, benchmark/pytorch_residual_net.py:47-76, fused into one pass).  y:
 * device bfloat16 (bf16 = 1) or float32; bias: device float32[channels];
 * relu = 1 applies max(., 0).  device: the CUDA device y lives on. */
int swe_bias_act_nhwc(void *y, int64_t n, int32_t channels, const float *bias, int32_t relu, int32_t bf16,
                      int32_t device, void *stream);

/* Volume-preserving residual correction (apply_residual_correction,
 * hybrid/coupled_forecast.py:82-120), with the clip of :199-200 fused in:
 * res = clip(residual, -clip_limits, clip_limits) per channel (host
 * float[res_channels], or NULL for none); h' = max(h + r*res_h, 0) on active
 * cells, scaled back to the predicted water volume (sums in float64);
 * velocities + r*res_(u,v) when res_channels == 3; momenta rebuilt on wet
 * cells.  residual element (row, col, ch) is residual[row*sr + col*sc + ch*sch]
 * in float32 or bfloat16 (residual_bf16), on the device.  Outputs may alias
 * the inputs. */
int swe_apply_correction(swe_domain_t d, const float *h, const float *hu, const float *hv, int64_t pitch,
                         const void *residual, int32_t residual_bf16, int64_t res_stride_row,
                         int64_t res_stride_col, int64_t res_stride_channel, int32_t res_channels,
                         const float *clip_limits, double relaxation, float *h_out, float *hu_out,
                         float *hv_out, int64_t out_pitch, void *stream);

/* ---- Batched ensemble (no single counterpart in the reference: it batches many
 * reference runs -- NumpyShallowWaterSolver.run per member, numpy_solver/
 * shallow_water_2d.py:382-424 -- into one launch per step). ---- */
typedef struct swe_ensemble *swe_ensemble_t;

/* Create an ensemble of n_members domains of any sizes (one swe_domain_desc
 * each, all with the same arithmetic).  Every member keeps its own float64
 * clock, CFL dt and mass ledger; one kernel launch advances all of them. */
int swe_ensemble_create(const swe_domain_desc *descs, int32_t n_members, swe_ensemble_t *out);
int swe_ensemble_destroy(swe_ensemble_t e);
int swe_ensemble_size(swe_ensemble_t e);

/* Rows each warp marches per work item (the tuning knob of the work list).
 * The default, chosen at creation, is the smallest march of at least 32 rows
 * whose work items fit the persistent grid in one round (256 when none does);
 * SWE_ENSEMBLE_ROWS overrides it.  swe_ensemble_rows_per_warp returns the
 * current value (-1 for a null handle). */
int swe_ensemble_set_rows_per_warp(swe_ensemble_t e, int32_t rows_per_warp);
int32_t swe_ensemble_rows_per_warp(swe_ensemble_t e);

/* Advance every member IN PLACE by n_steps of its own CFL dt, starting at
 * start_s[m] (NULL = 0).  h/hu/hv/pitch are arrays of n_members device
 * pointers / pitches; results receives n_members entries. */
int swe_ensemble_advance(swe_ensemble_t e, float *const *h, float *const *hu, float *const *hv,
                         const int64_t *pitch, int32_t n_steps, const double *start_s,
                         swe_run_result *results, void *stream);

/* Advance every member IN PLACE from start_s[m] to target_s with CFL-limited
 * steps, at most max_steps each: advance_physics_to_time
 * (hybrid/coupled_forecast.py:123-161) for a batch of members, as 50-step
 * graphs until all members are done.  dt_logs: NULL, or per member a device
 * float64 [max_steps] log of its dts (as swe_advance_to).  SWE_ERR_MAX_STEPS
 * when a member did not reach the target (its result says which).
 * Both advances return with their results final and the members' new states
 * queued on `stream` (stream-ordered, like every call that takes a stream). */
int swe_ensemble_advance_to(swe_ensemble_t e, float *const *h, float *const *hu, float *const *hv,
                            const int64_t *pitch, const double *start_s, double target_s, int32_t max_steps,
                            double *const *dt_logs, swe_run_result *results, void *stream);
/* Borrowed handle of member m (owned by the ensemble: do not destroy it), for
 * the per-domain calls (features, correction, step, cfl). */
int swe_ensemble_member(swe_ensemble_t e, int32_t m, swe_domain_t *out);
int swe_ensemble_set_timing(swe_ensemble_t e, int32_t enable);
int swe_ensemble_last_step_time(swe_ensemble_t e, double *ms, int64_t *steps);
int64_t swe_ensemble_last_launch_count(swe_ensemble_t e);

/* The coupling calls of every member in one call (the hybrid ensemble rollout's
 * per-interval features and corrections; each is swe_network_features /
 * swe_apply_correction on member m, queued in member order on `stream`).
 * Arrays hold one entry per member.  Features: mean/stddev are n_members rows
 * of 5 floats (the first 3 used by REFERENCE6); terrain/roughness NULL or
 * per-member device pointers (entries may be NULL); member m's features start
 * at out + m * out_member_stride elements.  Correction: member m's residual
 * starts at residual + m * res_stride_member elements; clip_limits NULL or
 * n_members rows of res_channels floats. */
int swe_ensemble_network_features(swe_ensemble_t e, float *const *h, float *const *hu, float *const *hv,
                                  const int64_t *pitch, int32_t layout, const float *mean, const float *stddev,
                                  const float *rain_features, const float *const *terrain,
                                  const float *const *roughness, void *out, int64_t out_member_stride,
                                  int32_t out_bf16, void *stream);
int swe_ensemble_apply_correction(swe_ensemble_t e, float *const *h, float *const *hu, float *const *hv,
                                  const int64_t *pitch, const void *residual, int32_t residual_bf16,
                                  int64_t res_stride_member, int64_t res_stride_row, int64_t res_stride_col,
                                  int64_t res_stride_channel, int32_t res_channels, const float *clip_limits,
                                  double relaxation, float *const *h_out, float *const *hu_out,
                                  float *const *hv_out, const int64_t *out_pitch, void *stream);

/* ---- Row strips: one domain split across GPUs ----------------------------
 * (No counterpart in the reference, which runs one domain on one device; the
 * strip step is the reference step, finite_volume_step, over the strip's rows.)
 * A strip owns global rows [row_begin, row_end) and also holds the row below
 * and the row above when they exist (halo rows: read as neighbours, never
 * updated), so its local planes have row_end - row_begin + (number of halo
 * rows) rows, local row 0 being global row max(row_begin - 1, 0).  Every step
 * of the whole domain: the step kernel over the owned rows, the CFL maximum
 * over all strips, the same dt planned on every strip, and the exchange of the
 * new boundary rows.  The result matches one domain stepped whole, bit for bit. */
typedef struct swe_comm *swe_comm_t;
#define SWE_COMM_ID_BYTES 128

/* Create a strip of the domain `global` describes (its fields on the host or the
 * device, as for swe_domain_create). */
int swe_strip_create(const swe_domain_desc *global, int32_t row_begin, int32_t row_end, swe_domain_t *out);
/* The strip's local row count and its owned local rows [upd_lo, upd_hi). */
int swe_strip_layout(swe_domain_t d, int32_t *local_rows, int32_t *upd_lo, int32_t *upd_hi);

/* n strips of one domain, bottom to top, all on the current device (one
 * process): n_steps steps from t0; (h, hu, hv)[i] are strip i's local planes,
 * updated in place (halo rows included).  The maximum over strips is a kernel and
 * the exchange device-to-device copies. */
int swe_strips_advance(const swe_domain_t *strips, int32_t n, float *const *h, float *const *hu,
                       float *const *hv, const int64_t *pitch, int32_t n_steps, double t0,
                       swe_run_result *results, void *stream);

/* One strip per process and GPU over NCCL (opened at run time, libnccl.so.2):
 * the maximum is an all-reduce and the exchange point-to-point sends between
 * neighbour ranks (-1 where the strip has no halo row on that side).  Every rank
 * must call it with the same n_steps and t0.  swe_comm_unique_id writes
 * SWE_COMM_ID_BYTES bytes on one rank; pass them to swe_comm_create on all. */
int swe_comm_unique_id(void *id_out);
int swe_comm_create(const void *id, int32_t world, int32_t rank, swe_comm_t *out);
int swe_comm_destroy(swe_comm_t c);
int swe_strip_advance_nccl(swe_domain_t d, swe_comm_t comm, int32_t rank_below, int32_t rank_above, float *h,
                           float *hu, float *hv, int64_t pitch, int32_t n_steps, double t0,
                           swe_run_result *result, void *stream);

/* ---- Device generators of the synthetic inputs ------------------------------
 * The reference conditions its terrain on the host from GIS inputs
 * (src/hybrid_flood/dem/synthetic_terrain.py:114 generate_base_terrain,
 * src/hybrid_flood/dem/urban_conditioning.py:128 condition_urban_terrain); the
 * measurement workloads are seeded synthetic fields of the same kind, built
 * here directly in device memory.  Random draws come from a counter-based
 * generator (Philox-4x32-10), so a field depends only on its seed and sizes.
 * Outputs are caller-owned DEVICE buffers; the calls allocate their own
 * scratch and synchronise the stream before returning. */
typedef struct {
    int32_t rows, cols;
    double dx;                 /* cell size (m) */
    double slope;              /* plane falling toward +x: slope * (cols*dx - x), x at cell centres */
    double coverage;           /* block fraction to reach (0.30) */
    int32_t min_side, max_side;/* block side range in cells (5, 20) */
    double block_raise_m;      /* +10 m on blocks */
    double street_offset_m;    /* -0.2 m on streets */
    double n_block, n_street;  /* Manning n on blocks / streets (0.05, 0.015) */
    double n_scale;            /* multiplies both */
    uint64_t seed;
    int32_t n_rects;           /* > 0: use these rectangles in order instead of drawing them */
    const int32_t *rects;      /* HOST int32[n_rects][4]: row0, col0, height, width */
} swe_urban_desc;

/* Urban DEM: rectangles are added in order until the covered cells reach
 * coverage * rows * cols (a cell covered by several counts once); bed =
 * float32(plane + raise on blocks, + street offset elsewhere) and manning_n =
 * float32(n * n_scale), both formed in float64.  block_mask (uint8, may be
 * NULL) receives 1 on blocks; *blocks_used (may be NULL) the rectangles used. */
int swe_generate_urban(const swe_urban_desc *q, float *bed, float *manning_n, uint8_t *block_mask,
                       int32_t *blocks_used, void *stream);

/* Hyetograph of n values step_s apart: times[i] = i*step_s and rates[i] =
 * Gamma(shape_k, scale) * to_m_s (e.g. scale in mm/h, to_m_s = 1e-3/3600),
 * Gamma variates by Marsaglia and Tsang's method, rounded to float32. */
int swe_generate_gamma_hyetograph(int32_t n, double step_s, double shape_k, double scale, double to_m_s,
                                  uint64_t seed, float *times, float *rates, void *stream);

/* Smoothed log-normal field (a Manning n field): standard normal noise per
 * cell (or the caller's DEVICE float64 noise[rows*cols] when non-NULL),
 * smoothed by a reflect-padded separable Gaussian smooth_cells wide (sigma =
 * smooth_cells/6, taps normalised), divided by its standard deviation, and
 * out = float32(median * exp(sigma_log * x)). */
int swe_generate_lognormal_field(int32_t rows, int32_t cols, double median, double sigma_log, int32_t smooth_cells,
                                 uint64_t seed, const double *noise, float *out, void *stream);

/* Largest cell count swe_max_inverse_dt_noalloc accepts (a 4096 x 4096 grid). */
#define SWE_NOALLOC_MAX_CELLS 16777216

/* swe_max_inverse_dt without any memory allocation.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc when they need
 * a CFL step -- code running under a framework's caching allocator, where a
 * direct cudaMalloc can fail although the framework's pool has room, and
 * time-stepping loops that forbid allocation once running.  It needs no
 * domain: the caller passes the state, the uint8 domain mask (rows*cols,
 * contiguous) and the controls, and a DEVICE float that receives the maximum.
 * Its scratch (32 KiB of per-CTA maxima plus a counter) is one fixed device
 * array inside the library, held on every GPU that loads the library until the
 * process exits, so grids above SWE_NOALLOC_MAX_CELLS cells are rejected with
 * SWE_ERR_INVALID.  The first call on each device looks up that array's
 * address; make that first call before any stream capture.  All calls share
 * the array: calls that can overlap on the GPU (different streams, or
 * different host threads) race and must be serialised by the caller.
 * Arithmetic is the exact (reference-rounded) one. */
int swe_max_inverse_dt_noalloc(const float *h, const float *hu, const float *hv, int64_t pitch,
                               const uint8_t *domain_mask, int32_t rows, int32_t cols,
                               double gravity, double dry_tolerance, double dx, double dy,
                               float *max_inverse_dt_out, void *stream);

/* Copy the message of the last error on this thread into buf (NUL-terminated);
 * returns the full message length. */
int swe_last_error(char *buf, size_t n);

/* Library version string, e.g. "swe_b200 0.1.0 sm_100a". */
const char *swe_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SWE_B200_H */
