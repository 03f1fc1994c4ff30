/*
 * svpf.h -- C ABI of the B200 SVPF step engine (libsvpf_b200.so).
 *
 * Drop-in for the reference's include/svpf.cuh: same type names, same field
 * names for every SVPFState field a caller configures, same entry points and
 * argument meaning.  Field offsets differ: callers recompile against this
 * header.  Plain C types only (cudaStream_t is an opaque pointer).
 *
 * Every tick of a filter runs as ONE kernel launch: predict, EKF guide,
 * bandwidth, the annealed Newton-Stein loop with KSD, rejuvenation and the
 * output moments, with particles resident in shared memory.  The batch API
 * runs many independent filters (own N, own theta) in one persistent launch
 * per tick.
 */
#ifndef SVPF_B200_H
#define SVPF_B200_H

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- constants (include/svpf.cuh:47-64) ---------------------------------- */
#define SVPF_DEFAULT_PARTICLES     512
#define SVPF_DEFAULT_STEIN_STEPS   5
#define SVPF_DEFAULT_NU            5.0f
#define SVPF_STEIN_STEP_SIZE       0.1f
#define SVPF_H_MIN                 -15.0f
#define SVPF_H_MAX                 5.0f
#define SVPF_SMOOTH_MAX_LAG        8
#define SVPF_STEIN_SIGN_LEGACY     0
#define SVPF_STEIN_SIGN_PAPER      1
#ifndef SVPF_STEIN_SIGN_DEFAULT
#define SVPF_STEIN_SIGN_DEFAULT    SVPF_STEIN_SIGN_LEGACY
#endif

/* Engine limits. */
#define SVPF_MAX_PARTICLES         8192   /* per filter */
#define SVPF_MAX_ANNEAL_STEPS      16
#define SVPF_MAX_STEIN_STEPS       256    /* Stein iterations of one tick, all stages */

/* Error codes returned by svpf_last_error() and the batch API. */
#define SVPF_OK                    0
#define SVPF_ERR_INVALID_ARG       1
#define SVPF_ERR_CUDA              2
#define SVPF_ERR_NOT_INITIALIZED   3
#define SVPF_ERR_TAPE_SHORT        4   /* noise tape has fewer slots than the tick draws */
#define SVPF_ERR_NONFINITE         5   /* NaN/Inf y_t: the tick is refused (the filter's state is
                                           left exactly as it was; loglik, vol and h_mean NaN,
                                           steps_used 0); NaN/Inf y_prev: read
                                           as 0 and the tick runs; or NaN/Inf in the outputs */
#define SVPF_ERR_UNSUPPORTED       6
#define SVPF_ERR_BUDGET            7   /* request loop: the instrument's state does not fit the HBM budget */

/* ---- model parameters (include/svpf.cuh:257-262) ------------------------- */
typedef struct {
    float rho;
    float sigma_z;
    float mu;
    float gamma;
} SVPFParams;

/* ---- step result (include/svpf.cuh:552-558) ------------------------------ */
typedef struct {
    float log_lik_increment;
    float vol_mean;
    float vol_std;
    float h_mean;
    float mu_estimate;
} SVPFResult;

/* ---- per-filter configuration ---------------------------------------------
 * Field names and meaning follow the SVPFState configuration fields of the
 * reference (include/svpf.cuh:337-545).  Used directly by the batch API; the
 * single-filter API keeps the same fields inside SVPFState.                */
#define SVPF_CONFIG_FIELDS(X_INT, X_FLOAT)                                     \
    X_INT(n_stein_steps) X_FLOAT(nu) X_FLOAT(student_t_implied_offset)        \
    X_FLOAT(lik_offset) X_INT(use_exact_gradient) X_INT(use_svld)             \
    X_INT(use_annealing) X_INT(use_adaptive_beta) X_INT(n_anneal_steps)       \
    X_FLOAT(temperature) X_FLOAT(rmsprop_rho) X_FLOAT(rmsprop_eps)            \
    X_INT(use_mim) X_FLOAT(mim_jump_prob) X_FLOAT(mim_jump_scale)             \
    X_INT(use_local_params) X_FLOAT(delta_rho) X_FLOAT(delta_sigma)           \
    X_INT(use_asymmetric_rho) X_FLOAT(rho_up) X_FLOAT(rho_down)               \
    X_INT(use_newton) X_INT(use_full_newton) X_INT(use_guided)                \
    X_FLOAT(guided_alpha_base) X_FLOAT(guided_alpha_shock)                    \
    X_FLOAT(guided_innovation_threshold) X_INT(use_rejuvenation)              \
    X_FLOAT(rejuv_ksd_threshold) X_FLOAT(rejuv_prob) X_FLOAT(rejuv_blend)     \
    X_INT(use_guide) X_INT(use_guide_preserving) X_FLOAT(guide_strength)      \
    X_INT(use_adaptive_guide) X_FLOAT(guide_strength_base)                    \
    X_FLOAT(guide_strength_max) X_FLOAT(guide_innovation_threshold)           \
    X_INT(use_adaptive_mu) X_FLOAT(mu_process_var) X_FLOAT(mu_obs_var_scale)  \
    X_FLOAT(mu_min) X_FLOAT(mu_max) X_INT(use_adaptive_sigma)                 \
    X_FLOAT(sigma_boost_threshold) X_FLOAT(sigma_boost_max)                   \
    X_INT(stein_repulsive_sign) X_INT(use_fan_mode) X_INT(stein_min_steps)    \
    X_INT(stein_max_steps) X_FLOAT(ksd_improvement_threshold)                 \
    X_INT(use_student_t_state) X_FLOAT(nu_state) X_INT(use_smoothing)         \
    X_INT(smooth_lag) X_INT(smooth_output_lag) X_INT(use_heun)                \
    X_INT(use_two_factor) X_FLOAT(rho_fast) X_FLOAT(sigma_fast)               \
    X_FLOAT(rho_slow) X_FLOAT(sigma_slow) X_FLOAT(bw_floor_fast)              \
    X_FLOAT(bw_floor_slow)

#define SVPF_DECL_INT_(f) int f;
#define SVPF_DECL_FLOAT_(f) float f;
typedef struct {
    SVPF_CONFIG_FIELDS(SVPF_DECL_INT_, SVPF_DECL_FLOAT_)
} svpf_config_t;

/* Per-filter control record carried from tick to tick (device resident in the
 * batch engine; mirrored into SVPFState fields for the single-filter API). */
typedef struct {
    double guide_mean;        /* EKF posterior mean (FP64 recursion) */
    double guide_var;         /* EKF posterior variance (FP64 recursion) */
    double guide_K;
    double loglik_sum;        /* FP64 sum of per-tick log-likelihoods */
    double guide_mean_fast;   /* two-factor EKF (innovation split), FP64 */
    double guide_mean_slow;
    double guide_var_fast;
    double guide_var_slow;
    int    timestep;
    int    guide_initialized;
    int    stein_steps_used;
    int    smooth_head;
    int    guide_2f_initialized;
    float  ksd_prev;          /* KSD of the previous tick: budget, beta, rejuvenation */
    float  ksd_last;          /* last KSD computed */
    float  vol_prev;
    float  h_mean_prev;
    float  bw;
    float  bw_sq;
    float  return_ema;
    float  return_var;
    float  sigma_z_effective;
    float  mu_state;
    float  mu_var;
    float  y_prev;
    float  h_fast_mean;       /* two-factor: factor means of the previous tick */
    float  h_slow_mean;
    float  smooth_h_mean[SVPF_SMOOTH_MAX_LAG];
    float  smooth_h_var[SVPF_SMOOTH_MAX_LAG];
    float  smooth_y[SVPF_SMOOTH_MAX_LAG];
    int    status;            /* SVPF_OK or an SVPF_ERR_* code of the last tick */
    int    reserved;
} svpf_ctl_t;

/* Per-tick outputs of one filter. */
typedef struct {
    float loglik;
    float vol;
    float h_mean;             /* smoothed when use_smoothing */
    float h_mean_raw;
    float bw;
    float ksd;
    int   steps_used;
    int   rejuv_fired;
} svpf_out_t;

/* ---- single-filter state (include/svpf.cuh:290-547) ---------------------- */
typedef struct {
    /* particle arrays (device, [n_particles]) */
    float* h;
    float* h_prev;
    float* h_pred;            /* kept for source compatibility; not written */
    float* grad_log_p;        /* kept for source compatibility; not written */
    float* log_weights;       /* log importance weights of the last gradient pass */
    float* d_grad_v;          /* RMSProp second moment */
    void*  rng_states;        /* unused: the engine's RNG is counter based */

    int    n_particles;
    int    n_stein_steps;
    float  nu;
    float  student_t_const;
    float  student_t_implied_offset;
    int    timestep;
    float  y_prev;
    cudaStream_t stream;

    float lik_offset;
    int   use_exact_gradient;
    int   use_svld;
    int   use_annealing;
    int   use_adaptive_beta;
    int   n_anneal_steps;
    float temperature;
    float rmsprop_rho;
    float rmsprop_eps;
    int   use_mim;
    float mim_jump_prob;
    float mim_jump_scale;
    int   use_local_params;
    float delta_rho;
    float delta_sigma;
    int   use_asymmetric_rho;
    float rho_up;
    float rho_down;
    int   use_newton;
    int   use_full_newton;
    int   use_guided;
    float guided_alpha_base;
    float guided_alpha_shock;
    float guided_innovation_threshold;
    int   use_rejuvenation;
    float rejuv_ksd_threshold;
    float rejuv_prob;
    float rejuv_blend;
    int   use_guide;
    int   use_guide_preserving;
    float guide_strength;
    float guide_mean;
    float guide_var;
    float guide_K;
    int   guide_initialized;
    int   use_adaptive_guide;
    float guide_strength_base;
    float guide_strength_max;
    float guide_innovation_threshold;
    float vol_prev;
    int   use_adaptive_mu;
    float mu_state;
    float mu_var;
    float mu_process_var;
    float mu_obs_var_scale;
    float mu_min;
    float mu_max;
    int   use_adaptive_sigma;
    float sigma_boost_threshold;
    float sigma_boost_max;
    float sigma_z_effective;
    int   stein_repulsive_sign;
    int   use_fan_mode;
    int   stein_min_steps;
    int   stein_max_steps;
    float ksd_improvement_threshold;
    float ksd_prev;
    int   stein_steps_used;
    int   use_student_t_state;
    float nu_state;
    int   use_smoothing;
    int   smooth_lag;
    int   smooth_output_lag;
    int   smooth_head;
    float smooth_h_mean[SVPF_SMOOTH_MAX_LAG];
    float smooth_h_var[SVPF_SMOOTH_MAX_LAG];
    float smooth_y[SVPF_SMOOTH_MAX_LAG];
    int   use_persistent_kernel;   /* accepted, no effect: every tick is one launch */
    int   persistent_kernel_supported;
    int   use_heun;

    /* two-factor volatility h = mu + h_fast + h_slow (include/svpf.cuh:533-544) */
    int   use_two_factor;
    float rho_fast;
    float sigma_fast;
    float rho_slow;
    float sigma_slow;
    float bw_floor_fast;
    float bw_floor_slow;
    float guide_mean_fast;
    float guide_mean_slow;
    float guide_var_fast;
    float guide_var_slow;
    int   guide_2f_initialized;

    void* impl;                    /* engine-private state */
} SVPFState;

/* ---- core API (include/svpf.cuh:573-603, src/svpf_optimized_graph.cu) ---- */

/* svpf_create (include/svpf.cuh:573): allocates the filter; NULL on failure
 * (n_particles outside [1, SVPF_MAX_PARTICLES], no device, out of memory). */
SVPFState* svpf_create(int n_particles, int n_stein_steps, float nu, cudaStream_t stream);

/* svpf_destroy (include/svpf.cuh:578). NULL is a no-op. */
void svpf_destroy(SVPFState* state);

/* svpf_initialize (include/svpf.cuh:587): particles from the stationary law;
 * synchronous.  The seed keys the engine's counter-based Philox generator. */
void svpf_initialize(SVPFState* state, const SVPFParams* params, unsigned long long seed);

/* svpf_step (include/svpf.cuh:597): one tick with y_prev = state->y_prev. */
void svpf_step(SVPFState* state, float y_t, const SVPFParams* params, SVPFResult* result);

/* svpf_step_seeded (include/svpf.cuh:602-603): as svpf_step, but this tick's
 * noise is keyed by rng_seed (the reference ignores the seed; here the same
 * seed and state reproduce the same tick). */
void svpf_step_seeded(SVPFState* state, float y_t, const SVPFParams* params,
                      unsigned long long rng_seed, SVPFResult* result);

/* svpf_step_adaptive (include/svpf.cuh:768-776): same as svpf_step_graph. */
void svpf_step_adaptive(SVPFState* state, float y_t, float y_prev, const SVPFParams* params,
                        float* h_loglik_out, float* h_vol_out, float* h_mean_out);

/* svpf_step_optimized (include/svpf.cuh:726-733): declared by the reference but
 * defined nowhere in its sources; here the production tick without the h_mean
 * output (svpf_step_graph with h_mean_out = NULL). */
void svpf_step_optimized(SVPFState* state, float y_t, float y_prev, const SVPFParams* params,
                         float* h_loglik_out, float* h_vol_out);

/* svpf_step_graph (include/svpf.cuh:843-851): the production tick.  Blocking;
 * NULL output pointers are allowed.  One kernel launch per call. */
void svpf_step_graph(SVPFState* state, float y_t, float y_prev, const SVPFParams* params,
                     float* h_loglik_out, float* h_vol_out, float* h_mean_out);

/* svpf_run_sequence[_device] (include/svpf.cuh:689-708). */
void svpf_run_sequence(SVPFState* state, const float* h_observations, int T,
                       const SVPFParams* params, float* h_loglik_out, float* h_vol_out);
void svpf_run_sequence_device(SVPFState* state, const float* d_observations, int T,
                              const SVPFParams* params, float* d_loglik_out, float* d_vol_out);

/* diagnostics (include/svpf.cuh:795-811, src/svpf_optimized_graph.cu:1490) */
void  svpf_get_particles(const SVPFState* state, float* h_out);
void  svpf_get_stats(const SVPFState* state, float* h_mean, float* h_std);
float svpf_get_ess(const SVPFState* state);
void  svpf_get_ksd_stats(const SVPFState* state, float* ksd_out, int* steps_used_out);

/* graph API (include/svpf.cuh:856-869).  A tick is already one launch; these
 * report/drop the cached launch configuration. */
bool svpf_graph_is_captured(SVPFState* state);
void svpf_graph_invalidate(SVPFState* state);
void svpf_optimized_cleanup_state(SVPFState* state);

/* sign / Fan mode setters (include/svpf.cuh:626-673) */
static inline void svpf_set_stein_sign_mode(SVPFState* state, int mode) {
    state->stein_repulsive_sign = (mode == SVPF_STEIN_SIGN_PAPER) ? 1 : 0;
}
static inline int svpf_get_stein_sign_mode(const SVPFState* state) {
    return state->stein_repulsive_sign;
}
static inline void svpf_set_fan_mode(SVPFState* state, int enable) {
    state->use_fan_mode = enable ? 1 : 0;
    if (enable) state->stein_repulsive_sign = SVPF_STEIN_SIGN_PAPER;
}
static inline int svpf_get_fan_mode(const SVPFState* state) { return state->use_fan_mode; }

/* ---- additions (no reference counterpart) -------------------------------- */

/* Error of the last call on this state (the reference's step returns void). */
int svpf_last_error(const SVPFState* state);

/* Fill cfg with the svpf_create defaults for (n_stein_steps, nu), including
 * the create-time Student-t implied offset.  Needs no device. */
void svpf_config_init(svpf_config_t* cfg, int n_stein_steps, float nu);

/* Copy the configuration fields of the state into a svpf_config_t and back. */
void svpf_get_config(const SVPFState* state, svpf_config_t* cfg);
void svpf_set_config(SVPFState* state, const svpf_config_t* cfg);

/* Full state snapshot / restore: control record plus host arrays [n].  Used for
 * checkpointing and for per-tick parity checks with state re-sync. */
int svpf_get_state(const SVPFState* state, svpf_ctl_t* ctl, float* h, float* h_prev,
                   float* v, float* log_w);
int svpf_set_state(SVPFState* state, const svpf_ctl_t* ctl, const float* h,
                   const float* h_prev, const float* v, const float* log_w);

/* Two-factor particle arrays [n] each (any pointer may be NULL). */
int svpf_get_state_2f(const SVPFState* state, float* h_fast, float* h_slow, float* h_fast_prev,
                      float* h_slow_prev, float* v_fast, float* v_slow);
int svpf_set_state_2f(SVPFState* state, const float* h_fast, const float* h_slow,
                      const float* h_fast_prev, const float* h_slow_prev, const float* v_fast,
                      const float* v_slow);

/* Test hook: drive the next ticks' noise from a host tape instead of Philox.
 * normals[k*n + i] is the k-th normal of particle i within a tick; uniforms
 * likewise.  Pass NULL to return to Philox.  The tape is copied. */
int svpf_set_noise_tape(SVPFState* state, const float* normals, int n_normal_slots,
                        const float* uniforms, int n_uniform_slots);

/* Last tick's full outputs. */
int svpf_get_last_output(const SVPFState* state, svpf_out_t* out);

/* Cluster size used by the single-filter kernel for this state (0 = auto). */
int svpf_set_cluster_size(SVPFState* state, int cluster_ctas);

/* ---- batch API: many independent filters, one persistent launch per tick -- */
typedef struct svpf_batch svpf_batch_t;

/* Create a batch of n_filters filters; filter f has ns[f] particles,
 * configuration cfgs[f] and parameters params[f].  stream may be NULL. */
svpf_batch_t* svpf_batch_create(int n_filters, const int* ns, const svpf_config_t* cfgs,
                                const SVPFParams* params, cudaStream_t stream);
void svpf_batch_destroy(svpf_batch_t* b);

/* Stationary initialisation of every filter; filter f is keyed by (seed, f). */
int svpf_batch_initialize(svpf_batch_t* b, unsigned long long seed);

/* One tick of every filter from HOST observations y_t[f], y_prev[f]; outputs
 * (may be NULL) land in host arrays [n_filters].  Copies in and out are part
 * of the call.  Blocking. */
int svpf_batch_step(svpf_batch_t* b, const float* y_t, const float* y_prev,
                    float* loglik, float* vol, float* h_mean);

/* One tick from DEVICE observations (d_y_t/d_y_prev [n_filters]); outputs go
 * to device arrays (may be NULL).  Asynchronous on the batch stream. */
int svpf_batch_step_device(svpf_batch_t* b, const float* d_y_t, const float* d_y_prev,
                           svpf_out_t* d_out);

/* Capture one device tick in a CUDA graph and replay it: the observations are
 * read from d_y_t/d_y_prev (fixed device buffers the caller refills). */
int svpf_batch_graph_launch(svpf_batch_t* b, const float* d_y_t, const float* d_y_prev,
                            svpf_out_t* d_out);

int svpf_batch_sync(svpf_batch_t* b);
int svpf_batch_n_filters(const svpf_batch_t* b);
int svpf_batch_kernel_launches(const svpf_batch_t* b);  /* launches issued so far */
int svpf_batch_get_ctl(const svpf_batch_t* b, svpf_ctl_t* ctl_host);          /* [n_filters] */
/* h_out receives n values, or 2n (fast then slow) for a two-factor filter. */
int svpf_batch_get_particles(const svpf_batch_t* b, int filter, float* h_out);
/* Model parameters of filter f.  Setting them is stream ordered (ticks already
 * enqueued keep the old ones) and waits for the batch's stream; the next
 * svpf_batch_initialize draws the stationary law from them. */
int svpf_batch_get_params(const svpf_batch_t* b, int filter, SVPFParams* params);
int svpf_batch_set_params(svpf_batch_t* b, int filter, const SVPFParams* params);
/* State of filter f (host arrays; any pointer may be NULL): control record,
 * h / h_prev / RMSProp v of n values (2n, fast then slow, for a two-factor
 * filter) and the n log-weights.  Both wait for the batch's stream.  Used for
 * checkpoints and for per-tick parity checks with state re-sync. */
int svpf_batch_get_state(const svpf_batch_t* b, int filter, svpf_ctl_t* ctl, float* h, float* h_prev, float* v,
                         float* log_w);
int svpf_batch_set_state(svpf_batch_t* b, int filter, const svpf_ctl_t* ctl, const float* h, const float* h_prev,
                         const float* v, const float* log_w);
int svpf_batch_set_noise_tape(svpf_batch_t* b, const float* normals, int n_normal_slots,
                              const float* uniforms, int n_uniform_slots);   /* same tape for all, [k][n_max] */
/* Tile shape (rows per thread R, column split S) used for filters of size n;
 * -1 when no choice was made. */
int svpf_batch_tile_of(const svpf_batch_t* b, int n, int* rows_per_thread, int* col_split);
/* The tile shape filter f runs with, and -- to test or pin a shape -- force
 * one: (rows_per_thread, col_split) must be a compiled batch tile, (1,4)
 * (1,2) (1,1) (2,1) (4,1); SVPF_ERR_INVALID_ARG otherwise.  Forcing a tile
 * waits for the batch's stream and drops its captured graph. */
int svpf_batch_tile_of_filter(const svpf_batch_t* b, int filter, int* rows_per_thread, int* col_split);
int svpf_batch_set_tile(svpf_batch_t* b, int filter, int rows_per_thread, int col_split);

/* One tick of a batch whose buffers the caller owns, with no allocation of any
 * kind.  No counterpart in the reference: it serves callers that cannot call
 * cudaMalloc (a host application that owns all device memory in a fixed arena,
 * a plugin inside another framework's memory manager, a latency-critical loop
 * that must not take the device synchronisation an allocation may cause).
 * Every buffer is a device pointer the caller allocated: particle counts d_n,
 * packed-array offsets d_off, per-filter configuration, parameters and control
 * records (updated in place), the packed particle arrays (updated in place),
 * this tick's observations and, optionally, the outputs.
 * Single-factor filters only.  Each filter must have 1 <= d_n[f] <= n_max, an
 * offset d_off[f] >= 0 that is a multiple of 16 floats, use_heun only when
 * any_heun is 1, and loop counts within SVPF_MAX_STEIN_STEPS; its n floats at
 * d_off[f] must lie inside each packed array (that size is not passed and is
 * not checked).  A filter that breaks one of the checked rules is left out of
 * the tick on the device, before anything reads its particles: its control
 * record's status becomes SVPF_ERR_INVALID_ARG (SVPF_ERR_UNSUPPORTED for a
 * two-factor filter) and its arrays and outputs are not written; the other
 * filters tick as usual.
 * The kernel's scratch (work counter, work order, tile per filter) is a fixed
 * array inside the library, resident on every GPU that loads it until the
 * process exits; at most SVPF_NOALLOC_MAX_FILTERS filters per call, larger
 * batches are rejected with SVPF_ERR_INVALID_ARG.  The first call on a device
 * looks up that array's device address (make it before any stream capture).
 * All calls share the one array and each call rewrites what it uses; calls
 * that overlap on the GPU race, so issue them in one stream or order them.
 * Asynchronous on `stream`. */
#define SVPF_NOALLOC_MAX_FILTERS   16384
int svpf_batch_tick_noalloc(int n_filters, const int* d_n, const long long* d_off,
                            const svpf_config_t* d_cfg, const SVPFParams* d_params,
                            svpf_ctl_t* d_ctl, float* d_h, float* d_h_prev, float* d_v,
                            float* d_log_w, const float* d_y_t, const float* d_y_prev,
                            svpf_out_t* d_out, int n_max, int any_heun,
                            unsigned long long seed, cudaStream_t stream);
int svpf_noalloc_max_filters(void);

/* Autotuner: time each compiled tile shape on a synthetic filter of each
 * particle count in ns[] and keep the fastest per size for this process. */
int svpf_autotune(const int* ns, int count, int ticks);
int svpf_tile_choice(int n, int* rows_per_thread, int* col_split);

/* Library facts. */
const char* svpf_build_info(void);


/* ---- gradients of the log-likelihood (adjoint) ---------------------------
 * d(sum_t w_t loglik_t)/d(mu, rho, sigma_z, nu) of every filter of a batch
 * over a run of T ticks that starts with svpf_initialize from theta, under
 * common random numbers (the engine's counter-based noise keyed by seed and
 * filter index).  Reverse mode: the forward keeps a checkpoint every
 * `checkpoint_every` ticks, the backward recomputes one segment at a time.
 * The configuration must be inside the differentiable set
 * (svpf_grad_supported): single factor, plain or MIM predict with the
 * model's rho (use_asymmetric_rho = use_local_params = use_guided = 0), EKF
 * guide without adaptive strength, Gaussian prior, vanilla or full-Newton
 * transport, fixed beta schedule (no adaptive beta), no rejuvenation, no
 * adaptive mu / sigma, no Heun / fan mode. */
typedef struct svpf_grad svpf_grad_t;

int svpf_grad_supported(const svpf_config_t* cfg);
svpf_grad_t* svpf_grad_create(int n_filters, const int* n_particles, const svpf_config_t* cfgs,
                              int T_max, int checkpoint_every, cudaStream_t stream);
void svpf_grad_destroy(svpf_grad_t* g);
/* theta [F][4] = (mu, rho, sigma_z, nu); gamma [F] leverage or NULL; y [F][T].
 * Outputs (host, may be NULL): loglik [F][T] (FP32), loglik_sum [F] (FP64). */
int svpf_grad_forward(svpf_grad_t* g, const float* theta, const float* gamma, const float* y, int T,
                      unsigned long long seed, float* loglik, double* loglik_sum);
/* w [F][T]: weight of each tick's loglik (NULL = all ones); grad [F][4]. */
int svpf_grad_backward(svpf_grad_t* g, const float* w, double* grad);
/* Device-pointer variants, stream ordered, no host synchronisation; the
 * device arrays given to the forward must stay valid until the backward. */
int svpf_grad_forward_device(svpf_grad_t* g, const float* d_theta, const float* d_gamma,
                             const float* d_y, int T, unsigned long long seed, float* d_loglik);
int svpf_grad_backward_device(svpf_grad_t* g, const float* d_w, double* d_grad);
int svpf_grad_checkpoint_every(const svpf_grad_t* g);
/* Parameter domain: every theta component finite, nu > 0, sigma_z > 0,
 * |rho| < 1, leverage finite.  svpf_grad_forward checks the host theta and
 * returns SVPF_ERR_INVALID_ARG before any launch.  With device theta
 * (svpf_grad_forward_device, the torch path) a filter outside the domain is
 * left out on the device: its status becomes SVPF_ERR_INVALID_ARG, its
 * log-likelihoods and gradient NaN; the other filters are unaffected.
 * status [n_filters] (host): the status of each filter after the last
 * forward / backward (waits for the engine's stream). */
int svpf_grad_get_status(svpf_grad_t* g, int* status);
/* 1 if the backward records a whole checkpoint segment in one forward pass
 * (k tick records per CTA in device memory) instead of re-running each tick's
 * forward once more before its adjoint; chosen at create by free memory.
 * set: 1 forces segment records (SVPF_ERR_CUDA if they do not fit), 0 the
 * per-tick records.  Both give the same bits. */
int svpf_grad_segment_records(const svpf_grad_t* g);
int svpf_grad_set_segment_records(svpf_grad_t* g, int on);
/* 1 if the forward keeps every tick's record (T_max records per filter in
 * device memory) so that the backward recomputes nothing; chosen at create
 * when they take at most half of the free device memory.  Checkpoints are
 * still written.  set: 1 allocates them (SVPF_ERR_CUDA if they do not fit),
 * 0 frees them (the backward then recomputes from the checkpoints); either
 * way a new forward must run before the next backward.  All modes give the
 * same bits. */
int svpf_grad_run_records(const svpf_grad_t* g);
int svpf_grad_set_run_records(svpf_grad_t* g, int on);
/* Truncated backpropagation through time (the reference's torch model cuts
 * its particle path the same way, py-torch/diff_svpf_torch.py:177-179): for
 * t > 0 with t % every == 0, the state carried into tick t (particles,
 * RMSProp moments, EKF guide, bandwidth average, previous mean) is held
 * constant in theta, so each tick's log-likelihood is differentiated through
 * at most `every` ticks of the filter.  0 (default): the exact gradient of the
 * whole run.  The exact gradient can grow exponentially with the run's length
 * (narrow state noise makes the particle map expanding); a filter whose
 * gradient overflows gets SVPF_ERR_NONFINITE in svpf_grad_get_status.
 * Applies to the next backward. */
int svpf_grad_set_truncation(svpf_grad_t* g, int every);
int svpf_grad_truncation(const svpf_grad_t* g);
/* What the run's log-likelihood is made of (before the next forward):
 * SVPF_GRAD_TICK_LOGLIK (default): each tick's loglik as svpf_step_graph
 * reports it (log-mean-exp of the log-weights of the tick's last gradient
 * pass, after the Stein moves); SVPF_GRAD_PREDICTIVE: log p(y_t | y_1:t-1)
 * estimated at the predicted particles, before guide and Stein moves. */
#define SVPF_GRAD_TICK_LOGLIK 0
#define SVPF_GRAD_PREDICTIVE  1
int svpf_grad_set_objective(svpf_grad_t* g, int objective);

/* ---- request loop over instruments in a fixed HBM budget ------------------
 * The reference serves each instrument with its own svpf_step_graph call
 * (svpf_optimized_graph.cu:915-928 dispatching to :744-897 for two factors).
 * Here a fleet of instruments -- single- or two-factor, each with its own N,
 * configuration and parameters -- lives in one device pool allocated at
 * creation: `hbm_budget_bytes` covers the pool and the per-instrument records.
 * Admission places an instrument's particle state first-fit in the pool and
 * refuses it with SVPF_ERR_BUDGET when it does not fit; eviction frees it.
 * A call carries (instrument, y_t) requests; each instrument keeps its own
 * y_prev on the device.  Requests are served in rounds (the k-th request of
 * an instrument in round k, so its ticks keep their order), each round one
 * persistent launch per model pulling work largest cost first.  Tick noise is
 * keyed by (stream seed, slot, tick), initial draws by (admission seed, slot),
 * so slot f matches filter f of a batch with the same seeds.  Heun is not
 * supported here (SVPF_ERR_UNSUPPORTED). */
typedef struct svpf_stream svpf_stream_t;

svpf_stream_t* svpf_stream_create(int max_instruments, size_t hbm_budget_bytes, int n_max,
                                  cudaStream_t stream);
void svpf_stream_destroy(svpf_stream_t* s);
void svpf_stream_set_seed(svpf_stream_t* s, unsigned long long seed);
/* Returns the instrument's slot (>= 0) or -SVPF_ERR_* (-SVPF_ERR_BUDGET when
 * its state does not fit).  The instrument starts as after svpf_initialize. */
int svpf_stream_admit(svpf_stream_t* s, int n_particles, const svpf_config_t* cfg,
                      const SVPFParams* params, unsigned long long seed);
int svpf_stream_evict(svpf_stream_t* s, int slot);
size_t svpf_stream_bytes_in_use(const svpf_stream_t* s);
size_t svpf_stream_bytes_budget(const svpf_stream_t* s);
/* Serve `count` requests (host arrays); out[r] (may be NULL) gets request r's
 * outputs.  Blocking. */
int svpf_stream_process(svpf_stream_t* s, int count, const int* slots, const float* y, svpf_out_t* out);
/* One round from device arrays, stream ordered: d_slots[0, count1) are
 * single-factor instruments, d_slots[count1, count1 + count2) two-factor
 * ones, each instrument at most once; d_y and d_out are indexed alike. */
int svpf_stream_process_device(svpf_stream_t* s, int count1, int count2, const int* d_slots,
                               const float* d_y, svpf_out_t* d_out);
int svpf_stream_get_ctl(const svpf_stream_t* s, int slot, svpf_ctl_t* ctl);
/* n values, or 2n (fast then slow) for a two-factor instrument. */
int svpf_stream_get_particles(const svpf_stream_t* s, int slot, float* h_out);
long long svpf_stream_kernel_launches(const svpf_stream_t* s);

/* ---- svpf_fully_fused_step_v2 (include/svpf_fully_fused_v2.cuh:43-119) ------
 * The reference's second, single-kernel tick with its own semantics (Silverman
 * bandwidth, fixed beta ramp, EKF inside the kernel, adaptive guide strength),
 * same argument list.  One launch of a thread-block cluster; N up to 8064
 * (shared memory; svpf_fully_fused_v2_supported tells; the reference: 1024).
 * Where the reference takes
 * curandStatePhilox4_32_10_t*, this takes a device svpf_v2_rng_t record: the
 * engine's counter-based Philox keyed by (seed, filter) and counted by
 * (particle, draw, tick), tick advanced by every call, or -- a test hook -- a
 * device noise tape normals[k*n + i], uniforms[k*n + i]. */
typedef struct {
    unsigned long long seed;
    unsigned int tick;            /* advanced by one per call */
    unsigned int filter;
    int status;                   /* SVPF_OK or SVPF_ERR_TAPE_SHORT of the last call */
    int slots_n, slots_u;
    int reserved;
    const float* tape_normals;    /* device, or NULL for Philox */
    const float* tape_uniforms;
} svpf_v2_rng_t;

bool svpf_fully_fused_v2_supported(int n_particles);
cudaError_t svpf_fully_fused_step_v2(
    float* h, float* h_prev, float* grad_log_p, float* log_weights, float* d_grad_v, float* d_inv_hessian,
    svpf_v2_rng_t* rng, float y_t, float y_prev, float h_mean_prev, float vol_prev, float ksd_prev,
    float* d_h_mean, float* d_vol, float* d_loglik, float* d_bandwidth, float* d_ksd, float* d_guide_mean,
    float* d_guide_var, float rho, float sigma_z, float mu, float nu, float lik_offset, float student_t_const,
    float student_t_implied_offset, float gamma, float delta_rho, float delta_sigma, float mim_jump_prob,
    float mim_jump_scale, float guide_strength_base, float guide_strength_max, float guide_innovation_threshold,
    float guided_alpha_base, float guided_alpha_shock, float guided_innovation_thresh_predict, int use_guide,
    int use_guided_predict, int use_guide_preserving, int use_newton, int use_full_newton, int use_rejuvenation,
    float rejuv_ksd_threshold, float rejuv_prob, float rejuv_blend, int use_adaptive_mu, float* d_mu_state,
    float mu_ema_alpha, int use_adaptive_sigma, float sigma_boost_threshold, float sigma_boost_max,
    float step_size, float temperature, float rmsprop_rho, float rmsprop_eps, int n_stein_steps,
    int n_anneal_steps, int stein_sign_mode, int n, int timestep, cudaStream_t stream);
/* Device record helpers (the record may also be filled by the caller). */
svpf_v2_rng_t* svpf_fully_fused_v2_rng_create(unsigned long long seed, unsigned int filter);
void svpf_fully_fused_v2_rng_destroy(svpf_v2_rng_t* rng);
int svpf_fully_fused_v2_rng_get(const svpf_v2_rng_t* rng, svpf_v2_rng_t* host);
int svpf_fully_fused_v2_rng_set(svpf_v2_rng_t* rng, const svpf_v2_rng_t* host);

/* ---- multiscale composition on the batch engine --------------------------
 * The reference's two-scale filter (include/svpf_multiscale.cuh: a REACTIVE
 * scout and an INERTIAL production filter per instrument, combined per tick)
 * for many instruments at once: the 2F filters of F instruments form one batch
 * stepped by one launch per tick (the reference steps two svpf_step_adaptive
 * calls per instrument).  Configuration, per-scale knobs, output fields and
 * their combination follow ms_svpf_default_config / ms_svpf_create /
 * ms_svpf_step (:145-536); field names are the reference's. */
typedef struct {
    int   n_particles_reactive, n_particles_inertial;
    int   n_stein_reactive, n_stein_inertial;
    float surprise_mild_threshold, surprise_high_threshold;
    float boost_mild_factor, boost_high_factor;
    float weight_reactive, weight_inertial;
} svpf_ms_config_t;

typedef struct {
    float vol_reactive, vol_inertial, h_reactive, h_inertial, loglik_reactive, loglik_inertial;
    float vol_combined, h_combined, loglik_combined;
    float transient_magnitude, transient_ratio;
    float ksd_reactive, ksd_inertial;
    int   stein_steps_reactive, stein_steps_inertial;
    float surprise_reactive;
    int   cross_scale_boost;
    float mim_prob_inertial_used;
    int   is_transient, is_regime_shift, is_calm;
} svpf_ms_output_t;

typedef struct svpf_ms_batch svpf_ms_batch_t;

svpf_ms_config_t svpf_ms_default_config(void);
/* base_params[F]: each instrument's model (the INERTIAL scale ticks with it as
 * is, the REACTIVE scale with rho 0.92, sigma_z 0.18).  As ms_svpf_init does,
 * svpf_ms_batch_init draws the INERTIAL scale's initial state from its own
 * dynamics (rho 0.98, sigma_z 0.10) and the base mu and gamma. */
svpf_ms_batch_t* svpf_ms_batch_create(int n_instruments, const svpf_ms_config_t* cfg,
                                      const SVPFParams* base_params, cudaStream_t stream);
void svpf_ms_batch_destroy(svpf_ms_batch_t* b);
int svpf_ms_batch_init(svpf_ms_batch_t* b, float initial_vol, unsigned long long seed);
/* y[F]: this tick's observation of every instrument; out[F]. */
int svpf_ms_batch_step(svpf_ms_batch_t* b, const float* y, svpf_ms_output_t* out);
/* The per-filter outputs of the last svpf_batch_step of a batch ([n_filters]). */
int svpf_batch_last_outputs(const svpf_batch_t* b, svpf_out_t* out);
/* Configuration of filter f of a batch. */
int svpf_batch_get_config(const svpf_batch_t* b, int f, svpf_config_t* cfg);
/* The batch holding the 2F filters (REACTIVE i, INERTIAL F + i). */
svpf_batch_t* svpf_ms_batch_inner(svpf_ms_batch_t* b);

/* ---- the reference's differentiable torch model --------------------------- */
/* SVPFParamEstimator (py-torch/diff_svpf_torch.py:147-217), which the reference
 * differentiates with torch autograd, as a batched CUDA forward and adjoint:
 * F paths of N particles (N even), Gaussian AR(1) prior score per particle,
 * IMQ^(-1/2) kernel, n_stein fixed Stein steps of size stein_lr, antithetic
 * predict noise, the predictive log-likelihood before the transport, and the
 * particle path cut every truncate_every ticks (0: never).  The engine has no
 * reference C counterpart; it replaces the torch model's forward/backward.
 * stream NULL: the engine makes its own stream; cudaStreamLegacy names the
 * legacy default stream. */
typedef struct svpf_estimator svpf_estimator_t;
svpf_estimator_t* svpf_estimator_create(int n_paths, int n_particles, int n_stein_steps, float stein_lr,
                                        int T_max, int checkpoint_every, int truncate_every, cudaStream_t stream);
void svpf_estimator_destroy(svpf_estimator_t* e);
/* Floats of one path's noise tape: n initial normals, then n/2 per tick. */
long long svpf_estimator_tape_floats(int n_particles, int T);
/* theta[F][4] = (mu, rho, sigma_z, nu), y[F][T] (host).  tape[F][tape_floats]
 * (host) replays given normals (the torch model's torch.randn draws); NULL
 * draws them from the counter-based generator keyed by seed.  Outputs (host,
 * NULL allowed): loglik[F][T] predictive log-likelihoods, vol[F][T] volatility
 * estimates (mean e^{h/2} after the transport), loglik_sum[F] (FP64). */
int svpf_estimator_forward(svpf_estimator_t* e, const float* theta, const float* y, int T, unsigned long long seed,
                           const float* tape, float* loglik, float* vol, double* loglik_sum);
/* grad[F][4] = d(sum_t w_t loglik_t)/d theta for w[F][T] (host; NULL: all ones),
 * under the noise of the last forward.  The reference's loss
 * -mean(loglik[burn_in:]) is w_t = -1/(T - burn_in) for t >= burn_in. */
int svpf_estimator_backward(svpf_estimator_t* e, const float* w, double* grad);
/* Device-pointer variants (stream-ordered, no synchronisation): the arrays
 * must stay valid until the backward has run. */
int svpf_estimator_forward_device(svpf_estimator_t* e, const float* d_theta, const float* d_y, int T,
                                  unsigned long long seed, const float* d_tape, float* d_loglik, float* d_vol);
int svpf_estimator_backward_device(svpf_estimator_t* e, const float* d_w, double* d_grad);
/* theta outside the domain (any component non-finite, nu <= 0, sigma_z <= 0,
 * |rho| >= 1): svpf_estimator_forward returns SVPF_ERR_INVALID_ARG before any
 * launch; the device variants mark that path SVPF_ERR_INVALID_ARG, NaN its
 * outputs and gradient and leave the other paths unaffected.  status [F]. */
int svpf_estimator_get_status(svpf_estimator_t* e, int* status);

/* ---- test and measurement hooks ------------------------------------------
 * Not part of the filtering surface and without reference counterparts; the
 * parity tests and the benchmark use them. */

/* The engine's counter-based Philox4x32-10 on the device: out4[4k..4k+3] for
 * key (k0, k1) and counter ctr4[4k..4k+3], count counters (host arrays). */
int svpf_debug_philox(uint32_t k0, uint32_t k1, const uint32_t* ctr4, uint32_t* out4, int count);

/* Measured issue rates of the pipes the pair sweeps run on, on the current
 * device, per SM clock: MUFU results (ex2.approx / rcp.approx) and FP32
 * results (packed FFMA2), medians over one CTA per SM.  The roofline of the
 * pair-iteration (one ex2 + one rcp + 13 FP32 operations) is
 * min(mufu / 2, fp32 / 13) pair-iterations per clock per SM; the benchmark
 * uses it as its roofline denominator. */
int svpf_measure_pipe_rates(double* mufu_per_clk_sm, double* fp32_per_clk_sm);

#ifdef __cplusplus
}
#endif
#endif
