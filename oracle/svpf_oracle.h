/*
 * svpf_oracle.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * CPU restatement of one Stein Variational Particle Filter tick as the
 * reference computes it (src/svpf_optimized_graph.cu:915-1389 driving the
 * kernels of src/svpf_opt_kernels.cu:125-1566 and the host EKF of
 * include/svpf_kernels.cuh:509-541).  Only tests/, the smoke check and the
 * CPU-baseline leg of bench.py may load it.  It is never part of the product
 * path.
 *
 * The structs below are laid out field for field like the product's
 * svpf_config_t / svpf_params_t / svpf_ctl_t so one ctypes definition can
 * fill both, but they are declared here independently.
 */
#ifndef SVPF_ORACLE_H
#define SVPF_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_SMOOTH_MAX_LAG 8

/* Filter configuration: same names and defaults as the SVPFState fields of the
 * reference (include/svpf.cuh:337-545, defaults svpf_optimized_graph.cu:116-283). */
typedef struct {
    int   n_stein_steps;
    float nu;
    float student_t_implied_offset;  /* fixed at create from nu (:127-138) */
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
    int   use_adaptive_guide;
    float guide_strength_base;
    float guide_strength_max;
    float guide_innovation_threshold;
    int   use_adaptive_mu;
    float mu_process_var;
    float mu_obs_var_scale;
    float mu_min;
    float mu_max;
    int   use_adaptive_sigma;
    float sigma_boost_threshold;
    float sigma_boost_max;
    int   stein_repulsive_sign;
    int   use_fan_mode;
    int   stein_min_steps;
    int   stein_max_steps;
    float ksd_improvement_threshold;
    int   use_student_t_state;
    float nu_state;
    int   use_smoothing;
    int   smooth_lag;
    int   smooth_output_lag;
    int   use_heun;
    int   use_two_factor;
    float rho_fast;
    float sigma_fast;
    float rho_slow;
    float sigma_slow;
    float bw_floor_fast;
    float bw_floor_slow;
} oracle_config;

/* SVPFParams of the reference (include/svpf.cuh:257-262). */
typedef struct {
    float rho;
    float sigma_z;
    float mu;
    float gamma;
} oracle_params;

/* Per-filter control state carried from tick to tick.  In the reference these
 * live partly in host fields of SVPFState (timestep, ksd_prev, vol_prev,
 * guide_*, mu_*, smooth_*) and partly in device scalars of the backend
 * (d_h_mean_prev, d_bandwidth[_sq], d_return_ema/var, d_ksd). */
typedef struct {
    double guide_mean;
    double guide_var;
    double guide_K;
    double loglik_sum;          /* FP64 running sum of per-tick log-likelihoods */
    double guide_mean_fast;     /* two-factor EKF, svpf_two_factor.cuh:245-300 */
    double guide_mean_slow;
    double guide_var_fast;
    double guide_var_slow;
    int    timestep;
    int    guide_initialized;
    int    stein_steps_used;
    int    smooth_head;
    int    guide_2f_initialized;
    float  ksd_prev;            /* host ksd_prev: drives budget/beta/rejuvenation */
    float  ksd_last;            /* device d_ksd: last KSD actually computed */
    float  vol_prev;
    float  h_mean_prev;         /* device d_h_mean_prev (-3.5 on first use) */
    float  bw;
    float  bw_sq;
    float  return_ema;
    float  return_var;
    float  sigma_z_effective;
    float  mu_state;
    float  mu_var;
    float  y_prev;              /* used by svpf_step(): previous observation */
    float  h_fast_mean;         /* device d_h_fast_mean / d_h_slow_mean */
    float  h_slow_mean;
    float  smooth_h_mean[ORACLE_SMOOTH_MAX_LAG];
    float  smooth_h_var[ORACLE_SMOOTH_MAX_LAG];
    float  smooth_y[ORACLE_SMOOTH_MAX_LAG];
    int    status;
    int    reserved;
} oracle_ctl;

typedef struct {
    float loglik;
    float vol;
    float h_mean;        /* output h mean (smoothed when smoothing is on) */
    float h_mean_raw;
    float bw;
    float ksd;
    int   steps_used;
    int   rejuv_fired;
} oracle_out;

/* Noise for one tick.  mode 0: tape; normals[k*n + i] is the k-th normal draw
 * of particle i within the tick, uniforms likewise.  mode 1: the project's
 * counter-based Philox4x32-10 keyed by (seed, filter) and counted by
 * (particle, draw, tick). */
typedef struct {
    int          mode;
    int          n_normal_slots;
    int          n_uniform_slots;
    int          filter_id;
    const float* normals;
    const float* uniforms;
    uint64_t     seed;
    uint64_t     tick;
} oracle_noise;

/* Run one tick.  Arrays are double on the interface; precision 0 computes in
 * FP64, precision 1 computes in FP32 (the CPU baseline).  Returns 0 on
 * success, a negative code on bad arguments or when the tape runs short.
 * With use_two_factor, h / h_prev / v hold 2n values: the fast factor then
 * the slow factor. */
/* ---- svpf_fully_fused_step_v2 (include/svpf_fully_fused_v2.cuh:43-119) ----- */
typedef struct {
    float rho, sigma_z, mu, nu, lik_offset, student_t_const, student_t_implied_offset, gamma;
    float delta_rho, delta_sigma;
    float mim_jump_prob, mim_jump_scale;
    float guide_strength_base, guide_strength_max, guide_innovation_threshold;
    float guided_alpha_base, guided_alpha_shock, guided_innovation_thresh_predict;
    int   use_guide, use_guided_predict, use_guide_preserving;
    int   use_newton, use_full_newton;
    int   use_rejuvenation;
    float rejuv_ksd_threshold, rejuv_prob, rejuv_blend;
    int   use_adaptive_mu;
    float mu_ema_alpha;
    int   use_adaptive_sigma;
    float sigma_boost_threshold, sigma_boost_max;
    float step_size, temperature, rmsprop_rho, rmsprop_eps;
    int   n_stein_steps, n_anneal_steps, stein_sign_mode;
} oracle_v2_params;

typedef struct {
    float h_mean, vol, loglik, bandwidth, ksd;
} oracle_v2_out;

/* One svpf_fully_fused_step_v2 call (src/svpf_fully_fused_v2.cu:90-745).
 * Arrays [n] (grad, lw, inv_hess: last Stein iteration's values); guide_mean,
 * guide_var and mu_state are the device scalars it reads and writes.  Noise
 * slots per particle: normals 0..3 from the curand_normal4 draw (0 state, 1
 * first diffusion), then one normal per Stein iteration with SVLD
 * (refresh), then the rejuvenation normal; uniforms 0 (MIM), 1 (rejuvenation). */
int svpf_oracle_v2_tick(const oracle_v2_params* p, int n, double* h, double* h_prev, double* grad,
                        double* lw, double* v, double* inv_hess, float y_t, float y_prev,
                        float h_mean_prev, float vol_prev, float ksd_prev, int timestep,
                        double* guide_mean, double* guide_var, double* mu_state,
                        const oracle_noise* noise, oracle_v2_out* out, int precision);

int svpf_oracle_tick(const oracle_config* cfg, const oracle_params* p,
                     oracle_ctl* ctl, int n,
                     double* h, double* h_prev, double* v, double* log_w,
                     float y_t, float y_prev, const oracle_noise* noise,
                     oracle_out* out, int precision);

/* FP32 batched baseline: filters are independent, OpenMP over filters.
 * Arrays are float [n_filters][n_max]; per-filter n in ns[]. */
int svpf_oracle_batch_tick_f32(int n_filters, const oracle_config* cfgs,
                               const oracle_params* ps, oracle_ctl* ctls,
                               const int* ns, int n_max,
                               float* h, float* h_prev, float* v, float* log_w,
                               const float* y_t, const float* y_prev,
                               uint64_t seed, uint64_t tick, int n_threads,
                               oracle_out* outs);

/* svpf_initialize (svpf_optimized_graph.cu:349-451): stationary draw, resets.
 * init_normals[i] is particle i's draw (tape) or NULL for Philox mode; with
 * use_two_factor the tape holds three draws per particle ([3][n]: the
 * single-factor draw, then fast, then slow) and h/h_prev/v hold 2n values. */
int svpf_oracle_initialize(oracle_config* cfg, const oracle_params* p,
                           oracle_ctl* ctl, int n, double* h, double* h_prev,
                           double* v, const float* init_normals,
                           uint64_t seed, int filter_id);

/* Fresh control record as svpf_create + the lazy backend init leave it. */
void svpf_oracle_ctl_defaults(oracle_ctl* ctl);
void svpf_oracle_config_defaults(oracle_config* cfg, int n_stein_steps, float nu);

/* Philox4x32-10 block (Salmon et al. 2011), for bit-exact checks of the GPU
 * generator: out[0..3] for key (k0,k1) and counter (c0..c3). */
void svpf_oracle_philox(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1,
                        uint32_t c2, uint32_t c3, uint32_t* out);


/* ---- gradient oracle (forward-mode AD in FP64) ---------------------------- */
int svpf_oracle_grad_supported(const oracle_config* cfg);
int svpf_oracle_grad_run(const oracle_config* cfg, int n, int T, const double* theta, double gamma,
                         const float* ys, const double* w, uint64_t seed, int filter_id,
                         double* loglik, double* grad, double* h_final);
/* objective 0: tick log-likelihood (as svpf_oracle_grad_run); 1: predictive
 * log-likelihood log mean_i p(y_t | predicted h_i). */
int svpf_oracle_grad_run2(const oracle_config* cfg, int n, int T, const double* theta, double gamma,
                          const float* ys, const double* w, uint64_t seed, int filter_id,
                          double* loglik, double* grad, double* h_final, int objective);
/* As svpf_oracle_grad_run2, with truncated backpropagation through time:
 * for t > 0 with t % truncate_every == 0 the state carried into tick t
 * (particles, RMSProp moments, EKF guide mean and variance, bandwidth
 * average, previous mean) is held constant in theta -- in forward mode its
 * tangents are zeroed (0: no truncation). */
int svpf_oracle_grad_run3(const oracle_config* cfg, int n, int T, const double* theta, double gamma,
                          const float* ys, const double* w, uint64_t seed, int filter_id,
                          double* loglik, double* grad, double* h_final, int objective, int truncate_every);

/* ---- the reference's differentiable torch model (forward-mode AD, FP64) --- */
/* SVPFParamEstimator.forward (py-torch/diff_svpf_torch.py:147-217) for one
 * path: n particles (even), n_stein Stein steps of size stein_lr, T ticks of
 * ys, the noise the model draws as a tape (tape_init[n]: initial particles;
 * tape_ticks[T][n/2]: the antithetic half per tick), theta = (mu, rho,
 * sigma_z, nu), TBPTT every truncate_every ticks (0: none).  Writes
 * loglik[T] (predictive, before the transport), vol[T] (mean e^{h/2} after
 * it) and grad[4] = d(sum_t w_t loglik_t)/d theta (w = NULL: all ones).
 * Returns 0, or -1 for invalid sizes. */
int svpf_oracle_estimator_run(int n, int n_stein, double stein_lr, int T, const float* ys,
                              const float* tape_init, const float* tape_ticks, const double* theta,
                              int truncate_every, const double* w, double* loglik, double* vol,
                              double* grad);
/* The same with the per-tick bandwidths replayed from bw_fixed[T] (NULL: the
 * model's own) and recorded into bw_out[T] (NULL: not recorded): central
 * differences with the bandwidth frozen are what the detached bandwidth's
 * derivative means. */
int svpf_oracle_estimator_run2(int n, int n_stein, double stein_lr, int T, const float* ys,
                               const float* tape_init, const float* tape_ticks, const double* theta,
                               int truncate_every, const double* w, double* loglik, double* vol,
                               double* grad, const double* bw_fixed, double* bw_out);

#ifdef __cplusplus
}
#endif
#endif
