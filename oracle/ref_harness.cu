/*
 * ref_harness.cu -- TEST INFRASTRUCTURE ONLY.
 *
 * Linked with the reference's own sources (compiled in place, see
 * oracle/Makefile) into oracle/_ref/libsvpf_ref.so.  Exposes a small C API so
 * a Python script can drive the reference's svpf_step_graph tick by tick with
 * a pre-drawn noise tape and with its full state loaded and read back between
 * ticks (per-tick parity with state re-sync).
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "svpf.cuh"
#include "svpf_fully_fused_v2.cuh"
#include "svpf_multiscale.cuh"
#include "svpf_oracle.h"

/* Built twice: with the tape header forced in (parity build), and stock
 * (SVPF_REF_STOCK, timing build: curand untouched, counters never reset). */
#ifndef SVPF_REF_STOCK
__device__ const float* svpf_ref_tape_normals = nullptr;
__device__ const float* svpf_ref_tape_uniforms = nullptr;
__device__ int svpf_ref_tape_n = 0;
__device__ int svpf_ref_tape_normal_slots = 0;
__device__ int svpf_ref_tape_uniform_slots = 0;
__device__ int svpf_ref_tape_flags = 0;
#endif

namespace {
float* g_dev_normals = nullptr;
float* g_dev_uniforms = nullptr;
size_t g_cap_normals = 0, g_cap_uniforms = 0;

#ifndef SVPF_REF_STOCK
__global__ void reset_counters_kernel(curandStatePhilox4_32_10_t* st, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        st[i].ctr.x = (unsigned int)i;
        st[i].ctr.y = 0u;
        st[i].ctr.z = 0u;
    }
}
#endif

int check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        fprintf(stderr, "svpf_ref harness: %s: %s\n", what, cudaGetErrorString(e));
        return -1;
    }
    return 0;
}
}  // namespace

extern "C" {

#ifndef SVPF_REF_STOCK
int svpf_ref_tape_set(const float* normals, int n_normal_slots, const float* uniforms,
                      int n_uniform_slots, int n) {
    size_t bn = (size_t)n_normal_slots * n * sizeof(float);
    size_t bu = (size_t)n_uniform_slots * n * sizeof(float);
    if (bn > g_cap_normals) {
        if (g_dev_normals) cudaFree(g_dev_normals);
        if (check(cudaMalloc(&g_dev_normals, bn), "malloc normals")) return -1;
        g_cap_normals = bn;
    }
    if (bu > g_cap_uniforms) {
        if (g_dev_uniforms) cudaFree(g_dev_uniforms);
        if (check(cudaMalloc(&g_dev_uniforms, bu), "malloc uniforms")) return -1;
        g_cap_uniforms = bu;
    }
    if (bn && check(cudaMemcpy(g_dev_normals, normals, bn, cudaMemcpyHostToDevice), "copy normals")) return -1;
    if (bu && check(cudaMemcpy(g_dev_uniforms, uniforms, bu, cudaMemcpyHostToDevice), "copy uniforms")) return -1;
    const float* pn = bn ? g_dev_normals : nullptr;
    const float* pu = bu ? g_dev_uniforms : nullptr;
    if (check(cudaMemcpyToSymbol(svpf_ref_tape_normals, &pn, sizeof(pn)), "sym normals")) return -1;
    if (check(cudaMemcpyToSymbol(svpf_ref_tape_uniforms, &pu, sizeof(pu)), "sym uniforms")) return -1;
    if (check(cudaMemcpyToSymbol(svpf_ref_tape_n, &n, sizeof(int)), "sym n")) return -1;
    if (check(cudaMemcpyToSymbol(svpf_ref_tape_normal_slots, &n_normal_slots, sizeof(int)), "sym ns")) return -1;
    if (check(cudaMemcpyToSymbol(svpf_ref_tape_uniform_slots, &n_uniform_slots, sizeof(int)), "sym us")) return -1;
    return 0;
}

int svpf_ref_tape_flags_take(void) {
    int f = 0, z = 0;
    cudaDeviceSynchronize();
    cudaMemcpyFromSymbol(&f, svpf_ref_tape_flags, sizeof(int));
    cudaMemcpyToSymbol(svpf_ref_tape_flags, &z, sizeof(int));
    return f;
}
#else
int svpf_ref_tape_set(const float*, int, const float*, int, int) { return 0; }
int svpf_ref_tape_flags_take(void) { return 0; }
#endif

SVPFState* svpf_ref_create(int n, int n_stein, float nu) {
    SVPFState* s = svpf_create(n, n_stein, nu, nullptr);
    if (!s) return nullptr;
    /* The backend buffers are allocated lazily by a file-static function that
     * svpf_initialize reaches only on its two-factor branch. */
    SVPFParams p = {0.9f, 0.1f, -1.0f, 0.0f};
    s->use_two_factor = 1;
    svpf_initialize(s, &p, 0ull);
    s->use_two_factor = 0;
    /* Buffers the step reads before ever writing them start at zero. */
    cudaMemset(s->log_weights, 0, n * sizeof(float));
    cudaMemset(s->opt_backend.d_ksd, 0, sizeof(float));
    cudaMemset(s->opt_backend.d_bandwidth, 0, sizeof(float));
    cudaMemset(s->opt_backend.d_h_fast_mean, 0, sizeof(float));
    cudaMemset(s->opt_backend.d_h_slow_mean, 0, sizeof(float));
    cudaDeviceSynchronize();
    svpf_ref_tape_flags_take();
    return s;
}

void svpf_ref_destroy(SVPFState* s) { svpf_destroy(s); }

#define SVPF_REF_CONFIG_FIELDS(X)                                                     \
    X(n_stein_steps) X(nu) X(student_t_implied_offset) X(lik_offset)                  \
    X(use_exact_gradient) X(use_svld) X(use_annealing) X(use_adaptive_beta)           \
    X(n_anneal_steps) X(temperature) X(rmsprop_rho) X(rmsprop_eps) X(use_mim)         \
    X(mim_jump_prob) X(mim_jump_scale) X(use_local_params) X(delta_rho)               \
    X(delta_sigma) X(use_asymmetric_rho) X(rho_up) X(rho_down) X(use_newton)          \
    X(use_full_newton) X(use_guided) X(guided_alpha_base) X(guided_alpha_shock)       \
    X(guided_innovation_threshold) X(use_rejuvenation) X(rejuv_ksd_threshold)         \
    X(rejuv_prob) X(rejuv_blend) X(use_guide) X(use_guide_preserving)                 \
    X(guide_strength) X(use_adaptive_guide) X(guide_strength_base)                    \
    X(guide_strength_max) X(guide_innovation_threshold) X(use_adaptive_mu)            \
    X(mu_process_var) X(mu_obs_var_scale) X(mu_min) X(mu_max) X(use_adaptive_sigma)   \
    X(sigma_boost_threshold) X(sigma_boost_max) X(stein_repulsive_sign)               \
    X(use_fan_mode) X(stein_min_steps) X(stein_max_steps)                             \
    X(ksd_improvement_threshold) X(use_student_t_state) X(nu_state) X(use_smoothing)  \
    X(smooth_lag) X(smooth_output_lag) X(use_heun) X(use_two_factor) X(rho_fast)       \
    X(sigma_fast) X(rho_slow) X(sigma_slow) X(bw_floor_fast) X(bw_floor_slow)

void svpf_ref_apply_config(SVPFState* s, const oracle_config* c) {
#define X(f) s->f = c->f;
    SVPF_REF_CONFIG_FIELDS(X)
#undef X
}

void svpf_ref_read_config(const SVPFState* s, oracle_config* c) {
#define X(f) c->f = s->f;
    SVPF_REF_CONFIG_FIELDS(X)
#undef X
}

/* init_normals holds one draw per particle, three ([3][n]) with two factors. */
int svpf_ref_initialize(SVPFState* s, const oracle_params* p, const float* init_normals) {
    int n = s->n_particles;
    float one = 1.0f;
    if (svpf_ref_tape_set(init_normals, s->use_two_factor ? 3 : 1, &one, 0, n)) return -1;
    SVPFParams sp = {p->rho, p->sigma_z, p->mu, p->gamma};
    svpf_initialize(s, &sp, 0ull);
    return svpf_ref_tape_flags_take();
}

/* With two factors h, hp and v hold [fast (n); slow (n)] and map onto the
 * backend's d_h_fast/d_h_slow, *_prev and d_grad_v_* buffers. */
int svpf_ref_set_state(SVPFState* s, const oracle_ctl* c, const double* h, const double* hp,
                       const double* v, const double* lw) {
    int n = s->n_particles;
    SVPFOptimizedState* o = &s->opt_backend;
    if (!o->initialized) return -2;
    std::vector<float> buf(n);
    auto put = [&](float* dst, const double* src) {
        for (int i = 0; i < n; ++i) buf[i] = (float)src[i];
        return check(cudaMemcpy(dst, buf.data(), n * sizeof(float), cudaMemcpyHostToDevice), "put");
    };
    if (s->use_two_factor) {
        if (put(o->d_h_fast, h) || put(o->d_h_slow, h + n) || put(o->d_h_fast_prev, hp) ||
            put(o->d_h_slow_prev, hp + n) || put(o->d_grad_v_fast, v) || put(o->d_grad_v_slow, v + n) ||
            put(s->log_weights, lw))
            return -1;
        s->guide_mean_fast = (float)c->guide_mean_fast;
        s->guide_mean_slow = (float)c->guide_mean_slow;
        s->guide_var_fast = (float)c->guide_var_fast;
        s->guide_var_slow = (float)c->guide_var_slow;
        s->guide_2f_initialized = c->guide_2f_initialized;
    } else if (put(s->h, h) || put(s->h_prev, hp) || put(s->d_grad_v, v) || put(s->log_weights, lw)) {
        return -1;
    }
    auto put1 = [&](float* dst, float val) {
        return check(cudaMemcpy(dst, &val, sizeof(float), cudaMemcpyHostToDevice), "put1");
    };
    if (put1(o->d_h_mean_prev, c->h_mean_prev) || put1(o->d_bandwidth, c->bw) ||
        put1(o->d_bandwidth_sq, c->bw_sq) || put1(s->d_return_ema, c->return_ema) ||
        put1(s->d_return_var, c->return_var) || put1(o->d_ksd, c->ksd_last) ||
        put1(o->d_h_fast_mean, c->h_fast_mean) || put1(o->d_h_slow_mean, c->h_slow_mean))
        return -1;
    s->timestep = c->timestep;
    s->guide_initialized = c->guide_initialized;
    s->stein_steps_used = c->stein_steps_used;
    s->smooth_head = c->smooth_head;
    s->guide_mean = (float)c->guide_mean;
    s->guide_var = (float)c->guide_var;
    s->guide_K = (float)c->guide_K;
    s->ksd_prev = c->ksd_prev;
    s->vol_prev = c->vol_prev;
    s->sigma_z_effective = c->sigma_z_effective;
    s->mu_state = c->mu_state;
    s->mu_var = c->mu_var;
    for (int i = 0; i < SVPF_SMOOTH_MAX_LAG && i < ORACLE_SMOOTH_MAX_LAG; ++i) {
        s->smooth_h_mean[i] = c->smooth_h_mean[i];
        s->smooth_h_var[i] = c->smooth_h_var[i];
        s->smooth_y[i] = c->smooth_y[i];
    }
    return 0;
}

int svpf_ref_get_state(SVPFState* s, oracle_ctl* c, double* h, double* hp, double* v, double* lw) {
    int n = s->n_particles;
    SVPFOptimizedState* o = &s->opt_backend;
    if (!o->initialized) return -2;
    cudaDeviceSynchronize();
    std::vector<float> buf(n);
    auto get = [&](double* dst, const float* src) {
        if (check(cudaMemcpy(buf.data(), src, n * sizeof(float), cudaMemcpyDeviceToHost), "get")) return -1;
        for (int i = 0; i < n; ++i) dst[i] = buf[i];
        return 0;
    };
    if (s->use_two_factor) {
        if (get(h, o->d_h_fast) || get(h + n, o->d_h_slow) || get(hp, o->d_h_fast_prev) ||
            get(hp + n, o->d_h_slow_prev) || get(v, o->d_grad_v_fast) || get(v + n, o->d_grad_v_slow) ||
            get(lw, s->log_weights))
            return -1;
        c->guide_mean_fast = s->guide_mean_fast;
        c->guide_mean_slow = s->guide_mean_slow;
        c->guide_var_fast = s->guide_var_fast;
        c->guide_var_slow = s->guide_var_slow;
        c->guide_2f_initialized = s->guide_2f_initialized;
    } else if (get(h, s->h) || get(hp, s->h_prev) || get(v, s->d_grad_v) || get(lw, s->log_weights)) {
        return -1;
    }
    auto get1 = [&](float* dst, const float* src) {
        return check(cudaMemcpy(dst, src, sizeof(float), cudaMemcpyDeviceToHost), "get1");
    };
    if (get1(&c->h_mean_prev, o->d_h_mean_prev) || get1(&c->bw, o->d_bandwidth) ||
        get1(&c->bw_sq, o->d_bandwidth_sq) || get1(&c->return_ema, s->d_return_ema) ||
        get1(&c->return_var, s->d_return_var) || get1(&c->ksd_last, o->d_ksd) ||
        get1(&c->h_fast_mean, o->d_h_fast_mean) || get1(&c->h_slow_mean, o->d_h_slow_mean))
        return -1;
    c->timestep = s->timestep;
    c->guide_initialized = s->guide_initialized;
    c->stein_steps_used = s->stein_steps_used;
    c->smooth_head = s->smooth_head;
    c->guide_mean = s->guide_mean;
    c->guide_var = s->guide_var;
    c->guide_K = s->guide_K;
    c->ksd_prev = s->ksd_prev;
    c->vol_prev = s->vol_prev;
    c->sigma_z_effective = s->sigma_z_effective;
    c->mu_state = s->mu_state;
    c->mu_var = s->mu_var;
    for (int i = 0; i < SVPF_SMOOTH_MAX_LAG && i < ORACLE_SMOOTH_MAX_LAG; ++i) {
        c->smooth_h_mean[i] = s->smooth_h_mean[i];
        c->smooth_h_var[i] = s->smooth_h_var[i];
        c->smooth_y[i] = s->smooth_y[i];
    }
    return 0;
}

/* One reference tick with the given tape.  Returns the tape flags (0 = ok). */
int svpf_ref_step(SVPFState* s, float y_t, float y_prev, const oracle_params* p,
                  const float* normals, int n_normal_slots, const float* uniforms,
                  int n_uniform_slots, float* ll, float* vol, float* hm) {
    int n = s->n_particles;
    if (svpf_ref_tape_set(normals, n_normal_slots, uniforms, n_uniform_slots, n)) return -1;
#ifndef SVPF_REF_STOCK
    reset_counters_kernel<<<(n + 255) / 256, 256, 0, s->stream>>>(s->rng_states, n);
#endif
    SVPFParams sp = {p->rho, p->sigma_z, p->mu, p->gamma};
    svpf_step_graph(s, y_t, y_prev, &sp, ll, vol, hm);
    if (check(cudaGetLastError(), "step")) return -1;
    return svpf_ref_tape_flags_take();
}

/* One svpf_fully_fused_step_v2 call (the reference's single-kernel step) on
 * host arrays [n], with the noise tape. Returns the tape flags, or -1. */
int svpf_ref_v2_step(const oracle_v2_params* p, int n, double* h, double* hp, double* grad, double* lw,
                     double* v, double* ih, float y_t, float y_prev, float h_mean_prev, float vol_prev,
                     float ksd_prev, int timestep, double* gmean, double* gvar, double* mustate,
                     const float* normals, int slots_n, const float* uniforms, int slots_u, oracle_v2_out* out) {
    std::vector<float> buf(7 * (size_t)n);
    float* d = nullptr;
    curandStatePhilox4_32_10_t* rng = nullptr;
    float* sc = nullptr;   // h_mean, vol, loglik, bw, ksd, guide_mean, guide_var, mu_state
    if (check(cudaMalloc(&d, 6 * (size_t)n * sizeof(float)), "v2 arrays") ||
        check(cudaMalloc(&rng, (size_t)n * sizeof(*rng)), "v2 rng") || check(cudaMalloc(&sc, 8 * sizeof(float)), "v2 sc"))
        return -1;
    double* arrs[6] = {h, hp, grad, lw, v, ih};
    for (int a = 0; a < 6; ++a)
        for (int i = 0; i < n; ++i) buf[(size_t)a * n + i] = (float)arrs[a][i];
    float scal[8] = {0, 0, 0, 0, 0, (float)*gmean, (float)*gvar, (float)*mustate};
    int rc = 0;
    if (check(cudaMemcpy(d, buf.data(), 6 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice), "v2 in") ||
        check(cudaMemcpy(sc, scal, sizeof(scal), cudaMemcpyHostToDevice), "v2 sc in"))
        rc = -1;
#ifndef SVPF_REF_STOCK
    if (!rc && svpf_ref_tape_set(normals, slots_n, uniforms, slots_u, n)) rc = -1;
    if (!rc) reset_counters_kernel<<<(n + 255) / 256, 256>>>(rng, n);
#endif
    if (!rc) {
        cudaError_t e = svpf_fully_fused_step_v2(
            d, d + n, d + 2 * n, d + 3 * n, d + 4 * n, d + 5 * n, rng, y_t, y_prev, h_mean_prev, vol_prev, ksd_prev,
            sc, sc + 1, sc + 2, sc + 3, sc + 4, sc + 5, sc + 6, p->rho, p->sigma_z, p->mu, p->nu, p->lik_offset,
            p->student_t_const, p->student_t_implied_offset, p->gamma, p->delta_rho, p->delta_sigma,
            p->mim_jump_prob, p->mim_jump_scale, p->guide_strength_base, p->guide_strength_max,
            p->guide_innovation_threshold, p->guided_alpha_base, p->guided_alpha_shock,
            p->guided_innovation_thresh_predict, p->use_guide, p->use_guided_predict, p->use_guide_preserving,
            p->use_newton, p->use_full_newton, p->use_rejuvenation, p->rejuv_ksd_threshold, p->rejuv_prob,
            p->rejuv_blend, p->use_adaptive_mu, sc + 7, p->mu_ema_alpha, p->use_adaptive_sigma,
            p->sigma_boost_threshold, p->sigma_boost_max, p->step_size, p->temperature, p->rmsprop_rho,
            p->rmsprop_eps, p->n_stein_steps, p->n_anneal_steps, p->stein_sign_mode, n, timestep, 0);
        if (check(e, "v2 step") || check(cudaDeviceSynchronize(), "v2 sync")) rc = -1;
    }
    if (!rc && (check(cudaMemcpy(buf.data(), d, 6 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost), "v2 out") ||
                check(cudaMemcpy(scal, sc, sizeof(scal), cudaMemcpyDeviceToHost), "v2 sc out")))
        rc = -1;
    if (!rc) {
        for (int a = 0; a < 6; ++a)
            for (int i = 0; i < n; ++i) arrs[a][i] = buf[(size_t)a * n + i];
        out->h_mean = scal[0]; out->vol = scal[1]; out->loglik = scal[2]; out->bandwidth = scal[3]; out->ksd = scal[4];
        *gmean = scal[5]; *gvar = scal[6]; *mustate = scal[7];
        rc = svpf_ref_tape_flags_take();
    }
    cudaFree(d);
    cudaFree(rng);
    cudaFree(sc);
    return rc;
}

namespace {
__global__ void v2_rng_init_kernel(curandStatePhilox4_32_10_t* st, int n, unsigned long long seed) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) curand_init(seed, i, 0, &st[i]);
}
}  // namespace

/* Latency of the reference's svpf_fully_fused_step_v2: T calls on one filter
 * (stationary start, its own cuRAND states), CUDA events around each call as
 * test/test_fully_fused_v2.cu:194-219 does; us_per_call[T].  Returns 0, or
 * -(1000 + cudaError_t) when the reference's launch itself failed. */
int svpf_ref_v2_time(const oracle_v2_params* p, int n, const float* ys, int T, float* us_per_call) {
    float* d = nullptr;
    curandStatePhilox4_32_10_t* rng = nullptr;
    float* sc = nullptr;
    if (check(cudaMalloc(&d, 6 * (size_t)n * sizeof(float)), "v2t arrays") ||
        check(cudaMalloc(&rng, (size_t)n * sizeof(*rng)), "v2t rng") || check(cudaMalloc(&sc, 8 * sizeof(float)), "v2t sc"))
        return -1;
    std::vector<float> h0(6 * (size_t)n, 0.0f);
    for (int i = 0; i < n; ++i) h0[i] = p->mu + 0.3f * (float)((i * 7919) % 1000 - 500) / 500.0f;
    float scal[8] = {0, 0, 0, 0, 0, 0, 0, p->mu};
    cudaMemcpy(d, h0.data(), h0.size() * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(sc, scal, sizeof(scal), cudaMemcpyHostToDevice);
    v2_rng_init_kernel<<<(n + 255) / 256, 256>>>(rng, n, 1234ull);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float y_prev = 0.0f, h_mean_prev = p->mu, vol_prev = expf(p->mu * 0.5f), ksd_prev = 0.1f;
    int launch_error = 0;
    for (int t = 0; t < T; ++t) {
        cudaEventRecord(a, 0);
        const cudaError_t le = svpf_fully_fused_step_v2(
            d, d + n, d + 2 * n, d + 3 * n, d + 4 * n, d + 5 * n, rng, ys[t], y_prev, h_mean_prev, vol_prev, ksd_prev,
            sc, sc + 1, sc + 2, sc + 3, sc + 4, sc + 5, sc + 6, p->rho, p->sigma_z, p->mu, p->nu, p->lik_offset,
            p->student_t_const, p->student_t_implied_offset, p->gamma, p->delta_rho, p->delta_sigma,
            p->mim_jump_prob, p->mim_jump_scale, p->guide_strength_base, p->guide_strength_max,
            p->guide_innovation_threshold, p->guided_alpha_base, p->guided_alpha_shock,
            p->guided_innovation_thresh_predict, p->use_guide, p->use_guided_predict, p->use_guide_preserving,
            p->use_newton, p->use_full_newton, p->use_rejuvenation, p->rejuv_ksd_threshold, p->rejuv_prob,
            p->rejuv_blend, p->use_adaptive_mu, sc + 7, p->mu_ema_alpha, p->use_adaptive_sigma,
            p->sigma_boost_threshold, p->sigma_boost_max, p->step_size, p->temperature, p->rmsprop_rho,
            p->rmsprop_eps, p->n_stein_steps, p->n_anneal_steps, p->stein_sign_mode, n, t, 0);
        if (le != cudaSuccess && !launch_error) launch_error = (int)le;
        cudaEventRecord(b, 0);
        cudaEventSynchronize(b);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        us_per_call[t] = ms * 1000.0f;
        cudaMemcpy(scal, sc, 5 * sizeof(float), cudaMemcpyDeviceToHost);
        h_mean_prev = scal[0];
        vol_prev = scal[1];
        ksd_prev = scal[4];
        y_prev = ys[t];
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    cudaFree(rng);
    cudaFree(sc);
    cudaGetLastError();
    /* a launch the reference's kernel could not make: its cudaError_t, as -(1000 + code) */
    return launch_error ? -(1000 + launch_error) : 0;
}

/* Latency probe: CUDA events around each svpf_step_graph call, the way the
 * reference's own profiler times it (test/profile_svpf.cu:131-143). */
int svpf_ref_time_steps(SVPFState* s, const float* ys, int T, const oracle_params* p,
                        float* us_per_step) {
    SVPFParams sp = {p->rho, p->sigma_z, p->mu, p->gamma};
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float yp = 0.0f;
    for (int t = 0; t < T; ++t) {
        float ll, vol, hm;
#ifndef SVPF_REF_STOCK
        reset_counters_kernel<<<(s->n_particles + 255) / 256, 256, 0, s->stream>>>(s->rng_states,
                                                                                   s->n_particles);
#endif
        cudaEventRecord(a, s->stream);
        svpf_step_graph(s, ys[t], yp, &sp, &ll, &vol, &hm);
        cudaEventRecord(b, s->stream);
        cudaEventSynchronize(b);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        us_per_step[t] = ms * 1000.0f;
        yp = ys[t];
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return check(cudaGetLastError(), "time");
}

/* ---- the reference's two-scale composition (include/svpf_multiscale.cuh),
 * driven unmodified: ms_svpf_create / ms_svpf_init / ms_svpf_step.  In the
 * tape build both scales draw from one tape of stride n_max, particle i of
 * either scale reading column i (the layout of one tape shared by a batch). */
MS_SVPF* svpf_ref_ms_create(void) { return ms_svpf_create(NULL); }

void svpf_ref_ms_destroy(MS_SVPF* ms) { ms_svpf_destroy(ms); }

/* which: 0 = REACTIVE, 1 = INERTIAL (for svpf_ref_get_state / set_state). */
SVPFState* svpf_ref_ms_filter(MS_SVPF* ms, int which) { return which ? ms->inertial : ms->reactive; }

int svpf_ref_ms_init(MS_SVPF* ms, float initial_vol, const oracle_params* p, const float* init_normals, int n_max) {
    float one = 1.0f;
    if (svpf_ref_tape_set(init_normals, 1, &one, 0, n_max)) return -1;
    SVPFParams sp = {p->rho, p->sigma_z, p->mu, p->gamma};
    ms_svpf_init(ms, initial_vol, &sp, 0u);
    cudaDeviceSynchronize();
    return svpf_ref_tape_flags_take();
}

int svpf_ref_ms_step(MS_SVPF* ms, float y_t, const oracle_params* p, const float* normals, int n_normal_slots,
                     const float* uniforms, int n_uniform_slots, int n_max, MS_SVPF_Output* out) {
#ifndef SVPF_REF_STOCK
    SVPFState* fs[2] = {ms->reactive, ms->inertial};
    for (SVPFState* s : fs)
        reset_counters_kernel<<<(s->n_particles + 255) / 256, 256, 0, s->stream>>>(s->rng_states, s->n_particles);
    cudaDeviceSynchronize();
#endif
    if (svpf_ref_tape_set(normals, n_normal_slots, uniforms, n_uniform_slots, n_max)) return -1;
    SVPFParams sp = {p->rho, p->sigma_z, p->mu, p->gamma};
    ms_svpf_step(ms, y_t, &sp, out);
    cudaDeviceSynchronize();
    return svpf_ref_tape_flags_take();
}

/* Stein iterations the last svpf_step_graph call ran (the reference keeps it
 * in the state, svpf_optimized_graph.cu:1490-1493). */
int svpf_ref_steps_used(const SVPFState* s) { return s->stein_steps_used; }

}  // extern "C"
