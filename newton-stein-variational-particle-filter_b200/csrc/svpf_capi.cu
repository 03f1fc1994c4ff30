// svpf_capi.cu -- the C ABI (include/svpf.h): the reference's single-filter
// entry points over the one-launch-per-tick kernel, and the batch API over the
// persistent kernel.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

#include "svpf.h"
#include "svpf_internal.h"
#include "svpf_trace.h"

using namespace svpf;

namespace {

#define SVPF_CFG_COPY_IN_(f) dst->f = src->f;

void config_from_state(const SVPFState* src, svpf_config_t* dst) {
    SVPF_CONFIG_FIELDS(SVPF_CFG_COPY_IN_, SVPF_CFG_COPY_IN_)
}
void config_to_state(const svpf_config_t* src, SVPFState* dst) {
    SVPF_CONFIG_FIELDS(SVPF_CFG_COPY_IN_, SVPF_CFG_COPY_IN_)
}

// svpf_create defaults (svpf_optimized_graph.cu:116-283)
void set_defaults(SVPFState* s, int n_stein_steps, float nu) {
    s->n_stein_steps = n_stein_steps;
    s->nu = nu;
    s->timestep = 0;
    s->y_prev = 0.0f;
    s->student_t_const = lgammaf((nu + 1.0f) / 2.0f) - lgammaf(nu / 2.0f) - 0.5f * logf(3.14159265358979f * nu);
    {
        // E[log t_nu^2] = log nu + psi(1/2) - psi(nu/2), psi by its asymptotic series (:127-138)
        const float psi_half = -1.9635100260214235f;
        const float nh = nu / 2.0f;
        const float psi = nh >= 1.0f ? logf(nh) - 1.0f / (2.0f * nh) - 1.0f / (12.0f * nh * nh)
                                     : -0.5772156649f - 1.0f / nh;
        s->student_t_implied_offset = -(logf(nu) + psi_half - psi);
    }
    s->lik_offset = 0.45f;
    s->use_exact_gradient = 0;
    s->use_svld = 1;
    s->use_annealing = 1;
    s->use_adaptive_beta = 1;
    s->n_anneal_steps = 3;
    s->temperature = 1.0f;
    s->rmsprop_rho = 0.9f;
    s->rmsprop_eps = 1e-6f;
    s->use_mim = 1;
    s->mim_jump_prob = 0.05f;
    s->mim_jump_scale = 5.0f;
    s->use_asymmetric_rho = 1;
    s->rho_up = 0.98f;
    s->rho_down = 0.93f;
    s->use_guide = 1;
    s->use_guide_preserving = 1;
    s->guide_strength = 0.05f;
    s->guide_mean = 0.0f;
    s->guide_var = 0.0f;
    s->guide_K = 0.0f;
    s->guide_initialized = 0;
    s->use_adaptive_guide = 0;
    s->guide_strength_base = 0.05f;
    s->guide_strength_max = 0.30f;
    s->guide_innovation_threshold = 1.0f;
    s->vol_prev = 0.05f;
    s->use_rejuvenation = 1;
    s->rejuv_ksd_threshold = 0.30f;
    s->rejuv_prob = 0.30f;
    s->rejuv_blend = 0.30f;
    s->use_newton = 0;
    s->use_full_newton = 0;
    s->use_guided = 0;
    s->guided_alpha_base = 0.0f;
    s->guided_alpha_shock = 0.5f;
    s->guided_innovation_threshold = 1.5f;
    s->use_local_params = 0;
    s->delta_rho = 0.02f;
    s->delta_sigma = 0.1f;
    s->use_adaptive_mu = 0;
    s->mu_state = -3.5f;
    s->mu_var = 1.0f;
    s->mu_process_var = 0.001f;
    s->mu_obs_var_scale = 10.0f;
    s->mu_min = -6.0f;
    s->mu_max = -1.0f;
    s->use_adaptive_sigma = 0;
    s->sigma_boost_threshold = 1.0f;
    s->sigma_boost_max = 3.0f;
    s->sigma_z_effective = 0.10f;
    s->stein_repulsive_sign = SVPF_STEIN_SIGN_DEFAULT;
    s->use_fan_mode = 0;
    s->use_student_t_state = 0;
    s->nu_state = 5.0f;
    s->stein_min_steps = 4;
    s->stein_max_steps = 12;
    s->ksd_improvement_threshold = 0.05f;
    s->ksd_prev = 1e10f;
    s->stein_steps_used = n_stein_steps;
    s->use_heun = 0;
    // two-factor (:257-271)
    s->use_two_factor = 0;
    s->rho_fast = 0.90f;
    s->sigma_fast = 0.15f;
    s->rho_slow = 0.99f;
    s->sigma_slow = 0.05f;
    s->bw_floor_fast = 0.01f;
    s->bw_floor_slow = 0.05f;
    s->guide_mean_fast = 0.0f;
    s->guide_mean_slow = 0.0f;
    s->guide_var_fast = 0.0f;
    s->guide_var_slow = 0.0f;
    s->guide_2f_initialized = 0;
    s->use_smoothing = 0;
    s->smooth_lag = 3;
    s->smooth_output_lag = 1;
    for (int i = 0; i < SVPF_SMOOTH_MAX_LAG; ++i) {
        s->smooth_h_mean[i] = 0.0f;
        s->smooth_h_var[i] = 1.0f;
        s->smooth_y[i] = 0.0f;
    }
    s->smooth_head = 0;
    s->use_persistent_kernel = 0;
    s->persistent_kernel_supported = 1;
}

// Engine-private part of a single filter.
struct Impl {
    svpf_ctl_t* res_ctl = nullptr;   // host-mapped result record
    svpf_out_t* res_out = nullptr;
    svpf_ctl_t* dev_res_ctl = nullptr;
    svpf_out_t* dev_res_out = nullptr;
    unsigned int* done = nullptr;     // host-mapped completion word of the last step
    unsigned int* dev_done = nullptr;
    unsigned int seq = 0;
    svpf_ctl_t cache;                 // control fields without an SVPFState counterpart
    svpf_out_t last{};
    float* tape_n = nullptr;
    float* tape_u = nullptr;
    int slots_n = 0, slots_u = 0;
    size_t cap_n = 0, cap_u = 0;
    bool tape_on = false;
    float* h2 = nullptr;              // two-factor particles [fast (n); slow (n)]
    float* hp2 = nullptr;
    float* v2 = nullptr;
    unsigned long long seed = 0;
    int cluster = 0;                  // 0 = automatic
    int tile = -1;
    int err = SVPF_OK;
    long long launches = 0;
};

Impl* impl_of(const SVPFState* s) { return s ? reinterpret_cast<Impl*>(s->impl) : nullptr; }

// Build the control record of the next tick from the state's fields and the
// engine cache (the state's fields win where both exist).
void ctl_gather(const SVPFState* s, const Impl* im, svpf_ctl_t* c) {
    *c = im->cache;
    if ((float)c->guide_mean != s->guide_mean) c->guide_mean = s->guide_mean;
    if ((float)c->guide_var != s->guide_var) c->guide_var = s->guide_var;
    c->guide_K = s->guide_K;
    c->timestep = s->timestep;
    c->guide_initialized = s->guide_initialized;
    c->stein_steps_used = s->stein_steps_used;
    c->smooth_head = s->smooth_head;
    c->ksd_prev = s->ksd_prev;
    c->vol_prev = s->vol_prev;
    c->sigma_z_effective = s->sigma_z_effective;
    c->mu_state = s->mu_state;
    c->mu_var = s->mu_var;
    c->y_prev = s->y_prev;
    if ((float)c->guide_mean_fast != s->guide_mean_fast) c->guide_mean_fast = s->guide_mean_fast;
    if ((float)c->guide_mean_slow != s->guide_mean_slow) c->guide_mean_slow = s->guide_mean_slow;
    if ((float)c->guide_var_fast != s->guide_var_fast) c->guide_var_fast = s->guide_var_fast;
    if ((float)c->guide_var_slow != s->guide_var_slow) c->guide_var_slow = s->guide_var_slow;
    c->guide_2f_initialized = s->guide_2f_initialized;
    for (int i = 0; i < SVPF_SMOOTH_MAX_LAG; ++i) {
        c->smooth_h_mean[i] = s->smooth_h_mean[i];
        c->smooth_h_var[i] = s->smooth_h_var[i];
        c->smooth_y[i] = s->smooth_y[i];
    }
}

void ctl_scatter(const svpf_ctl_t* c, SVPFState* s, Impl* im) {
    im->cache = *c;
    s->guide_mean = (float)c->guide_mean;
    s->guide_var = (float)c->guide_var;
    s->guide_K = (float)c->guide_K;
    s->timestep = c->timestep;
    s->guide_initialized = c->guide_initialized;
    s->stein_steps_used = c->stein_steps_used;
    s->smooth_head = c->smooth_head;
    s->ksd_prev = c->ksd_prev;
    s->vol_prev = c->vol_prev;
    s->sigma_z_effective = c->sigma_z_effective;
    s->mu_state = c->mu_state;
    s->mu_var = c->mu_var;
    s->guide_mean_fast = (float)c->guide_mean_fast;
    s->guide_mean_slow = (float)c->guide_mean_slow;
    s->guide_var_fast = (float)c->guide_var_fast;
    s->guide_var_slow = (float)c->guide_var_slow;
    s->guide_2f_initialized = c->guide_2f_initialized;
    for (int i = 0; i < SVPF_SMOOTH_MAX_LAG; ++i) {
        s->smooth_h_mean[i] = c->smooth_h_mean[i];
        s->smooth_h_var[i] = c->smooth_h_var[i];
        s->smooth_y[i] = c->smooth_y[i];
    }
}

void ctl_fresh(svpf_ctl_t* c) {
    std::memset(c, 0, sizeof(*c));
    c->ksd_prev = 1e10f;
    c->ksd_last = 0.0f;
    c->vol_prev = 0.05f;
    c->h_mean_prev = -3.5f;   // backend initial value (svpf_optimized_graph.cu:492-494)
    c->sigma_z_effective = 0.10f;
    c->mu_state = -3.5f;
    c->mu_var = 1.0f;
    for (int i = 0; i < SVPF_SMOOTH_MAX_LAG; ++i) c->smooth_h_var[i] = 1.0f;
}

int set_err(SVPFState* s, int code) {
    Impl* im = impl_of(s);
    if (im) im->err = code;
    return code;
}

bool grow(float** p, size_t* cap, size_t bytes) {
    if (bytes <= *cap) return true;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    if (cudaMalloc(p, bytes) != cudaSuccess) return false;
    *cap = bytes;
    return true;
}

int pick_cluster(const SVPFState* s, const Impl* im) {
    int C = im->cluster > 0 ? im->cluster : default_cluster(s->n_particles);
    while (C > 1 && tick_smem_bytes_single(s->n_particles, C, s->use_heun != 0) > max_dyn_smem()) C >>= 1;
    return C;
}

// Two-factor: the smallest cluster at least the default whose shared memory
// fits (every member holds both factors' positions); 0 if none does.
int pick_cluster_2f(const SVPFState* s, const Impl* im) {
    int C = im->cluster > 0 ? im->cluster : default_cluster(s->n_particles);
    while (C <= 16 && tick_smem_bytes_2f(s->n_particles, C) > max_dyn_smem()) C <<= 1;   // 16: largest cluster
    return C <= 16 ? C : 0;
}

// Wait for the step launched last: poll its host-mapped completion word for up
// to 2 ms (a blocking step's result is then read without a stream
// synchronisation), else synchronise the stream, which also reports a failed
// launch.  The kernel's other CTAs may still be retiring when the word
// arrives: every host function below that touches the filter's device arrays
// outside the stream synchronises it first (quiesce).
cudaError_t wait_done(Impl* im, cudaStream_t stream) {
    const volatile unsigned int* w = im->done;
    const unsigned int want = im->seq;
    const auto t0 = std::chrono::steady_clock::now();
    for (unsigned int k = 1;; ++k) {
        if (*w == want) {
            std::atomic_thread_fence(std::memory_order_acquire);   // the records written before the word
            return cudaSuccess;
        }
        if ((k & 1023u) == 0u && std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(2)) break;
    }
    return cudaStreamSynchronize(stream);
}

void quiesce(const SVPFState* s) {
    if (s->stream) cudaStreamSynchronize(s->stream);
    else cudaDeviceSynchronize();
}

void step_impl(SVPFState* s, float y_t, float y_prev, const SVPFParams* params,
               unsigned long long seed, float* ll, float* vol, float* hm) {
    Impl* im = impl_of(s);
    if (!s || !im || !params) {
        if (s) set_err(s, SVPF_ERR_INVALID_ARG);
        return;
    }
    const bool tf = s->use_two_factor != 0;
    if (tf && s->n_stein_steps < 1) {
        set_err(s, SVPF_ERR_INVALID_ARG);
        return;
    }
    SingleArgs a;
    std::memset(&a, 0, sizeof(a));
    config_from_state(s, &a.cfg);
    if (!config_loops_ok(a.cfg)) {
        set_err(s, SVPF_ERR_INVALID_ARG);
        return;
    }
    a.prm = *params;
    ctl_gather(s, im, &a.ctl);
    a.y_t = y_t;
    a.y_prev = y_prev;
    a.h = tf ? im->h2 : s->h;
    a.hp = tf ? im->hp2 : s->h_prev;
    a.v = tf ? im->v2 : s->d_grad_v;
    a.lw = s->log_weights;
    a.n = s->n_particles;
    a.seed = seed;
    if (im->tape_on) {
        a.tape_n = im->tape_n;
        a.tape_u = im->tape_u;
        a.slots_n = im->slots_n;
        a.slots_u = im->slots_u;
    }
    a.ctl_out = im->dev_res_ctl;
    a.out = im->dev_res_out;
    a.done = im->dev_done;
    a.seq = ++im->seq;
    // per-tick constants of the single-factor plan, on the host (svpf_optimized_graph.cu:951-953;
    // the EKF observation log y^2, include/svpf_kernels.cuh:509-541)
    a.host_consts = 1;
    a.stc = lgammaf((s->nu + 1.0f) * 0.5f) - lgammaf(s->nu * 0.5f) - 0.5f * logf(3.14159265358979f * s->nu);
    a.log_y2 = std::log((double)y_t * (double)y_t + 1e-8);
    const int C = tf ? pick_cluster_2f(s, im) : pick_cluster(s, im);
    if (C < 1) {
        set_err(s, SVPF_ERR_UNSUPPORTED);
        return;
    }
    const int tile = im->tile >= 0 ? im->tile : default_single_tile(s->n_particles, C);
    cudaError_t e = tf ? launch_single_2f(a, C, tile, s->stream) : launch_single(a, C, tile, s->stream);
    if (e == cudaSuccess) e = wait_done(im, s->stream);
    if (e != cudaSuccess) {
        set_err(s, SVPF_ERR_CUDA);
        return;
    }
    ++im->launches;
    svpf_ctl_t c = *im->res_ctl;
    im->last = *im->res_out;
    ctl_scatter(&c, s, im);
    im->err = c.status;
    if (ll) *ll = im->last.loglik;
    if (vol) *vol = im->last.vol;
    if (hm) *hm = im->last.h_mean;
}

}  // namespace

extern "C" {

SVPFState* svpf_create(int n_particles, int n_stein_steps, float nu, cudaStream_t stream) {
    SVPF_TRACE();
    if (n_particles < 1 || n_particles > SVPF_MAX_PARTICLES) return nullptr;
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count < 1) return nullptr;
    SVPFState* s = (SVPFState*)std::calloc(1, sizeof(SVPFState));
    if (!s) return nullptr;
    Impl* im = new Impl();
    s->impl = im;
    s->n_particles = n_particles;
    s->stream = stream;
    set_defaults(s, n_stein_steps, nu);
    ctl_fresh(&im->cache);
    const size_t bytes = (size_t)n_particles * sizeof(float);
    bool ok = cudaMalloc(&s->h, bytes) == cudaSuccess && cudaMalloc(&s->h_prev, bytes) == cudaSuccess &&
              cudaMalloc(&s->log_weights, bytes) == cudaSuccess && cudaMalloc(&s->d_grad_v, bytes) == cudaSuccess;
    ok = ok && cudaMalloc(&im->h2, 2 * bytes) == cudaSuccess && cudaMalloc(&im->hp2, 2 * bytes) == cudaSuccess &&
         cudaMalloc(&im->v2, 2 * bytes) == cudaSuccess;
    ok = ok && cudaHostAlloc(&im->res_ctl, sizeof(svpf_ctl_t), cudaHostAllocMapped) == cudaSuccess &&
         cudaHostAlloc(&im->res_out, sizeof(svpf_out_t), cudaHostAllocMapped) == cudaSuccess;
    ok = ok && cudaHostGetDevicePointer((void**)&im->dev_res_ctl, im->res_ctl, 0) == cudaSuccess &&
         cudaHostGetDevicePointer((void**)&im->dev_res_out, im->res_out, 0) == cudaSuccess;
    ok = ok && cudaHostAlloc(&im->done, sizeof(unsigned int), cudaHostAllocMapped) == cudaSuccess &&
         cudaHostGetDevicePointer((void**)&im->dev_done, im->done, 0) == cudaSuccess;
    if (ok) *im->done = 0;
    if (ok) {
        ok = cudaMemset(s->h, 0, bytes) == cudaSuccess && cudaMemset(s->h_prev, 0, bytes) == cudaSuccess &&
             cudaMemset(s->log_weights, 0, bytes) == cudaSuccess && cudaMemset(s->d_grad_v, 0, bytes) == cudaSuccess &&
             cudaMemset(im->h2, 0, 2 * bytes) == cudaSuccess && cudaMemset(im->hp2, 0, 2 * bytes) == cudaSuccess &&
             cudaMemset(im->v2, 0, 2 * bytes) == cudaSuccess;
    }
    if (!ok) {
        svpf_destroy(s);
        return nullptr;
    }
    return s;
}

void svpf_destroy(SVPFState* s) {
    if (!s) return;
    Impl* im = impl_of(s);
    if (s->stream) cudaStreamSynchronize(s->stream);
    else cudaDeviceSynchronize();
    cudaFree(s->h);
    cudaFree(s->h_prev);
    cudaFree(s->log_weights);
    cudaFree(s->d_grad_v);
    if (im) {
        if (im->res_ctl) cudaFreeHost(im->res_ctl);
        if (im->res_out) cudaFreeHost(im->res_out);
        if (im->done) cudaFreeHost(im->done);
        if (im->tape_n) cudaFree(im->tape_n);
        if (im->tape_u) cudaFree(im->tape_u);
        cudaFree(im->h2);
        cudaFree(im->hp2);
        cudaFree(im->v2);
        delete im;
    }
    std::free(s);
}

// svpf_initialize (svpf_optimized_graph.cu:349-451)
void svpf_initialize(SVPFState* s, const SVPFParams* p, unsigned long long seed) {
    SVPF_TRACE();
    Impl* im = impl_of(s);
    if (!s || !im || !p) {
        if (s) set_err(s, SVPF_ERR_INVALID_ARG);
        return;
    }
    quiesce(s);
    s->timestep = 0;
    s->y_prev = 0.0f;
    s->nu_state = fmaxf(s->nu_state, 2.5f);
    const float base_var = p->sigma_z * p->sigma_z / (1.0f - p->rho * p->rho + 1e-6f);
    const float var = s->use_student_t_state ? s->nu_state / (s->nu_state - 2.0f) * base_var : base_var;
    im->seed = seed;
    InitArgs a;
    std::memset(&a, 0, sizeof(a));
    a.h = s->h;
    a.hp = s->h_prev;
    a.v = s->d_grad_v;
    a.n0 = s->n_particles;
    a.F = 1;
    a.mu0 = p->mu;
    a.sd0 = sqrtf(var);
    a.seed = seed;
    a.tape0 = im->tape_on ? im->tape_n : nullptr;
    a.tape_stride = s->n_particles;
    const bool tf = s->use_two_factor != 0;
    if (tf && im->tape_on && im->slots_n < 3) {
        set_err(s, SVPF_ERR_TAPE_SHORT);
        return;
    }
    if (tf) {
        // svpf_optimized_graph.cu:414-447
        a.tf0 = 1;
        a.sdf0 = s->sigma_fast / sqrtf(1.0f - s->rho_fast * s->rho_fast + 1e-8f);
        a.sds0 = s->sigma_slow / sqrtf(1.0f - s->rho_slow * s->rho_slow + 1e-8f);
        a.h2 = im->h2;
        a.hp2 = im->hp2;
        a.v2 = im->v2;
    }
    cudaError_t e = launch_init(a, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (tf) {
        s->guide_2f_initialized = 0;
        s->guide_mean_fast = 0.0f;
        s->guide_mean_slow = 0.0f;
        s->guide_var_fast = s->sigma_fast * s->sigma_fast / (1.0f - s->rho_fast * s->rho_fast + 1e-6f);
        s->guide_var_slow = s->sigma_slow * s->sigma_slow / (1.0f - s->rho_slow * s->rho_slow + 1e-6f);
        im->cache.guide_mean_fast = s->guide_mean_fast;
        im->cache.guide_mean_slow = s->guide_mean_slow;
        im->cache.guide_var_fast = s->guide_var_fast;
        im->cache.guide_var_slow = s->guide_var_slow;
    }
    s->guide_initialized = 0;
    s->guide_mean = p->mu;
    s->guide_var = var;
    im->cache.guide_mean = p->mu;
    im->cache.guide_var = var;
    if (s->use_adaptive_mu) {
        s->mu_state = p->mu;
        s->mu_var = 1.0f;
    }
    if (s->use_adaptive_sigma) s->sigma_z_effective = p->sigma_z;
    s->ksd_prev = 1e10f;
    s->stein_steps_used = s->n_stein_steps;
    im->cache.loglik_sum = 0.0;
    im->err = e == cudaSuccess ? SVPF_OK : SVPF_ERR_CUDA;
}

void svpf_step_graph(SVPFState* s, float y_t, float y_prev, const SVPFParams* p, float* ll, float* vol,
                     float* hm) {
    SVPF_TRACE();
    Impl* im = impl_of(s);
    step_impl(s, y_t, y_prev, p, im ? im->seed : 0ull, ll, vol, hm);
}

void svpf_step_adaptive(SVPFState* s, float y_t, float y_prev, const SVPFParams* p, float* ll, float* vol,
                        float* hm) {
    SVPF_TRACE();
    svpf_step_graph(s, y_t, y_prev, p, ll, vol, hm);
}

void svpf_step_optimized(SVPFState* s, float y_t, float y_prev, const SVPFParams* p, float* ll, float* vol) {
    SVPF_TRACE();
    svpf_step_graph(s, y_t, y_prev, p, ll, vol, nullptr);
}

// svpf_step (svpf_optimized_graph.cu:1396-1407)
void svpf_step(SVPFState* s, float y_t, const SVPFParams* p, SVPFResult* r) {
    SVPF_TRACE();
    if (!s) return;
    float ll = 0.0f, vol = 0.0f, hm = 0.0f;
    svpf_step_graph(s, y_t, s->y_prev, p, &ll, &vol, &hm);
    if (r) {
        r->log_lik_increment = ll;
        r->vol_mean = vol;
        r->h_mean = hm;
        r->vol_std = 0.0f;
        r->mu_estimate = (s->use_adaptive_mu || !p) ? s->mu_state : p->mu;
    }
    if (std::isfinite(y_t)) s->y_prev = y_t;   // a refused observation is not the next tick's y_prev
}

void svpf_step_seeded(SVPFState* s, float y_t, const SVPFParams* p, unsigned long long rng_seed,
                      SVPFResult* r) {
    SVPF_TRACE();
    if (!s) return;
    float ll = 0.0f, vol = 0.0f, hm = 0.0f;
    step_impl(s, y_t, s->y_prev, p, rng_seed, &ll, &vol, &hm);
    if (r) {
        r->log_lik_increment = ll;
        r->vol_mean = vol;
        r->h_mean = hm;
        r->vol_std = 0.0f;
        r->mu_estimate = (s->use_adaptive_mu || !p) ? s->mu_state : p->mu;
    }
    if (std::isfinite(y_t)) s->y_prev = y_t;   // a refused observation is not the next tick's y_prev
}

void svpf_run_sequence(SVPFState* s, const float* obs, int T, const SVPFParams* p, float* ll_out,
                       float* vol_out) {
    SVPF_TRACE();
    if (!s || !obs || T < 0) {
        if (s) set_err(s, SVPF_ERR_INVALID_ARG);
        return;
    }
    float y_prev = 0.0f;
    for (int t = 0; t < T; ++t) {
        float ll, vol, hm;
        svpf_step_graph(s, obs[t], y_prev, p, &ll, &vol, &hm);
        if (ll_out) ll_out[t] = ll;
        if (vol_out) vol_out[t] = vol;
        if (std::isfinite(obs[t])) y_prev = obs[t];   // a refused observation is not the next y_prev
    }
}

void svpf_run_sequence_device(SVPFState* s, const float* d_obs, int T, const SVPFParams* p, float* d_ll,
                              float* d_vol) {
    SVPF_TRACE();
    if (!s || !d_obs || T < 0) {
        if (s) set_err(s, SVPF_ERR_INVALID_ARG);
        return;
    }
    std::vector<float> obs(T), ll(T), vol(T);
    quiesce(s);
    if (cudaMemcpy(obs.data(), d_obs, T * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_err(s, SVPF_ERR_CUDA);
        return;
    }
    svpf_run_sequence(s, obs.data(), T, p, ll.data(), vol.data());
    if ((d_ll && cudaMemcpy(d_ll, ll.data(), T * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) ||
        (d_vol && cudaMemcpy(d_vol, vol.data(), T * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess))
        set_err(s, SVPF_ERR_CUDA);
}

void svpf_get_particles(const SVPFState* s, float* h_out) {
    if (!s || !h_out) return;
    quiesce(s);
    // void, as the reference declares it: a failed copy is recorded for svpf_last_error
    if (cudaMemcpy(h_out, s->h, s->n_particles * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        set_err(const_cast<SVPFState*>(s), SVPF_ERR_CUDA);
}

void svpf_get_stats(const SVPFState* s, float* h_mean, float* h_std) {
    if (!s) return;
    const int n = s->n_particles;
    std::vector<float> h(n);
    quiesce(s);
    if (cudaMemcpy(h.data(), s->h, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_err(const_cast<SVPFState*>(s), SVPF_ERR_CUDA);
        if (h_mean) *h_mean = NAN;
        if (h_std) *h_std = NAN;
        return;
    }
    double sum = 0.0;
    for (float x : h) sum += x;
    const double m = sum / n;
    double sq = 0.0;
    for (float x : h) sq += (x - m) * (x - m);
    if (h_mean) *h_mean = (float)m;
    if (h_std) *h_std = (float)std::sqrt(sq / n);
}

float svpf_get_ess(const SVPFState* s) {
    if (!s) return 0.0f;
    const int n = s->n_particles;
    std::vector<float> lw(n);
    quiesce(s);
    if (cudaMemcpy(lw.data(), s->log_weights, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_err(const_cast<SVPFState*>(s), SVPF_ERR_CUDA);
        return 0.0f;
    }
    float mx = lw[0];
    for (float x : lw) mx = std::max(mx, x);
    double sw = 0.0, sw2 = 0.0;
    for (float x : lw) {
        const double w = std::exp((double)x - mx);
        sw += w;
        sw2 += w * w;
    }
    return (float)(sw * sw / (sw2 + 1e-10));
}

void svpf_get_ksd_stats(const SVPFState* s, float* ksd_out, int* steps_out) {
    if (!s) return;
    if (ksd_out) *ksd_out = s->ksd_prev;
    if (steps_out) *steps_out = s->stein_steps_used;
}

bool svpf_graph_is_captured(SVPFState* s) {
    const Impl* im = impl_of(s);
    return im && im->launches > 0;
}

void svpf_graph_invalidate(SVPFState* s) {
    Impl* im = impl_of(s);
    if (im) im->launches = 0;
}

void svpf_optimized_cleanup_state(SVPFState* s) { svpf_graph_invalidate(s); }

int svpf_last_error(const SVPFState* s) {
    const Impl* im = impl_of(s);
    return im ? im->err : SVPF_ERR_INVALID_ARG;
}

void svpf_config_init(svpf_config_t* cfg, int n_stein_steps, float nu) {
    if (!cfg) return;
    SVPFState tmp;
    std::memset(&tmp, 0, sizeof(tmp));
    set_defaults(&tmp, n_stein_steps, nu);
    config_from_state(&tmp, cfg);
}

void svpf_get_config(const SVPFState* s, svpf_config_t* c) {
    if (s && c) config_from_state(s, c);
}
void svpf_set_config(SVPFState* s, const svpf_config_t* c) {
    if (s && c) config_to_state(c, s);
}

int svpf_get_state(const SVPFState* s, svpf_ctl_t* ctl, float* h, float* hp, float* v, float* lw) {
    const Impl* im = impl_of(s);
    if (!s || !im) return SVPF_ERR_INVALID_ARG;
    if (s->stream) cudaStreamSynchronize(s->stream);
    const size_t b = (size_t)s->n_particles * sizeof(float);
    if (ctl) ctl_gather(s, im, ctl);
    if (h && cudaMemcpy(h, s->h, b, cudaMemcpyDeviceToHost) != cudaSuccess) return SVPF_ERR_CUDA;
    if (hp && cudaMemcpy(hp, s->h_prev, b, cudaMemcpyDeviceToHost) != cudaSuccess) return SVPF_ERR_CUDA;
    if (v && cudaMemcpy(v, s->d_grad_v, b, cudaMemcpyDeviceToHost) != cudaSuccess) return SVPF_ERR_CUDA;
    if (lw && cudaMemcpy(lw, s->log_weights, b, cudaMemcpyDeviceToHost) != cudaSuccess) return SVPF_ERR_CUDA;
    return SVPF_OK;
}

int svpf_set_state(SVPFState* s, const svpf_ctl_t* ctl, const float* h, const float* hp, const float* v,
                   const float* lw) {
    Impl* im = impl_of(s);
    if (!s || !im) return SVPF_ERR_INVALID_ARG;
    const size_t b = (size_t)s->n_particles * sizeof(float);
    quiesce(s);
    if (ctl) ctl_scatter(ctl, s, im);
    if (h && cudaMemcpy(s->h, h, b, cudaMemcpyHostToDevice) != cudaSuccess) return SVPF_ERR_CUDA;
    if (hp && cudaMemcpy(s->h_prev, hp, b, cudaMemcpyHostToDevice) != cudaSuccess) return SVPF_ERR_CUDA;
    if (v && cudaMemcpy(s->d_grad_v, v, b, cudaMemcpyHostToDevice) != cudaSuccess) return SVPF_ERR_CUDA;
    if (lw && cudaMemcpy(s->log_weights, lw, b, cudaMemcpyHostToDevice) != cudaSuccess) return SVPF_ERR_CUDA;
    return SVPF_OK;
}

int svpf_get_state_2f(const SVPFState* s, float* hf, float* hs, float* hfp, float* hsp, float* vf, float* vs) {
    const Impl* im = impl_of(s);
    if (!s || !im) return SVPF_ERR_INVALID_ARG;
    if (s->stream) cudaStreamSynchronize(s->stream);
    const size_t n = (size_t)s->n_particles, b = n * sizeof(float);
    const float* src[6] = {im->h2, im->h2 + n, im->hp2, im->hp2 + n, im->v2, im->v2 + n};
    float* dst[6] = {hf, hs, hfp, hsp, vf, vs};
    for (int k = 0; k < 6; ++k)
        if (dst[k] && cudaMemcpy(dst[k], src[k], b, cudaMemcpyDeviceToHost) != cudaSuccess) return SVPF_ERR_CUDA;
    return SVPF_OK;
}

int svpf_set_state_2f(SVPFState* s, const float* hf, const float* hs, const float* hfp, const float* hsp,
                      const float* vf, const float* vs) {
    Impl* im = impl_of(s);
    if (!s || !im) return SVPF_ERR_INVALID_ARG;
    const size_t n = (size_t)s->n_particles, b = n * sizeof(float);
    float* dst[6] = {im->h2, im->h2 + n, im->hp2, im->hp2 + n, im->v2, im->v2 + n};
    const float* src[6] = {hf, hs, hfp, hsp, vf, vs};
    quiesce(s);
    for (int k = 0; k < 6; ++k)
        if (src[k] && cudaMemcpy(dst[k], src[k], b, cudaMemcpyHostToDevice) != cudaSuccess) return SVPF_ERR_CUDA;
    return SVPF_OK;
}

int svpf_set_noise_tape(SVPFState* s, const float* normals, int ns, const float* uniforms, int nu_) {
    Impl* im = impl_of(s);
    if (!s || !im) return SVPF_ERR_INVALID_ARG;
    if (!normals) {
        im->tape_on = false;
        return SVPF_OK;
    }
    if (ns < 1 || nu_ < 0 || (nu_ > 0 && !uniforms)) return set_err(s, SVPF_ERR_INVALID_ARG);
    quiesce(s);
    const size_t n = (size_t)s->n_particles;
    if (!grow(&im->tape_n, &im->cap_n, ns * n * sizeof(float)) ||
        !grow(&im->tape_u, &im->cap_u, std::max(nu_, 1) * n * sizeof(float)))
        return set_err(s, SVPF_ERR_CUDA);
    if (cudaMemcpy(im->tape_n, normals, ns * n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return set_err(s, SVPF_ERR_CUDA);
    if (nu_ > 0 && cudaMemcpy(im->tape_u, uniforms, nu_ * n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return set_err(s, SVPF_ERR_CUDA);
    im->slots_n = ns;
    im->slots_u = nu_;
    im->tape_on = true;
    return SVPF_OK;
}

int svpf_get_last_output(const SVPFState* s, svpf_out_t* out) {
    const Impl* im = impl_of(s);
    if (!im || !out) return SVPF_ERR_INVALID_ARG;
    *out = im->last;
    return SVPF_OK;
}

int svpf_set_cluster_size(SVPFState* s, int C) {
    Impl* im = impl_of(s);
    if (!im || C < 0 || C > 16 || (C & (C - 1)) != 0) return SVPF_ERR_INVALID_ARG;
    im->cluster = C;
    return SVPF_OK;
}

int svpf_debug_philox(uint32_t k0, uint32_t k1, const uint32_t* ctr4, uint32_t* out4, int count) {
    if (count <= 0 || !ctr4 || !out4) return SVPF_ERR_INVALID_ARG;
    uint32_t *dc = nullptr, *dout = nullptr;
    const size_t b = (size_t)count * 4 * sizeof(uint32_t);
    if (cudaMalloc(&dc, b) != cudaSuccess) return SVPF_ERR_CUDA;
    if (cudaMalloc(&dout, b) != cudaSuccess) {
        cudaFree(dc);
        return SVPF_ERR_CUDA;
    }
    cudaError_t e = cudaMemcpy(dc, ctr4, b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = debug_philox(k0, k1, dc, dout, count);
    if (e == cudaSuccess) e = cudaMemcpy(out4, dout, b, cudaMemcpyDeviceToHost);
    cudaFree(dc);
    cudaFree(dout);
    return e == cudaSuccess ? SVPF_OK : SVPF_ERR_CUDA;
}

const char* svpf_build_info(void) {
    return "svpf_b200: sm_100a; single-filter tick = 1 cluster launch (<=16 CTAs, DSMEM); "
           "batch tick = 1 persistent launch; particles resident in shared memory";
}

}  // extern "C"
