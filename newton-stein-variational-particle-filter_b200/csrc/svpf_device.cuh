// svpf_device.cuh -- device side of the B200 SVPF step engine.
//
// One SVPF tick of one filter is executed by a "team": one CTA (batch engine)
// or a thread-block cluster of C CTAs (low-latency single-filter kernel).
// All particle data of a tick live in shared memory:
//
//   h[2][N]   particle positions, double buffered (Jacobi transport: every row
//             reads the pre-iteration positions; the reference updates in place
//             and races across blocks, svpf_opt_kernels.cu:545-598)
//   g[N]      transport score (raw gradient, or the Newton-preconditioned one)
//   c[N]      curvature (full Newton) or its reciprocal (plain Newton)
//   mu[M]     prior means mu_k = mu + rho (h_prev,k - mu) + leverage_k, sorted
//             once per tick; M >= N padded with a far value
//   v[L]      RMSProp second moment of the team member's own rows
//
// Rows (particles) are split across the team; within a CTA a tile <R, S>
// gives each thread R rows and 1/S of the columns (S lanes of a warp share a
// row and combine their partial sums with shuffles).  After the gradient pass
// g/c are all-gathered across the cluster through distributed shared memory,
// after the transport pass the new h is; every exchange is followed by one
// cluster barrier.  There are no spin waits anywhere.
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "svpf.h"

namespace svpf {
namespace cg = cooperative_groups;

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr float kMuPad = 1e18f;   // sorted-prior pad: exp weight is exactly 0, products stay finite
constexpr float kHPad = 1e15f;    // particle pad column: K ~ 1e-34, K^2 flushes to 0, no inf/NaN
constexpr float kHPadRaw = 1e12f; // the same in log-volatility units: |u| <= 1e12 / bw stays far below
                                  // sqrt(FLT_MAX) for any bandwidth the floors allow
constexpr int kMaxCluster = 16;

// ---------------------------------------------------------------------------
// Hardware approximations, as PTX instructions.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float ex2_approx(float x) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float lg2_approx(float x) {
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
// Packed FP32x2 arithmetic (sm_100): one issue slot for two FP32 results.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

constexpr float kLog2e = 1.4426950408889634f;
constexpr float kLn2 = 0.6931471805599453f;

__device__ __forceinline__ float clamp_h(float h) { return fminf(fmaxf(h, SVPF_H_MIN), SVPF_H_MAX); }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

// ---------------------------------------------------------------------------
// Counter-based RNG: Philox4x32-10 (Salmon et al., SC'11), written from the
// paper's round function.  key = (seed_lo, seed_hi + 0x9E3779B9 * filter),
// counter = (particle, draw index, tick, stream); stream 0 normals, 1
// uniforms, 2 the initial draw.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox10(uint2 key, uint4 c) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ key.x, lo1, hi0 ^ c.w ^ key.y, lo0);
        key.x += 0x9E3779B9u;
        key.y += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ uint2 philox_key(unsigned long long seed, int filter) {
    return make_uint2((uint32_t)seed, (uint32_t)(seed >> 32) + 0x9E3779B9u * (uint32_t)filter);
}

// Box-Muller on 24-bit uniforms: u1 in (0,1], u2 in [0,1).
__device__ __forceinline__ float normal_from_bits(uint32_t a, uint32_t b) {
    const float u1 = (float)((a >> 8) + 1u) * (1.0f / 16777216.0f);
    const float u2 = (float)(b >> 8) * (1.0f / 16777216.0f);
    return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}
__device__ __forceinline__ float uniform_from_bits(uint32_t a) {
    return (float)((a >> 8) + 1u) * (1.0f / 16777216.0f);
}

// Noise of one filter for one tick: Philox, or a pre-drawn tape (test mode).
struct Noise {
    uint2 key;
    uint32_t tick;
    const float* tape_n;   // [slots_n][n] or nullptr
    const float* tape_u;   // [slots_u][n]
    int slots_n, slots_u, stride;
    int* flag;             // shared flag: set to SVPF_ERR_TAPE_SHORT on overrun

    __device__ __forceinline__ float normal(int i, int k) const {
        if (tape_n != nullptr) {
            if (k >= slots_n) { *flag = SVPF_ERR_TAPE_SHORT; return 0.0f; }
            return tape_n[(size_t)k * stride + i];
        }
        const uint4 r = philox10(key, make_uint4((uint32_t)i, (uint32_t)k, tick, 0u));
        return normal_from_bits(r.x, r.y);
    }
    __device__ __forceinline__ float uniform(int i, int k) const {
        if (tape_u != nullptr) {
            if (k >= slots_u) { *flag = SVPF_ERR_TAPE_SHORT; return 1.0f; }
            return tape_u[(size_t)k * stride + i];
        }
        const uint4 r = philox10(key, make_uint4((uint32_t)i, (uint32_t)k, tick, 1u));
        return uniform_from_bits(r.x);
    }
};

// Transport coordinates and step of one factor of the two-factor tick (the
// single-factor tick keeps the same fields in its Plan).
struct FactorPlan {
    float eps_step, temp;
    float bw, inv_bw, inv_bw2;
    float center;
};

// ---------------------------------------------------------------------------
// Tick plan: every scalar decision of a tick, made by one thread before the
// particle phases (the reference makes them on the host between launches,
// svpf_optimized_graph.cu:933-1138, 1328-1341).
// ---------------------------------------------------------------------------
struct Plan {
    float mu_eff, sz_eff, stc, off;
    float rho_up, rho_dn, drho, dsig;
    float gs, guide_mean, gstd;
    float eps_step, temp;
    float y_t, y_prev;
    float bw, inv_bw, inv_bw2;
    float center;          // transport coordinates: hs = (h - center) / bw during the Stein loop
    float mu_center;       // prior coordinates: (h - mu_center) * prior_scale, in log2 units
    float prior_scale;     // sqrt(log2(e) / (2 sigma^2))
    float beta[SVPF_MAX_ANNEAL_STEPS];
    int budget, na, si_base;
    int rejuv;
    int kn_pred;
    int uses_uniform_predict;
    int transport;         // 0 vanilla, 1 Newton, 2 full Newton
    int fan;
    int flag;              // tape overrun etc.
    int have_consts;       // stc / log_y2 set by the launcher (single-filter tick)
    double log_y2;
    FactorPlan fac[2];     // two-factor: fast, slow
    float fmean[2];        // two-factor: factor means of the previous tick (guide)
    float gmean2[2];       // two-factor: EKF guide means
    float red[4][kWarps];  // block reduction scratch
    float ksd_slot[kMaxCluster];
};

// Adaptive beta (svpf_optimized_graph.cu:1066-1092).
__device__ __forceinline__ float adaptive_beta(float ksd_prev, int ai, int na) {
    if (ai == na - 1) return 1.0f;
    float b;
    if (ksd_prev > 0.50f) b = 0.30f;
    else if (ksd_prev < 0.05f) b = 0.80f;
    else b = 0.30f + (0.50f - ksd_prev) / (0.50f - 0.05f) * (0.80f - 0.30f);
    b *= 0.5f + 0.5f * ((float)(ai + 1) / (float)na);
    return clampf(b, 0.1f, 1.0f);
}

// Scalar control of a tick; writes the updated EKF/sigma fields into ctl.
// pl.have_consts: pl.stc and pl.log_y2 were filled by the caller (the
// single-filter launcher computes them on the host), else they are computed here.
__device__ inline void make_plan(const svpf_config_t& c, const SVPFParams& p, svpf_ctl_t& s,
                          float y_t, float y_prev, Plan& pl) {
    const int t = s.timestep;
    pl.y_t = y_t;
    pl.y_prev = y_prev;
    // effective parameters (:933-948)
    pl.mu_eff = c.use_adaptive_mu ? s.mu_state : p.mu;
    pl.sz_eff = p.sigma_z;
    if (c.use_adaptive_sigma && t > 0) {
        const float ve = fmaxf(s.vol_prev, 1e-4f);
        const float z = fabsf(y_t) / ve;
        float boost = 1.0f;
        if (z > c.sigma_boost_threshold) {
            const float sev = fminf((z - c.sigma_boost_threshold) / 3.0f, 1.0f);
            boost = 1.0f + (c.sigma_boost_max - 1.0f) * sev;
        }
        pl.sz_eff = p.sigma_z * boost;
        s.sigma_z_effective = pl.sz_eff;
    }
    // Student-t normaliser (:951-953) and the create-time implied offset
    if (!pl.have_consts)
        pl.stc = lgammaf((c.nu + 1.0f) * 0.5f) - lgammaf(c.nu * 0.5f) - 0.5f * logf(3.14159265358979f * c.nu);
    pl.off = c.student_t_implied_offset;
    pl.rho_up = c.use_asymmetric_rho ? c.rho_up : p.rho;
    pl.rho_dn = c.use_asymmetric_rho ? c.rho_down : p.rho;
    pl.drho = c.use_local_params ? c.delta_rho : 0.0f;
    pl.dsig = c.use_local_params ? c.delta_sigma : 0.0f;
    // adaptive guide strength (:1006-1021)
    pl.gs = c.guide_strength_base;
    if (c.use_guide && c.use_adaptive_guide && t > 0) {
        const float ve = fmaxf(s.vol_prev, 1e-4f);
        const float z = fabsf(y_t) / ve;
        const float ih = logf(y_t * y_t + 1e-8f) + pl.off;
        const float he = logf(ve * ve + 1e-8f);
        if (ih - he > 0.0f && z > c.guide_innovation_threshold) {
            const float sev = fminf((z - c.guide_innovation_threshold) / 3.0f, 1.0f);
            pl.gs = c.guide_strength_base + (c.guide_strength_max - c.guide_strength_base) * sev;
        }
    }
    // EKF guide on log y^2 (include/svpf_kernels.cuh:509-541), FP64 recursion
    if (c.use_guide) {
        const double mu = (double)pl.mu_eff, rho = (double)p.rho, sz = (double)p.sigma_z;
        double m = s.guide_mean, P = s.guide_var;
        if (!s.guide_initialized) {
            m = mu;
            P = sz * sz / (1.0 - rho * rho);
            s.guide_initialized = 1;
        }
        const double m_pred = mu + rho * (m - mu);
        const double P_pred = rho * rho * P + sz * sz;
        const double log_y2 = pl.have_consts ? pl.log_y2 : log((double)y_t * (double)y_t + 1e-8);
        const double S = P_pred + (4.93 + 2.0);
        const double K = P_pred / (S + 1e-8);
        s.guide_mean = m_pred + K * (log_y2 - (m_pred - (double)pl.off));
        s.guide_var = (1.0 - K) * P_pred;
        s.guide_K = K;
    }
    pl.guide_mean = (float)s.guide_mean;
    pl.gstd = sqrtf(fmaxf((float)s.guide_var, 1e-6f));
    // Stein budget from the previous tick's KSD (:1096-1112), split over stages
    const int na = c.use_annealing ? max(min(c.n_anneal_steps, SVPF_MAX_ANNEAL_STEPS), 1) : 1;
    int budget;
    if (t < 10) {
        budget = c.stein_max_steps;
    } else {
        float kn = (s.ksd_prev - 0.05f) / (0.50f - 0.05f);
        kn = fminf(fmaxf(kn, 0.0f), 1.0f);
        budget = c.stein_min_steps + (int)(kn * (float)(c.stein_max_steps - c.stein_min_steps));
    }
    pl.budget = max(budget, 0);
    pl.na = na;
    pl.si_base = pl.budget / na;
    for (int ai = 0; ai < na; ++ai) {
        float beta;
        if (!c.use_annealing) beta = 1.0f;
        else if (c.use_adaptive_beta) beta = adaptive_beta(s.ksd_prev, ai, na);
        else beta = (ai % 3 == 0) ? 0.30f : (ai % 3 == 1) ? 0.65f : 1.0f;
        pl.beta[ai] = beta;
    }
    pl.eps_step = SVPF_STEIN_STEP_SIZE * (c.use_guide ? 0.5f : 1.0f);
    pl.temp = c.use_svld ? c.temperature : 0.0f;
    pl.rejuv = (c.use_rejuvenation && c.use_guide && t > 10 && s.ksd_prev > c.rejuv_ksd_threshold) ? 1 : 0;
    // draws consumed by predict (svpf_opt_kernels.cu:31-53, 187-193)
    if (c.use_student_t_state && c.nu_state <= 30.0f) {
        const int nu_int = max((int)(c.nu_state + 0.5f), 3);
        pl.kn_pred = 1 + nu_int;
    } else {
        pl.kn_pred = 1;
    }
    pl.uses_uniform_predict = (c.use_mim || c.use_guided) ? 1 : 0;
    pl.transport = c.use_newton ? (c.use_full_newton ? 2 : 1) : 0;
    pl.fan = c.use_fan_mode;
}

// Stage of Stein iteration `it` and its beta (budget split :1136-1138).
__device__ __forceinline__ int stage_of(const Plan& pl, int it) {
    if (pl.si_base == 0) return pl.na - 1;
    const int a = it / pl.si_base;
    return a < pl.na - 1 ? a : pl.na - 1;
}

// ---------------------------------------------------------------------------
// Team: one CTA or one cluster.
// ---------------------------------------------------------------------------
struct Team {
    int rank, size;
    __device__ __forceinline__ void sync() const {
        if (size == 1) __syncthreads();
        else cg::this_cluster().sync();
    }
    template <class T>
    __device__ __forceinline__ T* at(T* local, int r) const {
        if (size == 1) return local;
        return cg::this_cluster().map_shared_rank(local, r);
    }
};

// ---------------------------------------------------------------------------
// Block reductions (kThreads threads).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Reduce up to four values (op per slot: 0 sum, 1 max, 2 min); result visible
// to all threads.  Contains two __syncthreads.
template <int K>
__device__ __forceinline__ void block_reduce(float (&v)[K], const int (&op)[K], Plan& pl) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        v[k] = op[k] == 0 ? warp_sum(v[k]) : op[k] == 1 ? warp_max(v[k]) : warp_min(v[k]);
        if (lane == 0) pl.red[k][w] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        float a = pl.red[k][0];
        for (int i = 1; i < kWarps; ++i) {
            const float b = pl.red[k][i];
            a = op[k] == 0 ? a + b : op[k] == 1 ? fmaxf(a, b) : fminf(a, b);
        }
        v[k] = a;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Bitonic sort of m[0..P) ascending (P a power of two), whole CTA.
// ---------------------------------------------------------------------------
__device__ inline void bitonic_sort(float* m, int P) {
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P; i += kThreads) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const float a = m[i], b = m[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) { m[i] = b; m[ixj] = a; }
                }
            }
            __syncthreads();
        }
    }
}

// Largest log-responsibility of row value x: attained at the nearest prior
// mean, found by binary search in the sorted means (the reference scans all N,
// svpf_opt_kernels.cu:453-459; the value is the same).
// Scaled Gaussian prior: the smallest squared distance from x to the sorted,
// scaled prior means (its negative is the row maximum of the exponent).
__device__ __forceinline__ float nearest_d2(const float* m, int n, float x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (m[mid] < x) lo = mid + 1; else hi = mid;
    }
    float best = 3.0e38f;
    if (lo < n) { const float d = x - m[lo]; best = fminf(best, d * d); }
    if (lo > 0) { const float d = x - m[lo - 1]; best = fminf(best, d * d); }
    return best;
}
__device__ __forceinline__ float nearest_lmax_student(const float* m, int n, float x, float inv_nus2,
                                                      float half_np1) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (m[mid] < x) lo = mid + 1; else hi = mid;
    }
    float best = -1e10f;
    if (lo < n) { const float d = x - m[lo]; best = fmaxf(best, -half_np1 * kLn2 * lg2_approx(1.0f + d * d * inv_nus2)); }
    if (lo > 0) { const float d = x - m[lo - 1]; best = fmaxf(best, -half_np1 * kLn2 * lg2_approx(1.0f + d * d * inv_nus2)); }
    return best;
}

// ---------------------------------------------------------------------------
// Shared-memory view of one tick.
// ---------------------------------------------------------------------------
struct Smem {
    float* h[2];
    float* g;
    float* c;
    float* mu;
    float* v;
    float* phi0;        // Heun: operator at the start point, own rows
    float* phi1;        // Heun: operator at the predicted point, own rows
    float* pre;         // SVLD normals of own rows drawn before the Stein loop, [kPreIters][Lp], or nullptr
    int n, np, m_len, p2;   // particles, padded row length, padded prior length, sort length
    int row0, row1;     // rows owned by this team member
    int Lp;             // own rows, padded to 4
};

__host__ __device__ inline int pow2_at_least(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}
__host__ __device__ inline int round_up(int a, int b) { return (a + b - 1) / b * b; }

// Floats of dynamic shared memory for N particles on a team of C CTAs; the two
// Heun operator buffers are present only when `heun`.
__host__ __device__ inline int smem_floats(int n, int C, bool heun) {
    const int np = round_up(n, 64);
    const int p2 = pow2_at_least(n);
    const int m_len = round_up(p2 > np ? p2 : np, 64);
    const int L = round_up((n + C - 1) / C, 4);
    return 2 * np + np + np + m_len + (heun ? 3 : 1) * L;
}

// Latency kernel: the SVLD normals of the first kPreIters Stein iterations of
// a member's own rows are drawn in parallel before the loop (each is a
// Philox block and a Box-Muller on the row's epilogue path otherwise), when
// the member owns at most kPreMaxRows rows.
constexpr int kPreIters = 16;
constexpr int kPreMaxRows = 256;
__host__ __device__ inline int pre_floats(int n, int C) {
    const int L = (n + C - 1) / C;
    return L <= kPreMaxRows ? kPreIters * round_up(L, 4) : 0;
}

// Two-factor tick: per factor x[2][np] (transport coordinates, double
// buffered), g[np], prev[np] (positions at tick start), v[L] of own rows.
__host__ __device__ inline int smem_floats_2f(int n, int C) {
    const int np = round_up(n, 64);
    const int L = round_up((n + C - 1) / C, 4);
    return 2 * (4 * np + L);
}

struct Smem2 {
    Smem f[2];          // per-factor views for transport_pass (c, mu unused)
    float* prev[2];     // positions at tick start, all n
};

__device__ inline Smem2 carve_2f(float* base, int n, int C, int rank) {
    Smem2 s;
    const int np = round_up(n, 64);
    const int L = (n + C - 1) / C;
    const int Lp = round_up(L, 4);
    for (int k = 0; k < 2; ++k) {
        float* b = base + k * (4 * np + Lp);
        Smem& f = s.f[k];
        f.h[0] = b;
        f.h[1] = b + np;
        f.g = b + 2 * np;
        s.prev[k] = b + 3 * np;
        f.v = b + 4 * np;
        f.c = nullptr;
        f.mu = nullptr;
        f.phi0 = f.phi1 = nullptr;
        f.pre = nullptr;
        f.Lp = Lp;
        f.n = n;
        f.np = np;
        f.m_len = 0;
        f.p2 = 0;
        f.row0 = min(rank * L, n);
        f.row1 = min(f.row0 + L, n);
    }
    return s;
}

__device__ inline Smem carve(float* base, int n, int C, int rank, bool heun) {
    Smem s;
    const int np = round_up(n, 64);
    s.n = n;
    s.p2 = pow2_at_least(n);
    s.m_len = round_up(s.p2 > np ? s.p2 : np, 64);
    s.h[0] = base;
    s.h[1] = base + np;
    s.g = base + 2 * np;
    s.c = base + 3 * np;
    s.mu = base + 4 * np;
    s.np = np;
    const int L = (n + C - 1) / C;
    const int Lp = round_up(L, 4);
    s.v = s.mu + s.m_len;
    s.phi0 = heun ? s.v + Lp : nullptr;
    s.phi1 = heun ? s.phi0 + Lp : nullptr;
    s.pre = nullptr;
    s.Lp = Lp;
    s.row0 = min(rank * L, n);
    s.row1 = min(s.row0 + L, n);
    return s;
}

// ---------------------------------------------------------------------------
// Gradient pass (svpf_fused_gradient_kernel, svpf_opt_kernels.cu:354-521) for
// the team member's rows.  Mixture prior over all N prior means in one exp per
// pair, likelihood, beta-combine and clamp, curvature.  Writes g/c on every
// team member and the log-weights to global memory.  The row maximum of the
// mixture's log-responsibilities (the reference scans all N twice,
// :453-459) comes either from the nearest of the means sorted once per tick
// (binary search; the throughput kernel, where the sort is amortised over a
// large filter) or, with SCAN, from a branch-free min pass over the unsorted
// means before the sum pass (the latency kernel: no sort, whose ~log2(N)^2/2
// block barriers cost more than the extra pass at N <= 1024 on a cluster).
// ---------------------------------------------------------------------------
// Column chunks per sweep unrolled in the cluster kernels (one warp pair per
// scheduler: four chunks' loads in flight).  The batch kernel, at its register
// limit, leaves the unrolling to the compiler.
constexpr int kClusterUnroll = 4;

// The column-chunk loop of the pair sweeps: cb = c0, c0 + step, ... < nv.
// U > 0 unrolls it U times; U = 0 leaves the unrolling to the compiler.
template <int U, class F>
__device__ __forceinline__ void chunk_loop(int c0, int nv, int step, F&& body) {
    if constexpr (U > 0) {
#pragma unroll U
        for (int cb = c0; cb < nv; cb += step) body(cb);
    } else {
        for (int cb = c0; cb < nv; cb += step) body(cb);
    }
}

// Pushes each row's values from lane 0 of its S lanes into every team
// member: the row's lanes take the members in turn (lane q: members q, q + S,
// ...), so that the remote stores of a row go out in parallel.  TWO: a second
// array b with values vb.  Every lane of the warp calls it.
template <int R, int S, bool TWO>
__device__ __forceinline__ void push_rows(float* a, float* b, const float (&va)[R], const float (&vb)[R],
                                          const int (&jl)[R], int nloc, int row0, int q, const Team& team) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const float x = S > 1 ? __shfl_sync(0xffffffffu, va[r], 0, S) : va[r];
        float y = 0.0f;
        if (TWO) y = S > 1 ? __shfl_sync(0xffffffffu, vb[r], 0, S) : vb[r];
        if (jl[r] >= nloc) continue;
        const int j = row0 + jl[r];
        for (int rk = q; rk < team.size; rk += S) {
            team.at(a, rk)[j] = x;
            if (TWO) team.at(b, rk)[j] = y;
        }
    }
}

template <int R, int S, bool STUDENT, bool SCAN = false, int U = 0>
__device__ void grad_pass(const Smem& sm, int cur, const Plan& pl, const svpf_config_t& cfg,
                          float beta, float* __restrict__ lw_out, const Team& team) {
    // Positions arrive in transport coordinates hs = (h - center) / bw.  The
    // Gaussian prior runs in scaled prior coordinates x = (h - mu_center) * sc
    // with sc^2 = log2(e) / (2 sigma^2), where the log-responsibility in base 2
    // is -(x - m)^2 and the sorted means m are stored scaled the same way; the
    // pair then costs one FADD, one FFMA, one ex2 and two accumulations.
    constexpr int G = kThreads / S;
    const int grp = threadIdx.x / S, q = threadIdx.x % S;
    const float* __restrict__ hc = sm.h[cur];
    const float* __restrict__ mu = sm.mu;
    const int nloc = sm.row1 - sm.row0;
    const int nv = round_up(sm.n, 4 * S);
    const float s2 = pl.sz_eff * pl.sz_eff;
    const float inv_s2 = 1.0f / s2;
    const float sc = pl.prior_scale;
    const float nu = cfg.nu;
    // Student-t prior constants (:406-447)
    const float nus2 = cfg.nu_state * s2, inv_nus2 = 1.0f / nus2, np1 = cfg.nu_state + 1.0f;
    const float half_np1 = 0.5f * np1;

    for (int base = 0; base < nloc; base += G * R) {
        float hj[R], xj[R], lm[R], sr[R], wg[R], wh[R];
        int jl[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            jl[r] = base + r * G + grp;
            const int j = sm.row0 + min(jl[r], nloc - 1);
            hj[r] = fmaf(hc[j], pl.bw, pl.center);
            xj[r] = STUDENT ? hj[r] : (hj[r] - pl.mu_center) * sc;
            if (!SCAN) {
                lm[r] = STUDENT ? nearest_lmax_student(mu, sm.n, hj[r], inv_nus2, half_np1)
                                : nearest_d2(mu, sm.n, xj[r]);
            }
            sr[r] = 0.0f; wg[r] = 0.0f; wh[r] = 0.0f;
        }
        if (SCAN) {
            // the smallest squared distance to any mean: a min over the row's
            // columns (this lane's slice, then across the S lanes); the same
            // value as the nearest sorted mean gives
            float mn[R];
            float2 x2[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                mn[r] = 3.0e38f;
                x2[r] = f2(xj[r]);
            }
            chunk_loop<U>(q * 4, nv, 4 * S, [&](int cb) {
                const float4 m4 = *reinterpret_cast<const float4*>(mu + cb);
                const float2 ma = make_float2(m4.x, m4.y), mb = make_float2(m4.z, m4.w);
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const float2 da = fma2(ma, f2(-1.0f), x2[r]), db = fma2(mb, f2(-1.0f), x2[r]);
                    const float2 qa = mul2(da, da), qb = mul2(db, db);
                    mn[r] = fminf(mn[r], fminf(fminf(qa.x, qa.y), fminf(qb.x, qb.y)));
                }
            });
#pragma unroll
            for (int o = S / 2; o > 0; o >>= 1) {
#pragma unroll
                for (int r = 0; r < R; ++r) mn[r] = fminf(mn[r], __shfl_xor_sync(0xffffffffu, mn[r], o));
            }
#pragma unroll
            for (int r = 0; r < R; ++r) lm[r] = STUDENT ? -half_np1 * kLn2 * lg2_approx(fmaf(mn[r], inv_nus2, 1.0f)) : mn[r];
        }
        if (!STUDENT) {
            // two columns per packed op: 3 issue slots and 2 ex2 per column pair
            float2 x2[R], nl2[R], sr2[R], wg2[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                x2[r] = f2(xj[r]);
                nl2[r] = f2(-lm[r]);
                sr2[r] = f2(0.0f);
                wg2[r] = f2(0.0f);
            }
            chunk_loop<U>(q * 4, nv, 4 * S, [&](int cb) {
                const float4 m4 = *reinterpret_cast<const float4*>(mu + cb);
                const float2 mm[2] = {make_float2(m4.x, m4.y), make_float2(m4.z, m4.w)};
#pragma unroll
                for (int hf = 0; hf < 2; ++hf) {
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const float2 d = fma2(mm[hf], f2(-1.0f), x2[r]);   // x - m
                        const float2 qq = fma2(d, d, nl2[r]);                // (x - m)^2 - min >= 0
                        const float2 w = make_float2(ex2_approx(-qq.x), ex2_approx(-qq.y));
                        sr2[r] = add2(sr2[r], w);
                        wg2[r] = fma2(w, d, wg2[r]);
                    }
                }
            });
#pragma unroll
            for (int r = 0; r < R; ++r) {
                sr[r] = sr2[r].x + sr2[r].y;
                wg[r] = wg2[r].x + wg2[r].y;
            }
        } else {
        for (int cb = q * 4; cb < nv; cb += 4 * S) {
            const float4 m4 = *reinterpret_cast<const float4*>(mu + cb);
            const float mm[4] = {m4.x, m4.y, m4.z, m4.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const float d = xj[r] - mm[e];
                    const float d2 = d * d;
                    const float den = nus2 + d2;
                    const float lr = -half_np1 * kLn2 * lg2_approx(fmaf(d2, inv_nus2, 1.0f));
                    const float w = ex2_approx((lr - lm[r]) * kLog2e);
                    const float iden = rcp_approx(den);
                    sr[r] += w;
                    wg[r] = fmaf(w * d, iden, wg[r]);
                    wh[r] = fmaf(w * (nus2 - d2), iden * iden, wh[r]);
                }
            }
        }
        }
        // combine the S column slices
#pragma unroll
        for (int o = S / 2; o > 0; o >>= 1) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                sr[r] += __shfl_xor_sync(0xffffffffu, sr[r], o);
                wg[r] += __shfl_xor_sync(0xffffffffu, wg[r], o);
                if (STUDENT) wh[r] += __shfl_xor_sync(0xffffffffu, wh[r], o);
            }
        }
        float psc[R], pcc[R];   // the row's pushed score and curvature (lane 0 of the row)
#pragma unroll
        for (int r = 0; r < R; ++r) psc[r] = pcc[r] = 0.0f;
        if (q == 0) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (jl[r] >= nloc) continue;
                const int j = sm.row0 + jl[r];
                const float h = hj[r];
                float gp, hp;
                if (!STUDENT) {
                    gp = -(wg[r] / sc) * inv_s2 / (sr[r] + 1e-8f);
                    hp = -inv_s2;
                } else {
                    gp = -np1 * wg[r] / (sr[r] + 1e-8f);
                    hp = -np1 * wh[r] / (sr[r] + 1e-8f);
                }
                // likelihood (:475-499)
                const float vol = expf(fminf(h, 20.0f));
                const float y2 = pl.y_t * pl.y_t;
                const float A = y2 / (vol + 1e-8f) / nu;
                const float opA = 1.0f + A;
                const float lw = pl.fan ? 0.0f
                                        : pl.stc - 0.5f * h - (nu + 1.0f) * 0.5f * log1pf(fmaxf(A, -0.999f));
                float glik;
                if (cfg.use_exact_gradient) glik = -0.5f + 0.5f * (nu + 1.0f) * A / opA - cfg.lik_offset;
                else glik = (logf(y2 + 1e-10f) - h + cfg.lik_offset) / 1.4f;
                const float eb = pl.fan ? 1.0f : beta;
                const float gg = clampf(gp + eb * glik, -10.0f, 10.0f);
                float score = gg, cc = 0.0f;
                if (pl.transport != 0) {
                    const float hl = -0.5f * (nu + 1.0f) * A / (opA * opA);
                    const float curv = clampf(-(hl + hp), 0.1f, 100.0f);
                    if (pl.transport == 2) {
                        cc = curv;
                    } else {
                        score = 0.7f * gg / curv;   // precond_grad (:519)
                        cc = 1.0f / curv;           // 1/curvature (:765)
                    }
                }
                if (team.size == 1) {
                    sm.g[j] = score;
                    sm.c[j] = cc;
                }
                psc[r] = score;
                pcc[r] = cc;
                lw_out[j] = lw;
            }
        }
        if (team.size > 1) push_rows<R, S, true>(sm.g, sm.c, psc, pcc, jl, nloc, sm.row0, q, team);
    }
}

// ---------------------------------------------------------------------------
// Transport pass (svpf_fused_stein_transport*_kernel, svpf_opt_kernels.cu:527-
// 1103): IMQ kernel K = 1 / (1 + d^2/bw^2), attraction K*score and repulsion
// 2 d/bw^2 K^2 (sign by stein_repulsive_sign), Newton scaling, optional KSD
// row sum, RMSProp, drift, SVLD diffusion, clamp.  KIND 0 vanilla, 1 Newton
// (precondition per column), 2 full Newton (kernel-weighted Hessian per row).
// Positions are read and written in transport coordinates hs = (h - center)/bw.
// Returns this thread's KSD row sums.
// ---------------------------------------------------------------------------
enum { kTransport = 0, kPhiOnly = 1, kKsdOnly = 2 };

// P is Plan (single factor: positions stored in transport coordinates
// (h - center) / bw) or FactorPlan (one factor of the two-factor tick:
// positions stored in log-volatility units, scaled inside the pair FMA as
// u = h_i / bw - h_j / bw, so the stiff per-factor priors read exact positions).
template <int R, int S, int KIND, bool KSD, int MODE = kTransport, class P = Plan, int U = 0>
__device__ float transport_pass(const Smem& sm, int cur, const P& pl, const svpf_config_t& cfg,
                                float bf, const Noise& nz, int kn, const Team& team,
                                float* __restrict__ phi_out = nullptr,
                                const float* __restrict__ pre = nullptr) {
    constexpr bool RAW = std::is_same<P, FactorPlan>::value;
    constexpr int G = kThreads / S;
    const int grp = threadIdx.x / S, q = threadIdx.x % S;
    const float* __restrict__ hc = sm.h[cur];
    float* __restrict__ hn = sm.h[cur ^ 1];
    const float* __restrict__ gs = sm.g;
    const float* __restrict__ cs = sm.c;
    const int n = sm.n;
    const int nloc = sm.row1 - sm.row0;
    const int nv = round_up(n, 4 * S);
    const float inv_bw = pl.inv_bw, inv_bw2 = pl.inv_bw2;
    const float sign = cfg.stein_repulsive_sign == 1 ? 1.0f : -1.0f;
    const float inv_n = 1.0f / (float)n;
    const float es = pl.eps_step * bf;
    const float rr = cfg.rmsprop_rho;
    float ksd_thread = 0.0f;

    for (int base = 0; base < nloc; base += G * R) {
        float hi[R], si[R];
        float ks[R], kg[R], gk[R], kc[R], nk[R], gkr[R], gdk[R], hs[R];
        int il[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            il[r] = base + r * G + grp;
            const int i = sm.row0 + min(il[r], nloc - 1);
            hi[r] = hc[i];
            si[r] = gs[i];
        }
        {
            // two columns per packed op: u = (h_i - h_j) / bw is one FFMA2 in
            // transport coordinates; columns past n hold a far pad whose terms
            // vanish.  Row sums are kept as two partial lanes and folded after.
            float2 hi2[R], ks2[R], kg2[R], gk2[R], kc2[R], gkr2[R], gdk2[R], hs2[R];
            float nks[R];
            const float2 colscale = f2(RAW ? -inv_bw : -1.0f);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                hi2[r] = f2(RAW ? hi[r] * inv_bw : hi[r]);
                ks2[r] = kg2[r] = gk2[r] = kc2[r] = gkr2[r] = gdk2[r] = hs2[r] = f2(0.0f);
                nks[r] = 0.0f;
            }
            chunk_loop<U>(q * 4, nv, 4 * S, [&](int cb) {
                const float4 h4 = *reinterpret_cast<const float4*>(hc + cb);
                const float4 g4 = *reinterpret_cast<const float4*>(gs + cb);
                float4 c4 = make_float4(0.f, 0.f, 0.f, 0.f);
                if (KIND != 0) c4 = *reinterpret_cast<const float4*>(cs + cb);
                const float2 hh[2] = {make_float2(h4.x, h4.y), make_float2(h4.z, h4.w)};
                const float2 gg[2] = {make_float2(g4.x, g4.y), make_float2(g4.z, g4.w)};
                const float2 cc[2] = {make_float2(c4.x, c4.y), make_float2(c4.z, c4.w)};
#pragma unroll
                for (int hf = 0; hf < 2; ++hf) {
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const float2 u = fma2(hh[hf], colscale, hi2[r]);
                        const float2 b2 = fma2(u, u, f2(1.0f));
                        const float2 K = make_float2(rcp_approx(b2.x), rcp_approx(b2.y));
                        const float2 K2 = mul2(K, K);
                        kg2[r] = fma2(K, gg[hf], kg2[r]);
                        if (KIND == 1 || KSD) {
                            const float2 uk2 = mul2(u, K2);
                            if (KIND == 1) gk2[r] = fma2(uk2, cc[hf], gk2[r]);
                            else gk2[r] = add2(gk2[r], uk2);
                            if (KSD) {
                                if (KIND == 1) gkr2[r] = add2(gkr2[r], uk2);
                                gdk2[r] = fma2(gg[hf], uk2, gdk2[r]);
                                hs2[r] = fma2(K2, fma2(K, f2(-4.0f), f2(3.0f)), hs2[r]);   // 4 (d/bw)^2 K - 1 = 3 - 4K
                            }
                        } else {
                            gk2[r] = fma2(u, K2, gk2[r]);
                        }
                        if (KIND == 2) {
                            ks2[r] = add2(ks2[r], K);
                            kc2[r] = fma2(K, cc[hf], kc2[r]);
                            const float2 w = fma2(b2, f2(3.0f), f2(-4.0f));             // 3 (d/bw)^2 - 1
                            nks[r] = fmaf(K2.x, fabsf(w.x), nks[r]);
                            nks[r] = fmaf(K2.y, fabsf(w.y), nks[r]);
                        }
                    }
                }
            });
#pragma unroll
            for (int r = 0; r < R; ++r) {
                ks[r] = ks2[r].x + ks2[r].y;
                kg[r] = kg2[r].x + kg2[r].y;
                gk[r] = gk2[r].x + gk2[r].y;
                kc[r] = kc2[r].x + kc2[r].y;
                nk[r] = nks[r];
                gkr[r] = gkr2[r].x + gkr2[r].y;
                gdk[r] = gdk2[r].x + gdk2[r].y;
                hs[r] = hs2[r].x + hs2[r].y;
            }
        }
#pragma unroll
        for (int o = S / 2; o > 0; o >>= 1) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                kg[r] += __shfl_xor_sync(0xffffffffu, kg[r], o);
                gk[r] += __shfl_xor_sync(0xffffffffu, gk[r], o);
                if (KIND == 2) {
                    ks[r] += __shfl_xor_sync(0xffffffffu, ks[r], o);
                    kc[r] += __shfl_xor_sync(0xffffffffu, kc[r], o);
                    nk[r] += __shfl_xor_sync(0xffffffffu, nk[r], o);
                }
                if (KSD) {
                    if (KIND == 1) gkr[r] += __shfl_xor_sync(0xffffffffu, gkr[r], o);
                    gdk[r] += __shfl_xor_sync(0xffffffffu, gdk[r], o);
                    hs[r] += __shfl_xor_sync(0xffffffffu, hs[r], o);
                }
            }
        }
        float pnew[R];   // the row's new position (lane 0 of the row)
#pragma unroll
        for (int r = 0; r < R; ++r) pnew[r] = 0.0f;
        if (q == 0) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (il[r] >= nloc) continue;
                const int i = sm.row0 + il[r];
                if constexpr (RAW && KIND == 0 && !KSD) {
                    // log-volatility positions are scaled inside the pair FMA, u =
                    // h_j (-1/bw) + round(h_i / bw): the row's own column enters with
                    // u = that rounding error, not 0; take its u K^2 back out
                    const float e = fmaf(hi[r], -inv_bw, __fmul_rn(hi[r], inv_bw));
                    const float Ke = rcp_approx(fmaf(e, e, 1.0f));
                    gk[r] -= e * (Ke * Ke);
                }
                // sums over u = d / bw carry one factor bw: 2 d K^2 / bw^2 = 2 u K^2 / bw
                float phi = (kg[r] + sign * 2.0f * inv_bw * gk[r]) * inv_n;
                if (KIND == 2) {
                    float H = (kc[r] + 2.0f * inv_bw2 * nk[r]) / fmaxf(ks[r], 1e-6f);
                    H = clampf(H, 0.1f, 100.0f);
                    phi = phi * (1.0f / H) * 0.7f;
                }
                if (KSD) {
                    const float gsum = (KIND == 1) ? gkr[r] : gk[r];
                    ksd_thread += si[r] * kg[r] + 2.0f * inv_bw * (si[r] * gsum - gdk[r]) + 2.0f * inv_bw2 * hs[r];
                }
                const int li = i - sm.row0;
                if (MODE == kPhiOnly) { phi_out[li] = phi; continue; }
                if (MODE == kKsdOnly) continue;
                const float vn = rr * sm.v[li] + (1.0f - rr) * phi * phi;
                sm.v[li] = vn;
                const float drift = es * phi * rsqrtf(vn + cfg.rmsprop_eps);
                float diff = 0.0f;
                if (pl.temp > 1e-6f) diff = sqrtf(2.0f * es * pl.temp) * (pre ? pre[li] : nz.normal(i, kn));
                const float h_new = clamp_h((RAW ? hi[r] : fmaf(hi[r], pl.bw, pl.center)) + drift + diff);
                const float hs_new = RAW ? h_new : (h_new - pl.center) * inv_bw;
                if (team.size == 1) hn[i] = hs_new;
                pnew[r] = hs_new;
            }
        }
        if (MODE == kTransport && team.size > 1)
            push_rows<R, S, false>(hn, hn, pnew, pnew, il, nloc, sm.row0, q, team);
    }
    return ksd_thread;
}

}  // namespace svpf
