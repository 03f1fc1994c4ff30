// svpf_estimator.cu -- the reference's differentiable torch model,
// SVPFParamEstimator (py-torch/diff_svpf_torch.py:147-217), as a batched CUDA
// forward and a hand-written reverse-mode adjoint, for F independent paths
// with their own theta = (mu, rho, sigma_z, nu).
//
// The model (per path, N particles, N even):
//   init    h = mu + sigma_z / sqrt(1 - rho^2 + 1e-6) z                 (:168-170)
//   tick t  TBPTT: the particle path is cut when t % truncate_every == 0 (:177-179)
//           eps = (z_1..z_{N/2}, -z_1..-z_{N/2})                        (:184-185)
//           m_i = mu + rho (h_i - mu),  hp_i = m_i + sigma_z eps_i      (:187-188)
//           loglik_t = logsumexp_i log t_nu(y_t; scale e^{hp_i/2}) - log N
//                      (before the transport; _student_t_log_prob :112-119)
//           b = (std(hp) + 0.1)^2 + 1e-8, no derivative through it      (:201)
//           n_stein times (Jacobi over particles):
//             g_i = clamp(-(h_i - m_i)/(sigma_z^2 + 1e-8) + lik score, +-10)  (:204-209)
//             h_i += lr/N sum_j [K_ij g_j - d_ij K_ij^3 / b],
//             d_ij = h_i - h_j, K_ij = (1 + d_ij^2/b)^(-1/2)            (:127-145)
//           vol_t = mean_i e^{h_i/2}                                     (:213)
//   loss    sum_t w_t loglik_t (the reference's NLL is w_t = -1/(T - burn_in)
//           after the burn-in, :214-215)
//
// One CTA per path (grid-stride over paths); all particle arrays of a tick
// live in shared memory.  The forward stores the particles every k ticks; the
// backward, segment by segment from the last, recomputes the segment from its
// checkpoint keeping each tick's input, then walks the ticks in reverse,
// recomputing each tick once more with every Stein iterate recorded in shared
// memory and sweeping its Stein steps backwards.
//
// Adjoint of one Stein step (a_i = lr xbar_i / N, G(d) = -d K^3 / b,
// G'(d) = -K^3/b + 3 d^2 K^5 / b^2, row sums over j with d = d_ij):
//   xbar_i += a_i (-S1/b + S2) - g_i C1/b - C2 + g'_i C3
//   S1 = sum g_j d K^3, S2 = sum G'(d), C1 = sum a_j d K^3, C2 = sum a_j G'(d),
//   C3 = sum a_j K = dL/dg_i;  g'_i = dg_i/dh_i (zero outside the clamp).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "svpf.h"
#include "svpf_device.cuh"
#include "svpf_internal.h"
#include "svpf_math.h"
#include "svpf_trace.h"

namespace svpf {
namespace est {

struct EArgs {
    int F, T, k, n, np, S, trunc, nseg;
    float lr;
    const float* theta;     // [F][4]
    const float* y;         // [F][T]
    const float* w;         // [F][T] or nullptr (all ones)
    const float* tape;      // [F][n + T n/2] or nullptr (Philox)
    unsigned long long seed;
    float* loglik;          // [F][T] or nullptr
    float* vol;             // [F][T] or nullptr
    double* ll_sum;         // [F]
    float* fx;              // [F][np] particles between forward launches
    float* ck;              // [F][nseg][np] checkpoints
    float* ax;              // [F][np] adjoint of the particles between backward launches
    double* ath;            // [F][4] accumulated d loss / d theta
    float* seg;             // [grid][k][np] tick inputs of the segment being reversed
    int* status;            // [F]
};

// Per-path scalars of the tick being processed (thread 0 writes, all read).
struct TickShared {
    float mu, rho, sz, nu, C;
    float mx, se, b;        // logsumexp max and sum, kernel scale b
    float red[8][kWarps];
    double acc[4];
    int bad;                // this path's theta is outside the domain (theta_ok)
};

__device__ __forceinline__ size_t tape_stride(const EArgs& a) { return (size_t)a.n + (size_t)a.T * (a.n / 2); }

// Initial standard normal of particle i (torch.randn(N), :170).
__device__ __forceinline__ float init_normal(const EArgs& a, int f, int i) {
    if (a.tape) return a.tape[(size_t)f * tape_stride(a) + i];
    const uint4 r = philox10(philox_key(a.seed, f), make_uint4((uint32_t)i, 0u, 0u, 2u));
    return normal_from_bits(r.x, r.y);
}

// Antithetic predict noise of particle i at tick t (:184-185).
__device__ __forceinline__ float tick_eps(const EArgs& a, int f, int t, int i) {
    const int half = a.n / 2;
    const int ii = i < half ? i : i - half;
    float z;
    if (a.tape) {
        z = a.tape[(size_t)f * tape_stride(a) + a.n + (size_t)t * half + ii];
    } else {
        const uint4 r = philox10(philox_key(a.seed, f), make_uint4((uint32_t)ii, 0u, (uint32_t)t, 0u));
        z = normal_from_bits(r.x, r.y);
    }
    return i < half ? z : -z;
}

template <int K>
__device__ __forceinline__ void block_sum(float (&v)[K], TickShared& sh) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < K; ++q) {
        v[q] = warp_sum(v[q]);
        if (lane == 0) sh.red[q][wp] = v[q];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; ++q) {
        float s = 0.0f;
        for (int i = 0; i < kWarps; ++i) s += sh.red[q][i];
        v[q] = s;
    }
    __syncthreads();
}
__device__ __forceinline__ float block_max(float v, TickShared& sh) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    v = warp_max(v);
    if (lane == 0) sh.red[0][wp] = v;
    __syncthreads();
    float m = sh.red[0][0];
    for (int i = 1; i < kWarps; ++i) m = fmaxf(m, sh.red[0][i]);
    __syncthreads();
    return m;
}

// Shared-memory arrays of one path (np floats each).
struct Arrays {
    float *xin, *h, *hn, *m, *lp, *g, *gd, *ab, *xb, *mb, *rec;
};
__device__ inline Arrays carve(float* base, int np, int S) {
    Arrays s;
    float* p = base;
    s.xin = p; p += np;
    s.h = p; p += np;
    s.hn = p; p += np;
    s.m = p; p += np;
    s.lp = p; p += np;
    s.g = p; p += np;
    s.gd = p; p += np;
    s.ab = p; p += np;
    s.xb = p; p += np;
    s.mb = p; p += np;
    s.rec = p;   // S np floats: h before each Stein step
    return s;
}
__host__ __device__ inline int smem_floats_est(int np, int S) { return (10 + S) * np; }

// Likelihood score (:205-207): A = y^2 / (e^h nu + 1e-8),
// g_lik = -1/2 + (nu+1)/2 A/(1+A).  With derivatives d/dh and d/dnu.
struct LikScore {
    float gl, dgl_dh, dgl_dnu;
};
__device__ __forceinline__ LikScore lik_score(float h, float y2, float nu) {
    const float v = expf(0.5f * h);
    const float ev = v * v;
    const float den = ev * nu + 1e-8f;
    const float A = y2 / den;
    const float opA = 1.0f + A;
    LikScore r;
    r.gl = -0.5f + 0.5f * (nu + 1.0f) * A / opA;
    const float dgl_dA = 0.5f * (nu + 1.0f) / (opA * opA);
    const float q = ev / den;               // dA/dh = -A nu q, dA/dnu = -A q
    r.dgl_dh = dgl_dA * (-A * nu * q);
    r.dgl_dnu = 0.5f * A / opA + dgl_dA * (-A * q);
    return r;
}

// Forward of tick t for path f: xin -> h (the tick's output particles).
// rec != nullptr records h before each Stein step (rec[0] = the predicted
// particles, also when there are no Stein steps).  Returns loglik_t on every
// thread; *vol_out (thread 0) the volatility estimate.
__device__ float fwd_tick(const EArgs& a, int f, int t, const Arrays& s, TickShared& sh, float* rec,
                          float* vol_out) {
    const int tid = threadIdx.x, n = a.n, np = a.np;
    const float mu = sh.mu, rho = sh.rho, sz = sh.sz, nu = sh.nu;
    const float y = a.y[(size_t)f * a.T + t];
    const float y2 = y * y;
    // predict + predictive log-likelihood terms (:183-198)
    float lmax = -3.0e38f, psum[1] = {0.0f};
    for (int i = tid; i < n; i += kThreads) {
        const float e = tick_eps(a, f, t, i);
        const float mi = mu + rho * (s.xin[i] - mu);
        const float hp = mi + sz * e;
        s.m[i] = mi;
        s.h[i] = hp;
        if (rec) rec[i] = hp;
        const float sc = expf(0.5f * hp);
        const float z = y / (sc + 1e-8f);
        const float lp = sh.C - logf(sc + 1e-8f) - (nu + 1.0f) * 0.5f * log1pf(z * z / nu);
        s.lp[i] = lp;
        lmax = fmaxf(lmax, lp);
        psum[0] += hp;
    }
    lmax = block_max(lmax, sh);
    float r2[2] = {0.0f, 0.0f};
    block_sum<1>(psum, sh);
    const float hm = psum[0] / (float)n;
    for (int i = tid; i < n; i += kThreads) {
        r2[0] += expf(s.lp[i] - lmax);
        const float d = s.h[i] - hm;
        r2[1] += d * d;
    }
    block_sum<2>(r2, sh);
    const float ll = lmax + logf(r2[0]) - logf((float)n);
    const float bw = sqrtf(r2[1] / (float)n) + 0.1f;
    const float b = bw * bw + 1e-8f;
    const float ib = 1.0f / b;
    if (tid == 0) {
        sh.mx = lmax;
        sh.se = r2[0];
        sh.b = b;
    }
    // Stein transport (:203-211)
    const float is2e = 1.0f / (sz * sz + 1e-8f);
    const float scale = a.lr / (float)n;
    for (int st = 0; st < a.S; ++st) {
        for (int i = tid; i < n; i += kThreads) {
            const float hi = s.h[i];
            if (rec && st > 0) rec[(size_t)st * np + i] = hi;
            const LikScore L = lik_score(hi, y2, nu);
            s.g[i] = clampf(-(hi - s.m[i]) * is2e + L.gl, -10.0f, 10.0f);
        }
        __syncthreads();
        for (int i = tid; i < n; i += kThreads) {
            const float hi = s.h[i];
            float att = 0.0f, rep = 0.0f;
            for (int j = 0; j < n; ++j) {
                const float d = hi - s.h[j];
                const float K = rsqrtf(fmaf(d * d, ib, 1.0f));
                att = fmaf(K, s.g[j], att);
                rep = fmaf(-d * K, K * K, rep);
            }
            s.hn[i] = hi + scale * (att + rep * ib);
        }
        __syncthreads();
        for (int i = tid; i < n; i += kThreads) s.h[i] = s.hn[i];
        __syncthreads();
    }
    float vs[1] = {0.0f};
    for (int i = tid; i < n; i += kThreads) vs[0] += expf(0.5f * s.h[i]);
    block_sum<1>(vs, sh);
    if (tid == 0 && vol_out) *vol_out = vs[0] / (float)n;
    return ll;
}

// Backward of tick t: s.xb holds d loss / d(output particles) on entry and
// d loss / d(input particles) on exit; theta adjoints accumulate in sh.acc.
// Requires the recorded forward of the same tick (s.m, s.lp, s.h, rec, sh.mx,
// sh.se, sh.b) just before.
__device__ void bwd_tick(const EArgs& a, int f, int t, const Arrays& s, TickShared& sh, const float* rec, float wt) {
    const int tid = threadIdx.x, n = a.n, np = a.np;
    const float mu = sh.mu, rho = sh.rho, sz = sh.sz, nu = sh.nu;
    const float y = a.y[(size_t)f * a.T + t];
    const float y2 = y * y;
    const float b = sh.b, ib = 1.0f / b, ib2 = ib * ib;
    const float is2e = 1.0f / (sz * sz + 1e-8f);
    const float scale = a.lr / (float)n;
    float pmu = 0.0f, prho = 0.0f, psz = 0.0f, pnu = 0.0f, ps2e = 0.0f;
    for (int i = tid; i < n; i += kThreads) s.mb[i] = 0.0f;
    for (int st = a.S - 1; st >= 0; --st) {
        const float* hs = rec + (size_t)st * np;
        for (int i = tid; i < n; i += kThreads) {
            const float hi = hs[i];
            const LikScore L = lik_score(hi, y2, nu);
            const float gpre = -(hi - s.m[i]) * is2e + L.gl;
            const bool in = gpre >= -10.0f && gpre <= 10.0f;   // torch.clamp passes the gradient inclusive
            s.g[i] = clampf(gpre, -10.0f, 10.0f);
            s.gd[i] = in ? -is2e + L.dgl_dh : 0.0f;
            s.ab[i] = scale * s.xb[i];
            s.hn[i] = in ? 1.0f : 0.0f;   // clamp mask of this step
        }
        __syncthreads();
        for (int i = tid; i < n; i += kThreads) {
            const float hi = hs[i];
            float S1 = 0.0f, S2 = 0.0f, C1 = 0.0f, C2 = 0.0f, C3 = 0.0f;
            for (int j = 0; j < n; ++j) {
                const float d = hi - hs[j];
                const float K = rsqrtf(fmaf(d * d, ib, 1.0f));
                const float K2 = K * K;
                const float dK3 = d * K * K2;
                const float Gp = K * K2 * fmaf(3.0f * d * d * K2, ib2, -ib);
                const float aj = s.ab[j];
                S1 = fmaf(s.g[j], dK3, S1);
                S2 += Gp;
                C1 = fmaf(aj, dK3, C1);
                C2 = fmaf(aj, Gp, C2);
                C3 = fmaf(aj, K, C3);
            }
            const float ai = s.ab[i];
            s.xb[i] += ai * (S2 - S1 * ib) - s.g[i] * C1 * ib - C2 + s.gd[i] * C3;
            const float gb = s.hn[i] * C3;   // d loss / d g_i
            s.mb[i] += gb * is2e;
            ps2e += gb * (hi - s.m[i]) * is2e * is2e;
            pnu += gb * lik_score(hi, y2, nu).dgl_dnu;
        }
        __syncthreads();
    }
    // predictive log-likelihood: d/dhp_i and d/dnu of w_t logsumexp(lp) (:192-198)
    const float mx = sh.mx, inv_se = 1.0f / sh.se;
    for (int i = tid; i < n; i += kThreads) {
        const float hp = rec[i];   // h before the first Stein step = hp
        const float pw = wt * expf(s.lp[i] - mx) * inv_se;
        const float sc = expf(0.5f * hp);
        const float se = sc + 1e-8f;
        const float z = y / se;
        const float q = z * z / nu;
        const float dlp_dsc = -1.0f / se + (nu + 1.0f) * q / ((1.0f + q) * se);
        s.xb[i] += pw * dlp_dsc * 0.5f * sc;
        pnu += pw * (-0.5f * log1pf(q) + 0.5f * (nu + 1.0f) * q / (nu * (1.0f + q)));
    }
    __syncthreads();
    // predict: hp = m + sigma_z eps, m = mu + rho (xin - mu)
    const bool cut = a.trunc > 0 && t > 0 && t % a.trunc == 0;
    for (int i = tid; i < n; i += kThreads) {
        const float hpb = s.xb[i];
        const float mt = s.mb[i] + hpb;
        const float xi = s.xin[i];
        pmu += (1.0f - rho) * mt;
        prho += (xi - mu) * mt;
        psz += hpb * tick_eps(a, f, t, i);
        s.xb[i] = cut ? 0.0f : rho * mt;
    }
    float v[5] = {pmu, prho, psz, pnu, ps2e};
    block_sum<5>(v, sh);
    if (tid == 0) {
        // d/dnu of the normaliser lgamma((nu+1)/2) - lgamma(nu/2) - log(nu pi)/2 (:75-80)
        const double dC = 0.5 * digamma_bounded(0.5 * ((double)nu + 1.0)) - 0.5 * digamma_bounded(0.5 * (double)nu) -
                          0.5 / (double)nu;
        sh.acc[0] += v[0];
        sh.acc[1] += v[1];
        sh.acc[2] += (double)v[2] + (double)v[4] * 2.0 * (double)sz;
        // the constant enters every log-density; the softmax weights sum to one
        sh.acc[3] += (double)v[3] + dC * (double)wt;
    }
    __syncthreads();
}

__device__ inline void load_theta(const EArgs& a, int f, TickShared& sh) {
    sh.mu = a.theta[4 * f + 0];
    sh.rho = a.theta[4 * f + 1];
    sh.sz = a.theta[4 * f + 2];
    sh.nu = a.theta[4 * f + 3];
    const float nu = sh.nu;
    sh.C = lgammaf((nu + 1.0f) * 0.5f) - lgammaf(nu * 0.5f) - 0.5f * logf(nu * 3.14159265358979f);
    sh.bad = !theta_ok(sh.mu, sh.rho, sh.sz, sh.nu);
}

__global__ void __launch_bounds__(kThreads) est_forward_kernel(const EArgs a, int t0, int t1) {
    extern __shared__ __align__(16) float smem[];
    __shared__ TickShared sh;
    const Arrays s = carve(smem, a.np, a.S);
    const int n = a.n;
    for (int f = blockIdx.x; f < a.F; f += gridDim.x) {
        if (threadIdx.x == 0) load_theta(a, f, sh);
        __syncthreads();
        if (sh.bad) {
            // parameters no filter can run with: report them and leave the path out
            for (int t = t0 + threadIdx.x; t < t1; t += kThreads) {
                if (a.loglik) a.loglik[(size_t)f * a.T + t] = NAN;
                if (a.vol) a.vol[(size_t)f * a.T + t] = NAN;
            }
            if (threadIdx.x == 0) {
                a.status[f] = SVPF_ERR_INVALID_ARG;
                a.ll_sum[f] = NAN;
            }
            __syncthreads();
            continue;
        }
        if (t0 == 0) {
            // :168-170
            const float hs = sh.sz / sqrtf(1.0f - sh.rho * sh.rho + 1e-6f);
            for (int i = threadIdx.x; i < n; i += kThreads) s.xin[i] = sh.mu + hs * init_normal(a, f, i);
            if (threadIdx.x == 0) a.ll_sum[f] = 0.0;
        } else {
            for (int i = threadIdx.x; i < n; i += kThreads) s.xin[i] = a.fx[(size_t)f * a.np + i];
        }
        __syncthreads();
        double lls = 0.0;
        for (int t = t0; t < t1; ++t) {
            if (t % a.k == 0) {
                float* ck = a.ck + ((size_t)f * a.nseg + t / a.k) * a.np;
                for (int i = threadIdx.x; i < n; i += kThreads) ck[i] = s.xin[i];
            }
            float vol = 0.0f;
            const float ll = fwd_tick(a, f, t, s, sh, nullptr, &vol);
            if (threadIdx.x == 0) {
                if (a.loglik) a.loglik[(size_t)f * a.T + t] = ll;
                if (a.vol) a.vol[(size_t)f * a.T + t] = vol;
                lls += (double)ll;
                if (!isfinite(ll)) a.status[f] = SVPF_ERR_NONFINITE;
            }
            for (int i = threadIdx.x; i < n; i += kThreads) s.xin[i] = s.h[i];
            __syncthreads();
        }
        for (int i = threadIdx.x; i < n; i += kThreads) a.fx[(size_t)f * a.np + i] = s.xin[i];
        if (threadIdx.x == 0) a.ll_sum[f] += lls;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads, 4) est_backward_kernel(const EArgs a, int sg) {
    extern __shared__ __align__(16) float smem[];
    __shared__ TickShared sh;
    const Arrays s = carve(smem, a.np, a.S);
    const int n = a.n, np = a.np;
    float* seg = a.seg + (size_t)blockIdx.x * a.k * np;
    const int t0 = sg * a.k;
    const int t1 = min(a.T, t0 + a.k);
    for (int f = blockIdx.x; f < a.F; f += gridDim.x) {
        if (threadIdx.x == 0) {
            load_theta(a, f, sh);
            for (int q = 0; q < 4; ++q) sh.acc[q] = a.ath[4 * (size_t)f + q];
        }
        __syncthreads();
        if (sh.bad) {
            if (threadIdx.x == 0) {
                for (int q = 0; q < 4; ++q) a.ath[4 * (size_t)f + q] = NAN;
                a.status[f] = SVPF_ERR_INVALID_ARG;
            }
            __syncthreads();
            continue;
        }
        const float* ck = a.ck + ((size_t)f * a.nseg + sg) * np;
        for (int i = threadIdx.x; i < n; i += kThreads) {
            s.xin[i] = ck[i];
            s.xb[i] = a.ax[(size_t)f * np + i];
        }
        __syncthreads();
        // recompute the segment, keeping each tick's input particles
        for (int t = t0; t < t1; ++t) {
            float* sx = seg + (size_t)(t - t0) * np;
            for (int i = threadIdx.x; i < n; i += kThreads) sx[i] = s.xin[i];
            fwd_tick(a, f, t, s, sh, nullptr, nullptr);
            for (int i = threadIdx.x; i < n; i += kThreads) s.xin[i] = s.h[i];
            __syncthreads();
        }
        // reverse over the segment's ticks
        for (int t = t1 - 1; t >= t0; --t) {
            const float* sx = seg + (size_t)(t - t0) * np;
            for (int i = threadIdx.x; i < n; i += kThreads) s.xin[i] = sx[i];
            __syncthreads();
            fwd_tick(a, f, t, s, sh, s.rec, nullptr);
            const float wt = a.w ? a.w[(size_t)f * a.T + t] : 1.0f;
            bwd_tick(a, f, t, s, sh, s.rec, wt);
        }
        if (t0 == 0) {
            // h0 = mu + hs z, hs = sigma_z / sqrt(q), q = 1 - rho^2 + 1e-6
            float v[2] = {0.0f, 0.0f};
            for (int i = threadIdx.x; i < n; i += kThreads) {
                v[0] += s.xb[i];
                v[1] += s.xb[i] * init_normal(a, f, i);
            }
            block_sum<2>(v, sh);
            if (threadIdx.x == 0) {
                const double rho = sh.rho, sz = sh.sz;
                const double q = 1.0 - rho * rho + 1e-6;
                sh.acc[0] += v[0];
                sh.acc[2] += (double)v[1] / sqrt(q);
                sh.acc[1] += (double)v[1] * sz * rho / (q * sqrt(q));
            }
        }
        for (int i = threadIdx.x; i < n; i += kThreads) a.ax[(size_t)f * np + i] = s.xb[i];
        if (threadIdx.x == 0)
            for (int q = 0; q < 4; ++q) a.ath[4 * (size_t)f + q] = sh.acc[q];
        __syncthreads();
    }
}

}  // namespace est
}  // namespace svpf

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using namespace svpf;
using namespace svpf::est;

struct svpf_estimator {
    int F = 0, n = 0, np = 0, S = 0, T_max = 0, k = 64, nseg = 0, trunc = 0, grid = 0, T = 0;
    float lr = 0.1f;
    size_t smem = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool forward_done = false;
    unsigned long long seed = 0;
    float *d_theta = nullptr, *d_y = nullptr, *d_w = nullptr, *d_tape = nullptr, *d_loglik = nullptr,
          *d_vol = nullptr, *d_fx = nullptr, *d_ck = nullptr, *d_ax = nullptr, *d_seg = nullptr;
    double *d_llsum = nullptr, *d_ath = nullptr;
    int* d_status = nullptr;
    const float *u_theta = nullptr, *u_y = nullptr, *u_tape = nullptr;
};

namespace {

template <class T>
bool ealloc(T** p, size_t count) {
    return cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T)) == cudaSuccess;
}

EArgs make_eargs(const svpf_estimator* e, const float* theta, const float* y, const float* tape, const float* w,
                 float* loglik, float* vol) {
    EArgs a;
    std::memset(&a, 0, sizeof(a));
    a.F = e->F;
    a.T = e->T;
    a.k = e->k;
    a.n = e->n;
    a.np = e->np;
    a.S = e->S;
    a.trunc = e->trunc;
    a.nseg = e->nseg;
    a.lr = e->lr;
    a.theta = theta;
    a.y = y;
    a.w = w;
    a.tape = tape;
    a.seed = e->seed;
    a.loglik = loglik;
    a.vol = vol;
    a.ll_sum = e->d_llsum;
    a.fx = e->d_fx;
    a.ck = e->d_ck;
    a.ax = e->d_ax;
    a.ath = e->d_ath;
    a.seg = e->d_seg;
    a.status = e->d_status;
    return a;
}

}  // namespace

extern "C" {

long long svpf_estimator_tape_floats(int n_particles, int T) {
    if (n_particles < 2 || T < 0) return 0;
    return (long long)n_particles + (long long)T * (n_particles / 2);
}

svpf_estimator_t* svpf_estimator_create(int n_filters, int n_particles, int n_stein_steps, float stein_lr,
                                        int T_max, int checkpoint_every, int truncate_every, cudaStream_t stream) {
    SVPF_TRACE();
    if (n_filters < 1 || n_particles < 2 || (n_particles & 1) || n_particles > SVPF_MAX_PARTICLES ||
        n_stein_steps < 0 || n_stein_steps > 64 || T_max < 1 || checkpoint_every < 1 || truncate_every < 0 ||
        !std::isfinite(stein_lr))
        return nullptr;
    svpf_estimator* e = new svpf_estimator();
    e->F = n_filters;
    e->n = n_particles;
    e->np = round_up(n_particles, 64);
    e->S = n_stein_steps;
    e->lr = stein_lr;
    e->T_max = T_max;
    e->k = checkpoint_every;
    e->nseg = (T_max + checkpoint_every - 1) / checkpoint_every;
    e->trunc = truncate_every;
    // the backward records the particles before each Stein step: at least one array
    e->smem = (size_t)smem_floats_est(e->np, std::max(e->S, 1)) * sizeof(float);
    int dev = 0, optin = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e->smem + sizeof(TickShared) + 64 > (size_t)optin) {
        delete e;
        return nullptr;
    }
    if (stream) {
        e->stream = stream;
    } else {
        cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
        e->own_stream = true;
    }
    // the opt-in is the device's whole limit (engines of different sizes share the kernels)
    if (configure_kernel((const void*)est_forward_kernel, (int)kernel_smem_cap((const void*)est_forward_kernel),
                         false) != cudaSuccess ||
        configure_kernel((const void*)est_backward_kernel, (int)kernel_smem_cap((const void*)est_backward_kernel),
                         false) != cudaSuccess) {
        cudaGetLastError();
        svpf_estimator_destroy(e);
        return nullptr;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, est_backward_kernel, kThreads, e->smem);
    e->grid = std::min(n_filters, std::max(1, per_sm) * std::max(sms, 1));
    const size_t F = (size_t)n_filters, np = (size_t)e->np;
    const bool ok = ealloc(&e->d_theta, 4 * F) && ealloc(&e->d_y, F * T_max) && ealloc(&e->d_w, F * T_max) &&
                    ealloc(&e->d_loglik, F * T_max) && ealloc(&e->d_vol, F * T_max) && ealloc(&e->d_fx, F * np) &&
                    ealloc(&e->d_ck, F * e->nseg * np) && ealloc(&e->d_ax, F * np) &&
                    ealloc(&e->d_seg, (size_t)e->grid * e->k * np) && ealloc(&e->d_llsum, F) &&
                    ealloc(&e->d_ath, 4 * F) && ealloc(&e->d_status, F);
    if (!ok) {
        svpf_estimator_destroy(e);
        return nullptr;
    }
    return e;
}

void svpf_estimator_destroy(svpf_estimator_t* e) {
    if (!e) return;
    if (e->stream) cudaStreamSynchronize(e->stream);
    void* ptrs[] = {e->d_theta, e->d_y, e->d_w, e->d_tape, e->d_loglik, e->d_vol, e->d_fx, e->d_ck,
                    e->d_ax, e->d_seg, e->d_llsum, e->d_ath, e->d_status};
    for (void* p : ptrs) cudaFree(p);
    if (e->own_stream) cudaStreamDestroy(e->stream);
    delete e;
}

int svpf_estimator_forward_device(svpf_estimator_t* e, const float* d_theta, const float* d_y, int T,
                                  unsigned long long seed, const float* d_tape, float* d_loglik, float* d_vol) {
    SVPF_TRACE();
    if (!e || !d_theta || !d_y || T < 1 || T > e->T_max) return SVPF_ERR_INVALID_ARG;
    e->T = T;
    e->seed = seed;
    e->u_theta = d_theta;
    e->u_y = d_y;
    e->u_tape = d_tape;
    if (cudaMemsetAsync(e->d_status, 0, e->F * sizeof(int), e->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    const EArgs a = make_eargs(e, d_theta, d_y, d_tape, nullptr, d_loglik ? d_loglik : e->d_loglik,
                               d_vol ? d_vol : e->d_vol);
    for (int t0 = 0; t0 < T; t0 += e->k) {
        est_forward_kernel<<<e->grid, kThreads, e->smem, e->stream>>>(a, t0, std::min(T, t0 + e->k));
        if (cudaGetLastError() != cudaSuccess) return SVPF_ERR_CUDA;
    }
    e->forward_done = true;
    return SVPF_OK;
}

int svpf_estimator_backward_device(svpf_estimator_t* e, const float* d_w, double* d_grad) {
    SVPF_TRACE();
    if (!e || !e->forward_done) return SVPF_ERR_NOT_INITIALIZED;
    if (cudaMemsetAsync(e->d_ax, 0, (size_t)e->F * e->np * sizeof(float), e->stream) != cudaSuccess ||
        cudaMemsetAsync(e->d_ath, 0, (size_t)e->F * 4 * sizeof(double), e->stream) != cudaSuccess)
        return SVPF_ERR_CUDA;
    const EArgs a = make_eargs(e, e->u_theta, e->u_y, e->u_tape, d_w, nullptr, nullptr);
    const int nseg = (e->T + e->k - 1) / e->k;
    for (int sg = nseg - 1; sg >= 0; --sg) {
        est_backward_kernel<<<e->grid, kThreads, e->smem, e->stream>>>(a, sg);
        if (cudaGetLastError() != cudaSuccess) return SVPF_ERR_CUDA;
    }
    if (d_grad && cudaMemcpyAsync(d_grad, e->d_ath, (size_t)e->F * 4 * sizeof(double), cudaMemcpyDeviceToDevice,
                                  e->stream) != cudaSuccess)
        return SVPF_ERR_CUDA;
    return SVPF_OK;
}

int svpf_estimator_forward(svpf_estimator_t* e, const float* theta, const float* y, int T, unsigned long long seed,
                           const float* tape, float* loglik, float* vol, double* loglik_sum) {
    SVPF_TRACE();
    if (!e || !theta || !y || T < 1 || T > e->T_max) return SVPF_ERR_INVALID_ARG;
    const size_t F = (size_t)e->F;
    for (size_t f = 0; f < F; ++f)
        if (!theta_ok(theta[4 * f], theta[4 * f + 1], theta[4 * f + 2], theta[4 * f + 3])) return SVPF_ERR_INVALID_ARG;
    if (cudaMemcpyAsync(e->d_theta, theta, 4 * F * sizeof(float), cudaMemcpyHostToDevice, e->stream) != cudaSuccess ||
        cudaMemcpyAsync(e->d_y, y, F * T * sizeof(float), cudaMemcpyHostToDevice, e->stream) != cudaSuccess)
        return SVPF_ERR_CUDA;
    const float* d_tape = nullptr;
    if (tape) {
        const size_t tf = F * (size_t)svpf_estimator_tape_floats(e->n, T);
        // the tape's size depends on T: keep one buffer, grown on demand
        if (cudaStreamSynchronize(e->stream) != cudaSuccess) return SVPF_ERR_CUDA;
        cudaFree(e->d_tape);
        e->d_tape = nullptr;
        if (!ealloc(&e->d_tape, tf)) return SVPF_ERR_CUDA;
        if (cudaMemcpyAsync(e->d_tape, tape, tf * sizeof(float), cudaMemcpyHostToDevice, e->stream) != cudaSuccess)
            return SVPF_ERR_CUDA;
        d_tape = e->d_tape;
    }
    int rc = svpf_estimator_forward_device(e, e->d_theta, e->d_y, T, seed, d_tape, e->d_loglik, e->d_vol);
    if (rc != SVPF_OK) return rc;
    if (loglik && cudaMemcpyAsync(loglik, e->d_loglik, F * T * sizeof(float), cudaMemcpyDeviceToHost, e->stream) !=
                      cudaSuccess)
        return SVPF_ERR_CUDA;
    if (vol && cudaMemcpyAsync(vol, e->d_vol, F * T * sizeof(float), cudaMemcpyDeviceToHost, e->stream) != cudaSuccess)
        return SVPF_ERR_CUDA;
    if (loglik_sum &&
        cudaMemcpyAsync(loglik_sum, e->d_llsum, F * sizeof(double), cudaMemcpyDeviceToHost, e->stream) != cudaSuccess)
        return SVPF_ERR_CUDA;
    if (cudaStreamSynchronize(e->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    std::vector<int> st(F);
    if (cudaMemcpy(st.data(), e->d_status, F * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SVPF_ERR_CUDA;
    for (int s : st)
        if (s) return s;
    return SVPF_OK;
}

int svpf_estimator_get_status(svpf_estimator_t* e, int* status) {
    if (!e || !status) return SVPF_ERR_INVALID_ARG;
    if (cudaStreamSynchronize(e->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    return cudaMemcpy(status, e->d_status, (size_t)e->F * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess
               ? SVPF_OK : SVPF_ERR_CUDA;
}

int svpf_estimator_backward(svpf_estimator_t* e, const float* w, double* grad) {
    SVPF_TRACE();
    if (!e || !grad) return SVPF_ERR_INVALID_ARG;
    if (!e->forward_done) return SVPF_ERR_NOT_INITIALIZED;
    const size_t F = (size_t)e->F;
    const float* dw = nullptr;
    if (w) {
        if (cudaMemcpyAsync(e->d_w, w, F * e->T * sizeof(float), cudaMemcpyHostToDevice, e->stream) != cudaSuccess)
            return SVPF_ERR_CUDA;
        dw = e->d_w;
    }
    int rc = svpf_estimator_backward_device(e, dw, nullptr);
    if (rc == SVPF_OK &&
        cudaMemcpyAsync(grad, e->d_ath, 4 * F * sizeof(double), cudaMemcpyDeviceToHost, e->stream) != cudaSuccess)
        rc = SVPF_ERR_CUDA;
    if (rc == SVPF_OK && cudaStreamSynchronize(e->stream) != cudaSuccess) rc = SVPF_ERR_CUDA;
    return rc;
}

}  // extern "C"
