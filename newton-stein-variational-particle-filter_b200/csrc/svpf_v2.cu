// svpf_v2.cu -- svpf_fully_fused_step_v2: the reference's second, single-kernel
// tick (include/svpf_fully_fused_v2.cuh:43-119, src/svpf_fully_fused_v2.cu),
// as one launch of a thread-block cluster of C <= 16 CTAs.
//
// Every member runs the O(N) phases for all N rows (predict, guide, Silverman
// bandwidth: deterministic, so the copies agree without an exchange); the
// O(N^2) gradient and transport of each Stein iteration are split by rows, and
// each member pushes its rows' scores and new positions into every member's
// shared memory (DSMEM), one cluster barrier after each push.  The log-weights
// and KSD partials of the rows are pushed to rank 0, which writes the
// outputs.  N is limited by shared memory (8192), not by one block (the
// reference's 1024).
//
// Semantics follow the reference kernel line by line, including its quirks:
// the prior score is clamped to +-10 before the annealed likelihood is added;
// with use_newton the repulsion is scaled by sh_hess[j] even in full-Newton
// mode (where it holds the curvature), and the KSD "raw" score divides by
// 0.7 sh_hess[j]; the guide strength is always adaptive; a uniform is drawn for
// MIM whatever its probability.  Noise: per particle, normal draws 0..3 (the
// reference's curand_normal4: 0 state, 1 first diffusion), then one normal per
// Stein iteration with SVLD, then the rejuvenation normal; uniforms 0 (MIM)
// and 1 (rejuvenation).  They come from the engine's counter-based Philox
// keyed by (seed, filter) and counted by (particle, draw, tick), or from a
// device noise tape -- both described by the svpf_v2_rng_t record the caller
// passes where the reference passes curand states.
#include <cooperative_groups.h>
#include <cstring>
#include <mutex>

#include "svpf.h"
#include "svpf_device.cuh"
#include "svpf_internal.h"
#include "svpf_trace.h"

namespace svpf {
namespace v2 {

constexpr int kT = 256;   // threads per CTA
constexpr int kW = kT / 32;

// The scalar arguments of svpf_fully_fused_step_v2.
struct Params {
    float rho, sigma_z, mu, nu, lik_offset, student_t_const, student_t_implied_offset, gamma;
    float delta_rho, delta_sigma, mim_jump_prob, mim_jump_scale;
    float guide_strength_base, guide_strength_max, guide_innovation_threshold;
    float guided_alpha_base, guided_alpha_shock, guided_innovation_thresh_predict;
    int use_guide, use_guided_predict, use_guide_preserving, use_newton, use_full_newton, use_rejuvenation;
    float rejuv_ksd_threshold, rejuv_prob, rejuv_blend;
    int use_adaptive_mu;
    float mu_ema_alpha;
    int use_adaptive_sigma;
    float sigma_boost_threshold, sigma_boost_max, step_size, temperature, rmsprop_rho, rmsprop_eps;
    int n_stein_steps, n_anneal_steps, stein_sign_mode;
};

struct Args {
    float *h, *h_prev, *grad, *lw, *v, *inv_hess;
    svpf_v2_rng_t* rng;
    float y_t, y_prev, h_mean_prev, vol_prev, ksd_prev;
    float *d_h_mean, *d_vol, *d_loglik, *d_bw, *d_ksd, *d_guide_mean, *d_guide_var, *d_mu_state;
    Params p;
    int n, timestep;
    int npre_cap;   // steps whose diffusion normals fit in shared memory to pre-draw
};

struct Shared {
    float red[4][kW];
    float eff_mu, eff_sigma, gm, gv, gs, bw, new_gm, new_gv;
    int write_guide;
    svpf_v2_rng_t rng;
    int flag;
};

__device__ __forceinline__ float wsum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float wmax(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
// block sum / max over kT threads; result on every thread
__device__ float bsum(float v, Shared& sh) {
    v = wsum(v);
    if ((threadIdx.x & 31) == 0) sh.red[0][threadIdx.x >> 5] = v;
    __syncthreads();
    float a = 0.0f;
    for (int w = 0; w < kW; ++w) a += sh.red[0][w];
    __syncthreads();
    return a;
}
__device__ float bmax(float v, Shared& sh) {
    v = wmax(v);
    if ((threadIdx.x & 31) == 0) sh.red[0][threadIdx.x >> 5] = v;
    __syncthreads();
    float a = -1e30f;
    for (int w = 0; w < kW; ++w) a = fmaxf(a, sh.red[0][w]);
    __syncthreads();
    return a;
}

struct V2Noise {
    uint2 key;
    uint32_t tick;
    const svpf_v2_rng_t* r;
    int n;
    int* flag;
    __device__ float normal(int i, int k) const {
        if (r->tape_normals) {
            if (k >= r->slots_n) { *flag = SVPF_ERR_TAPE_SHORT; return 0.0f; }
            return r->tape_normals[(size_t)k * n + i];
        }
        const uint4 b = philox10(key, make_uint4((uint32_t)i, (uint32_t)k, tick, 0u));
        return normal_from_bits(b.x, b.y);
    }
    __device__ float uniform(int i, int k) const {
        if (r->tape_uniforms) {
            if (k >= r->slots_u) { *flag = SVPF_ERR_TAPE_SHORT; return 1.0f; }
            return r->tape_uniforms[(size_t)k * n + i];
        }
        const uint4 b = philox10(key, make_uint4((uint32_t)i, (uint32_t)k, tick, 1u));
        return uniform_from_bits(b.x);
    }
};

// Steps whose diffusion normals are drawn before the Stein loop (at most).
constexpr int kPreSteps = 17;

// Lanes per row: a power of two <= 32, as many as fill the CTA with a
// member's share of rows (nloc of them).
__host__ __device__ __forceinline__ int lanes_per_row(int nloc) {
    int S = 1;
    while (S < 32 && 2 * S * (nloc > 1 ? nloc : 1) <= kT) S <<= 1;
    return S;
}

// Padded length of the particle arrays (far positions, zero scores, far
// means beyond n): a multiple of 32 and of the 4 S columns one chunk sweep
// covers, so that the pair loops need no masks.
__host__ __device__ __forceinline__ int padded_rows(int n, int C) {
    const int S = lanes_per_row((n + C - 1) / C);
    const int m = 4 * S > 32 ? 4 * S : 32;
    return (n + m - 1) / m * m;
}

// Transport row sums of row i over four-column chunks (two columns per packed
// op): ks = sum K s_j, gk = sum d K^2 (x hess_j with Newton), and for full
// Newton Hw = sum hess_j K + 2/bw^2 K^2 |3 d^2/bw^2 - 1|, Ks = sum K; LAST adds
// the KSD row sum kd.  d = h_i - h_j, K = 1 / (1 + d^2/bw^2).
template <bool FULL, bool LAST>
__device__ __forceinline__ void v2_transport_row(const float* __restrict__ hc, const float* __restrict__ sg,
                                                 const float* __restrict__ shs, int nv, int q, int S, float hi,
                                                 float gi, float ib2, bool use_newton, float& ks, float& gk,
                                                 float& Hw, float& Ks, float& kd) {
    const float2 h2 = f2(hi), vib2 = f2(ib2);
    float2 ks2 = f2(0.0f), gk2 = f2(0.0f), hw2 = f2(0.0f), kk2 = f2(0.0f);
    float hwa = 0.0f;
    kd = 0.0f;
    for (int cb = q * 4; cb < nv; cb += 4 * S) {
        const float4 x4 = *reinterpret_cast<const float4*>(hc + cb);
        const float4 s4 = *reinterpret_cast<const float4*>(sg + cb);
        const float4 e4 = *reinterpret_cast<const float4*>(shs + cb);
        const float2 xx[2] = {make_float2(x4.x, x4.y), make_float2(x4.z, x4.w)};
        const float2 ss[2] = {make_float2(s4.x, s4.y), make_float2(s4.z, s4.w)};
        const float2 ee[2] = {make_float2(e4.x, e4.y), make_float2(e4.z, e4.w)};
#pragma unroll
        for (int hf = 0; hf < 2; ++hf) {
            const float2 diff = fma2(xx[hf], f2(-1.0f), h2);
            const float2 dist2 = mul2(mul2(diff, diff), vib2);
            const float2 b = add2(dist2, f2(1.0f));
            const float2 K = make_float2(rcp_approx(b.x), rcp_approx(b.y));
            const float2 K2 = mul2(K, K);
            ks2 = fma2(K, ss[hf], ks2);
            const float2 rep = mul2(diff, K2);
            gk2 = use_newton ? fma2(rep, ee[hf], gk2) : add2(gk2, rep);
            if (FULL) {
                hw2 = fma2(ee[hf], K, hw2);
                const float2 t = fma2(dist2, f2(3.0f), f2(-1.0f));
                hwa = fmaf(K2.x, fabsf(t.x), hwa);
                hwa = fmaf(K2.y, fabsf(t.y), hwa);
                kk2 = add2(kk2, K);
            }
            if (LAST) {
                const float dd[2] = {diff.x, diff.y}, d2[2] = {dist2.x, dist2.y}, kv[2] = {K.x, K.y},
                            k2v[2] = {K2.x, K2.y}, sj[2] = {ss[hf].x, ss[hf].y}, hj[2] = {ee[hf].x, ee[hf].y};
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const float rj = use_newton ? __fdividef(sj[c], 0.7f * hj[c] + 1e-8f) : sj[c];
                    const float gxk = -2.0f * dd[c] * ib2 * k2v[c];
                    const float hxy = 2.0f * ib2 * k2v[c] * (4.0f * d2[c] * kv[c] - 1.0f);
                    kd += kv[c] * gi * rj + gi * (-gxk) + rj * gxk + hxy;
                }
            }
        }
    }
    ks = ks2.x + ks2.y;
    gk = gk2.x + gk2.y;
    Hw = FULL ? hw2.x + hw2.y + 2.0f * ib2 * hwa : 0.0f;
    Ks = FULL ? kk2.x + kk2.y : 0.0f;
}

__global__ void __launch_bounds__(kT) v2_kernel(const __grid_constant__ Args a) {
    namespace cg = cooperative_groups;
    extern __shared__ __align__(16) float smem[];
    __shared__ Shared sh;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank(), C = (int)cl.num_blocks();
    const int tid = threadIdx.x;
    const int n = a.n;
    const int np = padded_rows(n, C);
    const int L = (n + C - 1) / C;
    const int row0 = min(rank * L, n), row1 = min(row0 + L, n);
    float* hb[2] = {smem, smem + np};
    float* sg = smem + 2 * np;       // transport score of every row
    float* shs = smem + 3 * np;      // sh_hess of every row
    float* muk = smem + 4 * np;      // prior means
    float* lwa = smem + 5 * np;      // log-weights (rank 0 gathers)
    float* kq = smem + 6 * np;       // KSD row sums (rank 0 gathers), np
    float* vr = smem + 7 * np;       // own rows: RMSProp moment
    float* zd = vr + L;              // own rows: pending diffusion normal
    float* gown = zd + L;            // own rows: clamped score g (the KSD's raw score of row i)
    float* zpre = gown + L;          // own rows: the diffusion normals of the first npre_cap steps, [npre_cap][L]
    const Params& P = a.p;
    const float y_t = a.y_t, y_prev = a.y_prev, hmp = a.h_mean_prev;
    const float rho = P.rho, sz = P.sigma_z, mu = P.mu, nu = P.nu;
    // ---- phase 0 (:190-267), every member; rank 0 writes back at the end
    if (tid == 0) {
        sh.flag = 0;
        sh.rng = *a.rng;
        sh.eff_mu = P.use_adaptive_mu ? *a.d_mu_state : mu;
        float prev_gm = *a.d_guide_mean, gv = *a.d_guide_var;
        if (gv < 1e-6f) {
            prev_gm = mu;
            gv = sz * sz / (1.0f - rho * rho);
        }
        float boost = 1.0f;
        if (P.use_adaptive_sigma && a.timestep > 0) {
            const float rz = fabsf(y_t) / fmaxf(a.vol_prev, 1e-4f);
            if (rz > P.sigma_boost_threshold) {
                const float sev = fminf((rz - P.sigma_boost_threshold) / 3.0f, 1.0f);
                boost = 1.0f + (P.sigma_boost_max - 1.0f) * sev;
            }
        }
        sh.eff_sigma = sz * boost;
        sh.write_guide = 0;
        if (P.use_guide) {
            const float m_pred = sh.eff_mu + rho * (prev_gm - sh.eff_mu);
            const float P_pred = rho * rho * gv + sz * sz;
            const float ly2 = logf(y_t * y_t + 1e-8f);
            const float S = P_pred + (4.93f + 2.0f);
            const float K = P_pred / (S + 1e-8f);
            const float innov = ly2 - (m_pred - P.student_t_implied_offset);
            sh.gm = m_pred + K * innov;
            sh.gv = (1.0f - K) * P_pred;
            sh.write_guide = 1;
            const float rz = fabsf(y_t) / fmaxf(a.vol_prev, 1e-4f);
            if (rz > P.guide_innovation_threshold) {
                const float sev = fminf((rz - P.guide_innovation_threshold) / 3.0f, 1.0f);
                sh.gs = P.guide_strength_base + (P.guide_strength_max - P.guide_strength_base) * sev;
            } else {
                sh.gs = P.guide_strength_base;
            }
        } else {
            sh.gm = hmp;
            sh.gv = 1.0f;
            sh.gs = 0.0f;
        }
    }
    __syncthreads();
    const V2Noise nz{philox_key(sh.rng.seed, (int)sh.rng.filter), sh.rng.tick, &sh.rng, n, &sh.flag};
    const float eff_mu = sh.eff_mu, eff_sigma = sh.eff_sigma;
    const float inv_s2 = 1.0f / (eff_sigma * eff_sigma), inv_2s2 = 0.5f * inv_s2;
    // ---- phase 1-2: predict and guide, all rows (:274-378)
    float* h = hb[0];
    for (int i = tid; i < np; i += kT) {
        if (i >= n) { hb[0][i] = 1e15f; hb[1][i] = 1e15f; sg[i] = 0.0f; shs[i] = 0.0f; muk[i] = 1e18f; continue; }
        const float h_old = a.h[i];
        muk[i] = eff_mu + rho * (h_old - eff_mu) + P.gamma * y_prev / (expf(h_old * 0.5f) + 1e-8f);
        float lrho = rho, lsig = eff_sigma;
        if (P.delta_rho > 0.0f || P.delta_sigma > 0.0f) {
            const float dev = h_old - hmp;
            lrho = fminf(fmaxf(rho + P.delta_rho * tanhf(dev), 0.0f), 0.999f);
            lsig = eff_sigma * (1.0f + P.delta_sigma * fabsf(dev));
        }
        float lev = 0.0f;
        if (fabsf(P.gamma) > 1e-6f) lev = P.gamma * y_prev / (expf(h_old * 0.5f) + 1e-8f);
        const float prior = eff_mu + lrho * (h_old - eff_mu) + lev;
        const float z = nz.normal(i, 0);
        const float jump = nz.uniform(i, 0) < P.mim_jump_prob ? 1.0f : 0.0f;
        const float msig = lsig * (1.0f + jump * (P.mim_jump_scale - 1.0f));
        float hi;
        if (P.use_guided_predict) {
            const float implied = fmaxf(logf(y_t * y_t + 1e-10f) + P.student_t_implied_offset, -5.0f);
            const float zs = (implied - prior) / 2.5f;
            const float act = zs > P.guided_innovation_thresh_predict ? tanhf(zs - P.guided_innovation_thresh_predict)
                                                                      : 0.0f;
            const float al = P.guided_alpha_base + (P.guided_alpha_shock - P.guided_alpha_base) * act;
            hi = (1.0f - al) * prior + al * implied + msig * z;
        } else {
            hi = prior + msig * z;
        }
        hi = clamp_h(hi);
        if (rank == 0) a.h_prev[i] = h_old;
        if (P.use_guide && sh.gs > 0.0f)
            hi = clamp_h(P.use_guide_preserving ? hi + sh.gs * (sh.gm - hmp) : (1.0f - sh.gs) * hi + sh.gs * sh.gm);
        h[i] = hi;
    }
    // own rows' moments; the diffusion normals, drawn in parallel up front:
    // entry g is draw 1 (g = 0) or draw 3 + g, the normal step g + 1 adds
    // (entry n_stein_steps is the draw the last step takes and leaves unused).
    // The row epilogue draws the rest one by one, so the set of draws is the
    // same whatever fits.
    const int nsteps = P.n_stein_steps < 1 ? 1 : P.n_stein_steps;
    const int npre = P.temperature > 1e-6f ? min(nsteps + 1, a.npre_cap) : 0;
    for (int li = tid; li < row1 - row0; li += kT) {
        vr[li] = a.v[row0 + li];
        if (npre == 0) zd[li] = nz.normal(row0 + li, 1);
    }
    for (int k = tid; k < npre * (row1 - row0); k += kT) {
        const int g = k / (row1 - row0), li = k - g * (row1 - row0);
        zpre[g * L + li] = nz.normal(row0 + li, g == 0 ? 1 : 3 + g);
    }
    __syncthreads();
    // ---- phase 3: Silverman bandwidth (:384-410)
    {
        float s = 0.0f;
        for (int i = tid; i < n; i += kT) s += h[i];
        const float mean = bsum(s, sh) / (float)n;
        float q = 0.0f;
        for (int i = tid; i < n; i += kT) q += (h[i] - mean) * (h[i] - mean);
        const float var = bsum(q, sh) / (float)n;
        if (tid == 0) {
            const float sd = sqrtf(fmaxf(var, 1e-6f));
            sh.bw = fminf(fmaxf(1.06f * sd * powf((float)n, -0.2f), 0.05f), 2.0f);
        }
        __syncthreads();
    }
    const float bw = sh.bw, ib2 = 1.0f / (bw * bw);
    cl.sync();   // every member has read a.h / a.v before anyone writes them
    // ---- phase 4: Stein loop (:416-640)
    const int na = P.n_anneal_steps < 1 ? 1 : P.n_anneal_steps;
    const int ns = P.n_stein_steps < 1 ? 1 : P.n_stein_steps;
    const int spa = ns / na, rem = ns - spa * na;
    const float sign = P.stein_sign_mode == 1 ? 1.0f : -1.0f;
    const float hess_prior = -inv_s2;
    const float nu1 = nu + 1.0f;
    const float y2 = y_t * y_t;
    int cur = 0, gstep = 0;
    const int kn0 = 4;
    // S lanes per row (a power of two <= 32 filling the CTA with L rows; the
    // same on every member, so that the padding covers its chunks), G rows
    // per sweep
    const int nloc = row1 - row0;
    const int S = lanes_per_row(L);
    const int G = kT / S;
    const int grp = tid / S, q = tid % S;
    const int nv = round_up(n, 4 * S);   // <= np: four columns per chunk, pads beyond n
    const float c2 = inv_2s2 * 1.4426950408889634f;   // log2(e) / (2 sigma^2)
    const bool use_newton = P.use_newton != 0, full = P.use_full_newton != 0;
    for (int ai = 0; ai < na; ++ai) {
        const float beta = (na <= 1 || ai == na - 1) ? 1.0f : 0.3f + ((float)ai / (float)(na - 1)) * 0.5f;
        const int si = spa + (ai == na - 1 ? rem : 0);
        for (int s = 0; s < si; ++s) {
            ++gstep;
            const bool last = gstep == ns;
            const float* hc = hb[cur];
            // gradient of own rows (S lanes per row split the columns); push
            // score and hess to every member
            for (int base = 0; base < nloc; base += G) {
                const int li = base + grp;
                const bool valid = li < nloc;
                const int i = valid ? row0 + li : 0;
                const float hi = hc[i];
                // row maximum of -d^2 c2: the smallest d^2 over the row's
                // columns (four per chunk, two per packed op; far-value pads)
                const float2 h2 = f2(hi);
                float mn = 3.0e38f;
                for (int cb = q * 4; cb < nv; cb += 4 * S) {
                    const float4 m4 = *reinterpret_cast<const float4*>(muk + cb);
                    const float2 da = fma2(make_float2(m4.x, m4.y), f2(-1.0f), h2);
                    const float2 db = fma2(make_float2(m4.z, m4.w), f2(-1.0f), h2);
                    const float2 qa = mul2(da, da), qb = mul2(db, db);
                    mn = fminf(mn, fminf(fminf(qa.x, qa.y), fminf(qb.x, qb.y)));
                }
                for (int o = S >> 1; o > 0; o >>= 1) mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
                const float lmax = -(mn * c2);
                float2 sr2 = f2(0.0f), wd2 = f2(0.0f);
                const float2 nc2 = f2(-c2), nl = f2(-lmax);
                for (int cb = q * 4; cb < nv; cb += 4 * S) {
                    const float4 m4 = *reinterpret_cast<const float4*>(muk + cb);
                    const float2 da = fma2(make_float2(m4.x, m4.y), f2(-1.0f), h2);
                    const float2 db = fma2(make_float2(m4.z, m4.w), f2(-1.0f), h2);
                    const float2 ta = fma2(mul2(da, da), nc2, nl), tb = fma2(mul2(db, db), nc2, nl);
                    const float2 wa = make_float2(ex2_approx(ta.x), ex2_approx(ta.y));
                    const float2 wb = make_float2(ex2_approx(tb.x), ex2_approx(tb.y));
                    sr2 = add2(sr2, wa);
                    wd2 = fma2(wa, da, wd2);
                    sr2 = add2(sr2, wb);
                    wd2 = fma2(wb, db, wd2);
                }
                float sr = sr2.x + sr2.y, wd = wd2.x + wd2.y;
                for (int o = S >> 1; o > 0; o >>= 1) {
                    sr += __shfl_xor_sync(0xffffffffu, sr, o);
                    wd += __shfl_xor_sync(0xffffffffu, wd, o);
                }
                if (!valid || q != 0) continue;
                const float gp = fminf(fmaxf(-wd * inv_s2 / (sr + 1e-8f), -10.0f), 10.0f);
                const float vol = expf(hi * 0.5f);
                const float A = y2 / (vol * vol + 1e-8f) / nu;
                const float opA = 1.0f + A;
                const float lwi = P.student_t_const - 0.5f * hi - 0.5f * nu1 * logf(opA);
                const float gl = -0.5f + 0.5f * nu1 * A / opA - P.lik_offset;
                const float g = fminf(fmaxf(gp + beta * gl, -10.0f), 10.0f);
                const float hl = -0.5f * nu1 * A / (opA * opA);
                const float curv = fminf(fmaxf(-(hl + hess_prior), 0.1f), 100.0f);
                const float invH = 1.0f / curv;
                float s_i, h_i;
                if (P.use_full_newton) { s_i = g; h_i = curv; }
                else if (P.use_newton) { s_i = 0.7f * g * invH; h_i = invH; }
                else { s_i = g; h_i = 1.0f; }
                a.grad[i] = g;
                if (P.use_newton || P.use_full_newton) a.inv_hess[i] = curv;
                for (int r = 0; r < C; ++r) {
                    cl.map_shared_rank(sg, r)[i] = s_i;
                    cl.map_shared_rank(shs, r)[i] = h_i;
                }
                if (last) cl.map_shared_rank(lwa, 0)[i] = lwi;
                gown[li] = g;   // the reference keeps it in a register
            }
            cl.sync();
            // transport of own rows; push new positions to every member
            float* hn = hb[cur ^ 1];
            const float es = P.step_size * sqrtf(beta);
            for (int base = 0; base < nloc; base += G) {
                const int li = base + grp;
                const bool valid = li < nloc;
                const int i = valid ? row0 + li : 0;
                const float hi = hc[i];
                const float gi = valid ? gown[li] : 0.0f;
                float ks, gk, Hw, Ks, kd;
                if (full) {
                    if (last) v2_transport_row<true, true>(hc, sg, shs, nv, q, S, hi, gi, ib2, use_newton, ks, gk, Hw, Ks, kd);
                    else v2_transport_row<true, false>(hc, sg, shs, nv, q, S, hi, gi, ib2, use_newton, ks, gk, Hw, Ks, kd);
                } else {
                    if (last) v2_transport_row<false, true>(hc, sg, shs, nv, q, S, hi, gi, ib2, use_newton, ks, gk, Hw, Ks, kd);
                    else v2_transport_row<false, false>(hc, sg, shs, nv, q, S, hi, gi, ib2, use_newton, ks, gk, Hw, Ks, kd);
                }
                for (int o = S >> 1; o > 0; o >>= 1) {
                    ks += __shfl_xor_sync(0xffffffffu, ks, o);
                    gk += __shfl_xor_sync(0xffffffffu, gk, o);
                    if (full) {
                        Hw += __shfl_xor_sync(0xffffffffu, Hw, o);
                        Ks += __shfl_xor_sync(0xffffffffu, Ks, o);
                    }
                    if (last) kd += __shfl_xor_sync(0xffffffffu, kd, o);
                }
                if (!valid || q != 0) continue;
                gk *= sign * 2.0f * ib2;
                float phi;
                if (full) {
                    const float H = fminf(fmaxf(Hw / fmaxf(Ks, 1e-6f), 0.1f), 100.0f);
                    phi = (ks + gk) / (float)n * (1.0f / H) * 0.7f;
                } else {
                    phi = (ks + gk) / (float)n;
                }
                const float vn = P.rmsprop_rho * vr[li] + (1.0f - P.rmsprop_rho) * phi * phi;
                vr[li] = vn;
                const float drift = es * phi * rsqrtf(vn + P.rmsprop_eps);
                float diffu = 0.0f;
                if (P.temperature > 1e-6f) {
                    diffu = sqrtf(2.0f * es * P.temperature) * (gstep - 1 < npre ? zpre[(gstep - 1) * L + li] : zd[li]);
                    if (gstep >= npre) zd[li] = nz.normal(i, kn0 + gstep - 1);   // past the pre-drawn steps
                }
                const float hnew = clamp_h(hi + drift + diffu);
                for (int r = 0; r < C; ++r) cl.map_shared_rank(hn, r)[i] = hnew;
                if (last) cl.map_shared_rank(kq, 0)[i] = kd;
            }
            cl.sync();
            cur ^= 1;
        }
    }
    // own rows' moments back
    for (int li = tid; li < row1 - row0; li += kT) a.v[row0 + li] = vr[li];
    if (rank != 0) return;
    // ---- phase 5: rejuvenation (:646-658), rank 0, all rows
    h = hb[cur];
    const int kn_rejuv = kn0 + (P.temperature > 1e-6f ? ns : 0);
    if (P.use_rejuvenation && a.ksd_prev > P.rejuv_ksd_threshold && a.timestep > 10) {
        for (int i = tid; i < n; i += kT) {
            if (nz.uniform(i, 1) < P.rejuv_prob) {
                const float gstd = sqrtf(fmaxf(sh.gv, 1e-6f));
                const float target = sh.gm + gstd * nz.normal(i, kn_rejuv);
                h[i] = clamp_h((1.0f - P.rejuv_blend) * h[i] + P.rejuv_blend * target);
            }
        }
    }
    __syncthreads();
    // ---- phase 6: outputs (:664-706)
    float s1 = 0.0f, s2 = 0.0f, s3 = 0.0f, mx = -1e10f;
    for (int i = tid; i < n; i += kT) {
        s1 += kq[i];
        s2 += h[i];
        s3 += expf(h[i] * 0.5f);
        mx = fmaxf(mx, lwa[i]);
    }
    const float ksum = bsum(s1, sh), hsum = bsum(s2, sh), vsum = bsum(s3, sh);
    mx = bmax(mx, sh);
    float s4 = 0.0f;
    for (int i = tid; i < n; i += kT) s4 += expf(lwa[i] - mx);
    const float wsumv = bsum(s4, sh);
    for (int i = tid; i < n; i += kT) {
        a.h[i] = h[i];
        a.lw[i] = lwa[i];
    }
    if (tid == 0) {
        const float inv_n = 1.0f / (float)n;
        const float hm = hsum * inv_n;
        *a.d_ksd = sqrtf(fmaxf(ksum * inv_n * inv_n, 0.0f));
        *a.d_h_mean = hm;
        *a.d_vol = vsum * inv_n;
        *a.d_loglik = mx + logf(fmaxf(wsumv, 1e-10f) * inv_n);
        *a.d_bw = sh.bw;
        if (sh.write_guide) {
            *a.d_guide_mean = sh.gm;
            *a.d_guide_var = sh.gv;
        }
        if (P.use_adaptive_mu && a.timestep > 10) {
            const float mo = *a.d_mu_state;
            *a.d_mu_state = fminf(fmaxf(P.mu_ema_alpha * hm + (1.0f - P.mu_ema_alpha) * mo, -10.0f), 0.0f);
        }
        a.rng->tick = sh.rng.tick + 1;
        a.rng->status = sh.flag;
    }
}

}  // namespace v2
}  // namespace svpf

using namespace svpf;

namespace {

// Dynamic shared memory of one member: seven padded particle arrays, then
// three own-row arrays and `pre` pre-drawn normals per own row.
size_t v2_smem_bytes(int n, int C, int pre) {
    const int np = v2::padded_rows(n, C);
    const int L = (n + C - 1) / C;
    return (size_t)(7 * np + (3 + pre) * L) * sizeof(float);
}

// Dynamic shared memory a v2 member may take: the device's opt-in limit per
// block less the kernel's own static shared memory.
size_t v2_smem_cap() {
    static std::mutex mu;
    static size_t cached[kMaxDevices] = {};
    const int dev = current_device();
    if (dev < 0) return 0;
    std::lock_guard<std::mutex> lk(mu);
    if (cached[dev] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
        cudaFuncAttributes fa{};
        if (cudaFuncGetAttributes(&fa, v2::v2_kernel) != cudaSuccess) return 0;
        cached[dev] = (size_t)v > fa.sharedSizeBytes ? (size_t)v - fa.sharedSizeBytes : 0;
    }
    return cached[dev];
}

int v2_cluster(int n) {
    int C = default_cluster(n);
    while (C > 1 && v2_smem_bytes(n, C, 0) > v2_smem_cap()) C >>= 1;
    return C;
}

// Pre-drawn steps that fit beside the cluster's arrays (up to kPreSteps).
int v2_pre_steps(int n, int C) {
    const size_t base = v2_smem_bytes(n, C, 0), cap = v2_smem_cap();
    if (base >= cap) return 0;
    const size_t row = (size_t)((n + C - 1) / C) * sizeof(float);
    const size_t fit = (cap - base) / row;
    return (int)(fit < (size_t)v2::kPreSteps ? fit : (size_t)v2::kPreSteps);
}

}  // namespace

extern "C" {

bool svpf_fully_fused_v2_supported(int n_particles) {
    return n_particles >= 1 && n_particles <= SVPF_MAX_PARTICLES &&
           v2_smem_bytes(n_particles, 16, 0) <= v2_smem_cap();
}

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
    int n_anneal_steps, int stein_sign_mode, int n, int timestep, cudaStream_t stream) {
    SVPF_TRACE();
    if (!svpf_fully_fused_v2_supported(n)) return cudaErrorInvalidConfiguration;
    if (n_stein_steps > SVPF_MAX_STEIN_STEPS || n_anneal_steps > SVPF_MAX_ANNEAL_STEPS)
        return cudaErrorInvalidValue;   // bounded loop counts: no call keeps the kernel running for long
    if (!h || !h_prev || !grad_log_p || !log_weights || !d_grad_v || !d_inv_hessian || !rng || !d_h_mean ||
        !d_vol || !d_loglik || !d_bandwidth || !d_ksd || !d_guide_mean || !d_guide_var || !d_mu_state)
        return cudaErrorInvalidValue;
    v2::Args a;
    std::memset(&a, 0, sizeof(a));
    a.h = h; a.h_prev = h_prev; a.grad = grad_log_p; a.lw = log_weights; a.v = d_grad_v; a.inv_hess = d_inv_hessian;
    a.rng = rng;
    a.y_t = y_t; a.y_prev = y_prev; a.h_mean_prev = h_mean_prev; a.vol_prev = vol_prev; a.ksd_prev = ksd_prev;
    a.d_h_mean = d_h_mean; a.d_vol = d_vol; a.d_loglik = d_loglik; a.d_bw = d_bandwidth; a.d_ksd = d_ksd;
    a.d_guide_mean = d_guide_mean; a.d_guide_var = d_guide_var; a.d_mu_state = d_mu_state;
    v2::Params& p = a.p;
    p.rho = rho; p.sigma_z = sigma_z; p.mu = mu; p.nu = nu; p.lik_offset = lik_offset;
    p.student_t_const = student_t_const; p.student_t_implied_offset = student_t_implied_offset; p.gamma = gamma;
    p.delta_rho = delta_rho; p.delta_sigma = delta_sigma; p.mim_jump_prob = mim_jump_prob;
    p.mim_jump_scale = mim_jump_scale; p.guide_strength_base = guide_strength_base;
    p.guide_strength_max = guide_strength_max; p.guide_innovation_threshold = guide_innovation_threshold;
    p.guided_alpha_base = guided_alpha_base; p.guided_alpha_shock = guided_alpha_shock;
    p.guided_innovation_thresh_predict = guided_innovation_thresh_predict; p.use_guide = use_guide;
    p.use_guided_predict = use_guided_predict; p.use_guide_preserving = use_guide_preserving;
    p.use_newton = use_newton; p.use_full_newton = use_full_newton; p.use_rejuvenation = use_rejuvenation;
    p.rejuv_ksd_threshold = rejuv_ksd_threshold; p.rejuv_prob = rejuv_prob; p.rejuv_blend = rejuv_blend;
    p.use_adaptive_mu = use_adaptive_mu; p.mu_ema_alpha = mu_ema_alpha; p.use_adaptive_sigma = use_adaptive_sigma;
    p.sigma_boost_threshold = sigma_boost_threshold; p.sigma_boost_max = sigma_boost_max;
    p.step_size = step_size; p.temperature = temperature; p.rmsprop_rho = rmsprop_rho; p.rmsprop_eps = rmsprop_eps;
    p.n_stein_steps = n_stein_steps; p.n_anneal_steps = n_anneal_steps; p.stein_sign_mode = stein_sign_mode;
    a.n = n;
    a.timestep = timestep;
    const int C = v2_cluster(n);
    a.npre_cap = v2_pre_steps(n, C);
    {
        const cudaError_t e = configure_kernel((const void*)v2::v2_kernel, (int)v2_smem_cap(), true);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C, 1, 1);
    cfg.blockDim = dim3(v2::kT, 1, 1);
    cfg.dynamicSmemBytes = v2_smem_bytes(n, C, a.npre_cap);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, v2::v2_kernel, a);
}

svpf_v2_rng_t* svpf_fully_fused_v2_rng_create(unsigned long long seed, unsigned int filter) {
    svpf_v2_rng_t h;
    std::memset(&h, 0, sizeof(h));
    h.seed = seed;
    h.filter = filter;
    svpf_v2_rng_t* d = nullptr;
    if (cudaMalloc(&d, sizeof(h)) != cudaSuccess) return nullptr;
    if (cudaMemcpy(d, &h, sizeof(h), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d);
        return nullptr;
    }
    return d;
}

void svpf_fully_fused_v2_rng_destroy(svpf_v2_rng_t* rng) { cudaFree(rng); }

int svpf_fully_fused_v2_rng_get(const svpf_v2_rng_t* rng, svpf_v2_rng_t* host) {
    if (!rng || !host) return SVPF_ERR_INVALID_ARG;
    return cudaMemcpy(host, rng, sizeof(*host), cudaMemcpyDeviceToHost) == cudaSuccess ? SVPF_OK : SVPF_ERR_CUDA;
}

int svpf_fully_fused_v2_rng_set(svpf_v2_rng_t* rng, const svpf_v2_rng_t* host) {
    if (!rng || !host) return SVPF_ERR_INVALID_ARG;
    return cudaMemcpy(rng, host, sizeof(*host), cudaMemcpyHostToDevice) == cudaSuccess ? SVPF_OK : SVPF_ERR_CUDA;
}

}  // extern "C"
