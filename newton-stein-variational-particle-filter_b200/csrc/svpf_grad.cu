// svpf_grad.cu -- gradient of a run's log-likelihood, sum_t w_t loglik_t,
// with respect to theta = (mu, rho, sigma_z, nu) of every filter of a batch,
// under common random numbers (the project's counter-based Philox draws are
// replayed exactly), by a hand-written reverse-mode adjoint of the tick.
//
// Forward: one CTA per filter runs the ticks of a segment of k ticks and
// stores a checkpoint (state, particles, RMSProp moments) at the start of
// every segment.  Backward, segment by segment from the last: the CTA
// recomputes the segment from its checkpoint and keeps every tick's input
// state, then walks the ticks in reverse; for each tick it recomputes the tick
// once more while recording every Stein iterate and the per-row statistics
// the adjoint needs, and then sweeps the Stein iterations backwards.
//
// Differentiable configuration (svpf_grad_supported): single factor; plain or
// MIM predict with the model's rho (svpf_opt_kernels.cu:125-206); EKF guide,
// preserving or blending, with the base strength (svpf_kernels.cuh:509-541,
// svpf_optimized_graph.cu:1006-1039); Gaussian mixture prior and Student-t
// likelihood (svpf_opt_kernels.cu:354-521); vanilla IMQ or full-Newton
// transport with RMSProp and SVLD (:527-599, :912-1103); no rejuvenation and
// no adaptive mu/sigma/guide.  Decisions that are piecewise constant in theta
// (the KSD-driven Stein budget, adaptive beta, the MIM jump selection) are
// taken as in the forward pass; clamps contribute their one-sided derivative.
//
// Adjoint of one Stein iteration (x = positions, u = (x_i - x_j)/bw,
// K = 1/(1+u^2), a_i = dL/dphi_raw_i / n, s = repulsion sign):
//   phi_raw_i = (1/n) sum_j [K g_j + 2 s u K^2 / bw]
//   dx_i += (1/bw) [a_i (-2 S1 + 2 s S2/bw) - 2 g_i C1 - 2 s C2/bw]
//     S1 = sum_j g_j u K^2, S2 = sum_j K^2 (4K-3), C1 = sum_j a_j u K^2,
//     C2 = sum_j a_j K^2 (4K-3)   (d(uK^2)/du = K^2 (4K-3); column terms
//     written as row sums with u_ji = -u_ij)
//   dg_i = sum_j a_j K,  dbw += a_i (1/bw) [2 Q1 - 2 s Q2/bw],
//     Q1 = sum_j g_j u^2 K^2, Q2 = sum_j u K^2 (4K-2)
// and for full Newton H_i = hw_i/kn_i, hw_i = sum_j [c_j K + 2K^2 |3u^2-1|/bw^2],
// kn_i = sum_j K, the analogous row and column sums of their derivatives.
// Gaussian mixture score gp(x) = -E_w[d]/s2, d_k = x - mu_k, w = softmax(-d^2/2s2):
//   dgp/dx = -1/s2 + Var_w(d)/s2^2
//   dgp/ds2 = E[d]/s2^2 - (E[d^3] - E[d] E[d^2]) / (2 s2^3)
//   dgp/dmu_k = (w_k/s2) [1 - d_k (d_k - E[d]) / s2]   (a column pass)
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <vector>

#include "svpf.h"
#include "svpf_device.cuh"
#include "svpf_internal.h"
#include "svpf_math.h"
#include "svpf_trace.h"

namespace svpf {
namespace grad {

constexpr int kRecFixed = 4;       // XS, HPR, HGR, MUK
constexpr int kRecPerIt = 15;      // X V GPRE AL LMAX Z DBAR VARD SKEW PHIR HR HW KN XR NK
enum { XS = 0, HPR = 1, HGR = 2, MUK = 3 };
enum { IX = 0, IV, IGPRE, IAL, ILMAX, IZ, IDBAR, IVARD, ISKEW, IPHIR, IHR, IHW, IKN, IXR, INK };

struct GState {
    double m, P;                   // EKF guide mean / variance
    float bw_sq, h_mean_prev, return_ema, return_var, ksd_prev;
    int guide_init, timestep, pad;
};

struct GAdj {
    double m, P, bw_sq, h_mean;    // adjoints of the scalar state
    double th[4];                  // accumulated d/d(mu, rho, sigma_z, nu)
};

struct TickScalars;

struct GArgs {
    int F, T, k, np, bmax;
    const int* n;
    const svpf_config_t* cfg;
    const float* theta;            // [F][4]
    const float* gamma;            // [F] or nullptr
    const float* y;                // [F][T]
    const float* w;                // [F][T] or nullptr (all ones)
    float* loglik;                 // [F][T] or nullptr
    double* ll_sum;                // [F]
    unsigned long long seed;
    // per filter
    float* fx;                     // [F][np] forward positions
    float* fv;                     // [F][np]
    GState* fs;                    // [F]
    float* ck;                     // [F][nseg][2 np] checkpoints (x, v)
    GState* cks;                   // [F][nseg]
    float* ax;                     // [F][np] adjoint of positions
    float* av;                     // [F][np]
    GAdj* as;                      // [F]
    // per CTA
    float* seg;                    // [grid][k][2 np] tick inputs of the segment
    GState* segs;                  // [grid][k]
    float* rec;                    // [grid][k or 1][rec_floats] per-tick records
    size_t rec_floats;
    TickScalars* segts;            // [grid][k] the ticks' scalars (segment records)
    int seg_rec;                   // 1: record the whole segment in one forward
    // run records: the forward keeps every tick's record (nullptr: recompute)
    float* run_rec;                // [F][T_max][rec_floats]
    GState* run_st;                // [F][T_max] state at each tick's start
    TickScalars* run_ts;           // [F][T_max] the ticks' scalars
    int T_max;
    int trunc;                     // > 0: truncated backpropagation every trunc ticks
    int nseg;
    int* status;                   // [F]
    int objective;                 // 0: the tick's log-likelihood, 1: predictive log p(y_t | y_1:t-1)
};

__host__ __device__ inline size_t rec_floats_for(int np, int bmax) {
    return (size_t)np * (kRecFixed + kRecPerIt * bmax + 2);
}

// ---- block reductions over kThreads threads ----------------------------------
template <int K>
__device__ __forceinline__ void reduce_sum(float (&v)[K], float (*scr)[kWarps]) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < K; ++q) {
        v[q] = warp_sum(v[q]);
        if (lane == 0) scr[q][wp] = v[q];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; ++q) {
        float a = 0.0f;
        for (int i = 0; i < kWarps; ++i) a += scr[q][i];
        v[q] = a;
    }
    __syncthreads();
}
__device__ __forceinline__ float reduce_max(float v, float (*scr)[kWarps]) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    v = warp_max(v);
    if (lane == 0) scr[0][wp] = v;
    __syncthreads();
    float a = scr[0][0];
    for (int i = 1; i < kWarps; ++i) a = fmaxf(a, scr[0][i]);
    __syncthreads();
    return a;
}
// (value, index) minimum / maximum; ties go to the smaller index
__device__ __forceinline__ void reduce_argminmax(float& mn, int& imn, float& mx, int& imx, float (*scr)[kWarps],
                                                 int* iscr) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float m2 = __shfl_xor_sync(0xffffffffu, mn, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, imn, o);
        if (m2 < mn || (m2 == mn && i2 < imn)) { mn = m2; imn = i2; }
        const float x2 = __shfl_xor_sync(0xffffffffu, mx, o);
        const int j2 = __shfl_xor_sync(0xffffffffu, imx, o);
        if (x2 > mx || (x2 == mx && j2 < imx)) { mx = x2; imx = j2; }
    }
    if (lane == 0) {
        scr[0][wp] = mn; iscr[wp] = imn;
        scr[1][wp] = mx; iscr[kWarps + wp] = imx;
    }
    __syncthreads();
    mn = scr[0][0]; imn = iscr[0]; mx = scr[1][0]; imx = iscr[kWarps];
    for (int i = 1; i < kWarps; ++i) {
        if (scr[0][i] < mn || (scr[0][i] == mn && iscr[i] < imn)) { mn = scr[0][i]; imn = iscr[i]; }
        if (scr[1][i] > mx || (scr[1][i] == mx && iscr[kWarps + i] < imx)) { mx = scr[1][i]; imx = iscr[kWarps + i]; }
    }
    __syncthreads();
}

// Per-tick scalars shared by the forward and the backward of one tick.
struct TickScalars {
    float mu, rho, sz, nu, gamma, s2;
    float y_t, y_prev, stc, off, gs, cm, gm;
    double m_in, P_in, m_pred, P_pred, K;
    int init_here;
    float mean, var, mn, mx;
    int imn, imx;
    float bw2_new_raw, bw2_prev, pre, ratio, spread_f, comb, scale_raw, bw2, bw, ib;
    int budget, na;
    float es[64], beta[64];
    float mxl, se;
    float mxp, sep;                // predictive log-likelihood: max and sum of exp
    float ksd_last;
};

struct Shared {
    float red[8][kWarps];
    int ired[2 * kWarps];
    TickScalars ts;
    GState st;
    int flag;
    int bad;          // this filter's theta is outside the domain (theta_ok)
    double acc[8];
};

// Stage of Stein iteration `it` (budget split as the reference host loop).
__device__ inline int stage_of_it(int it, int budget, int na) {
    const int si = budget / na;
    if (si == 0) return na - 1;
    const int a = it / si;
    return a < na - 1 ? a : na - 1;
}

// ---- pair loops ------------------------------------------------------------
// Every O(N^2) pass handles two rows per thread in packed FP32x2 (one issue
// slot for both rows) over columns read four at a time; columns past n hold a
// far value (positions) or zero (weights) so their terms vanish.
//
// Mixture prior in scaled coordinates x' = x psc, psc^2 = log2(e) / (2 s2):
// exp(-(x - m)^2 / (2 s2)) = 2^-(x' - m')^2.  The row maximum is the nearest
// sorted mean (binary search: the same value as a scan over all means), so a
// pair is one FADD2, one FFMA2, one ex2 per row and the accumulations.

__device__ __forceinline__ int mix_len(int n, int np) {
    const int p2 = pow2_at_least(n);
    const int a = p2 > np ? p2 : np;
    return round_up(a, 4);
}

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }

// Sums over the sorted scaled means of w = 2^-(x' - m')^2 + min: sr = sum w,
// wg = sum w d', and with MOM the moments m2 = sum w d'^2, m3 = sum w d'^3.
template <bool MOM>
__device__ __forceinline__ void mixture_rows(const float* __restrict__ srt, int nk4, float2 xs2, float2 ndm,
                                             float2& sr, float2& wg, float2& m2, float2& m3) {
    for (int cb = 0; cb < nk4; cb += 4) {
        const float4 m4 = ld4(srt + cb);
        const float mm[4] = {m4.x, m4.y, m4.z, m4.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float2 d = add2(xs2, f2(-mm[e]));
            const float2 q = fma2(d, d, ndm);
            const float2 w = make_float2(ex2_approx(-q.x), ex2_approx(-q.y));
            sr = add2(sr, w);
            wg = fma2(w, d, wg);   // identical with and without the moments: records replay the forward
            if (MOM) {
                const float2 wdd = mul2(mul2(w, d), d);
                m2 = add2(m2, wdd);
                m3 = fma2(wdd, d, m3);
            }
        }
    }
}

// Transport row sums, u = (x_i - x_j)/bw, K = 1/(1 + u^2):
//   kg = sum K g_j, gk = sum u K^2; FULL: ks = sum K, kc = sum K c_j,
//   nk = sum K^2 |3u^2 - 1| = sum K |3 - 4K|; KSD: gdk = sum g_j u K^2,
//   ht = sum K^2 (3 - 4K)  (4 u^2 K - 1 = 3 - 4K).
template <bool FULL, bool KSD>
__device__ __forceinline__ void transport_rows(const float* __restrict__ x, const float* __restrict__ g,
                                               const float* __restrict__ cv, int nk4, float2 xi2, float ib,
                                               float2& kg, float2& gk, float2& ks, float2& kc, float2& nk,
                                               float2& gdk, float2& ht) {
    const float2 mib = f2(-ib);
    for (int cb = 0; cb < nk4; cb += 4) {
        const float4 x4 = ld4(x + cb), g4 = ld4(g + cb);
        float4 c4 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (FULL) c4 = ld4(cv + cb);
        const float xx[4] = {x4.x, x4.y, x4.z, x4.w};
        const float gg[4] = {g4.x, g4.y, g4.z, g4.w};
        const float cc[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float2 u = fma2(f2(xx[e]), mib, xi2);
            const float2 b = fma2(u, u, f2(1.0f));
            const float2 K = make_float2(rcp_approx(b.x), rcp_approx(b.y));
            const float2 K2 = mul2(K, K);
            kg = fma2(K, f2(gg[e]), kg);
            const float2 uk2 = mul2(u, K2);
            gk = add2(gk, uk2);
            if (FULL || KSD) {
                const float2 t = fma2(K, f2(-4.0f), f2(3.0f));
                if (FULL) {
                    ks = add2(ks, K);
                    kc = fma2(K, f2(cc[e]), kc);
                    const float2 kt = mul2(K, t);
                    nk.x += fabsf(kt.x);
                    nk.y += fabsf(kt.y);
                }
                if (KSD) {
                    gdk = fma2(f2(gg[e]), uk2, gdk);
                    ht = fma2(K2, t, ht);
                }
            }
        }
    }
}

__device__ __forceinline__ float flip_sign(float v, float s) {
    return __int_as_float(__float_as_int(v) ^ (__float_as_int(s) & 0x80000000));
}

// The pair loops form u = x_j (-1/bw) + x_i/bw in one FMA: the column's
// product is exact, the row's x_i/bw was rounded once, so a row's own column
// (j = i) enters with u = that rounding error instead of 0.  Its terms that
// are odd in u (u K^2 and what it weights) are then spurious: with one
// particle at the bandwidth floor (1/bw = 100) the repulsion picks up
// 2 u / bw ~ 1e-3.  self_uk2 gives the loop's own value of u K^2 for j = i
// (and K, for the Hessian term), so the row sums can take it back out.
__device__ __forceinline__ float2 self_uk2(float2 xr, float2 xi2, float ib, float2& K) {
    const float2 u = fma2(xr, f2(-ib), xi2);
    const float2 b = fma2(u, u, f2(1.0f));
    K = make_float2(rcp_approx(b.x), rcp_approx(b.y));
    return mul2(u, mul2(K, K));
}

// Transport adjoint row sums (the row and column terms of one Stein
// iteration, see the header), with K^2 |3u^2-1| = K |3-4K| and
// uK^2 (6 sgn - 4 K |3u^2-1|) = sgn(3-4K) uK^2 (16K - 6).  Accumulators:
//   0 S1 = sum g uK2     1 -S2 = sum K2 t      2 C1 = sum a uK2
//   3 -C2 = sum a K2 t   4 C3 = sum a K        5 R3 = sum uK2       (t = 3 - 4K)
//   FULL: 6 R1 = sum c uK2, 7 R2 = sum f6, 8 D1 = sum hb uK2, 9 D2 = sum hb f6,
//   10 D3 = sum kb uK2, 11 E1 = sum hb K.
// The bandwidth adjoint takes no pair sums of its own (bwd_tick derives it
// from the position adjoint by homogeneity).
constexpr int kAdjAcc = 12;
template <bool FULL>
__device__ __forceinline__ void adjoint_rows(const float* __restrict__ xs, const float* __restrict__ g,
                                             const float* __restrict__ a, const float* __restrict__ cv,
                                             const float* __restrict__ hwb, const float* __restrict__ knb, int nk4,
                                             float2 xi2, float ib, float2 (&acc)[kAdjAcc]) {
    const float2 mib = f2(-ib);
    for (int cb = 0; cb < nk4; cb += 4) {
        const float4 x4 = ld4(xs + cb), g4 = ld4(g + cb), a4 = ld4(a + cb);
        float4 c4 = make_float4(0.f, 0.f, 0.f, 0.f), h4 = c4, k4 = c4;
        if (FULL) {
            c4 = ld4(cv + cb);
            h4 = ld4(hwb + cb);
            k4 = ld4(knb + cb);
        }
        const float xx[4] = {x4.x, x4.y, x4.z, x4.w};
        const float gg[4] = {g4.x, g4.y, g4.z, g4.w};
        const float aa[4] = {a4.x, a4.y, a4.z, a4.w};
        const float cc[4] = {c4.x, c4.y, c4.z, c4.w};
        const float hh[4] = {h4.x, h4.y, h4.z, h4.w};
        const float kk[4] = {k4.x, k4.y, k4.z, k4.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float2 u = fma2(f2(xx[e]), mib, xi2);
            const float2 b = fma2(u, u, f2(1.0f));
            const float2 K = make_float2(rcp_approx(b.x), rcp_approx(b.y));
            const float2 K2 = mul2(K, K);
            const float2 uk2 = mul2(u, K2);
            const float2 t = fma2(K, f2(-4.0f), f2(3.0f));
            const float2 k2t = mul2(K2, t);
            const float2 gj = f2(gg[e]), aj = f2(aa[e]);
            acc[0] = fma2(gj, uk2, acc[0]);
            acc[1] = add2(acc[1], k2t);
            acc[2] = fma2(aj, uk2, acc[2]);
            acc[3] = fma2(aj, k2t, acc[3]);
            acc[4] = fma2(aj, K, acc[4]);
            acc[5] = add2(acc[5], uk2);
            if (FULL) {
                const float2 f6u = mul2(uk2, fma2(K, f2(16.0f), f2(-6.0f)));
                const float2 f6 = make_float2(flip_sign(f6u.x, t.x), flip_sign(f6u.y, t.y));
                const float2 cj = f2(cc[e]), hj = f2(hh[e]);
                acc[6] = fma2(cj, uk2, acc[6]);
                acc[7] = add2(acc[7], f6);
                acc[8] = fma2(hj, uk2, acc[8]);
                acc[9] = fma2(hj, f6, acc[9]);
                acc[10] = fma2(f2(kk[e]), uk2, acc[10]);
                acc[11] = fma2(hj, K, acc[11]);
            }
        }
    }
}

// Mixture column sums for dL/dmu_k (rows are prior means k, scaled mk2):
//   sum_j coef_j r_kj (1 - 2 ln2 d' (d' - dbar'_j)),  r_kj = 2^-(d'^2 - lmin'_j),
//   d' = x_j psc - m'_k.
__device__ __forceinline__ float2 mixture_cols(const float* __restrict__ xs, const float* __restrict__ lmx,
                                               const float* __restrict__ dbr, const float* __restrict__ coef, int nk4,
                                               float psc, float2 mk2) {
    const float2 nmk = make_float2(-mk2.x, -mk2.y);
    float2 acc = f2(0.0f);
    for (int cb = 0; cb < nk4; cb += 4) {
        const float4 x4 = ld4(xs + cb), l4 = ld4(lmx + cb), d4 = ld4(dbr + cb), c4 = ld4(coef + cb);
        const float xx[4] = {x4.x, x4.y, x4.z, x4.w};
        const float ll[4] = {l4.x, l4.y, l4.z, l4.w};
        const float db[4] = {d4.x, d4.y, d4.z, d4.w};
        const float co[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float2 d = fma2(f2(xx[e]), f2(psc), nmk);
            const float2 q = fma2(d, d, f2(-ll[e]));
            const float2 r = make_float2(ex2_approx(-q.x), ex2_approx(-q.y));
            const float2 uu = mul2(d, add2(d, f2(-db[e])));
            const float2 fct = fma2(uu, f2(-2.0f * kLn2), f2(1.0f));
            acc = fma2(mul2(r, f2(co[e])), fct, acc);
        }
    }
    return acc;
}

// One tick of one filter (CTA-wide).  x, v: positions and RMSProp moments
// (smem, updated in place; x has room for round_up(n, 4) columns); work:
// 5 np + mix_len floats of smem scratch.  rec: per-tick
// record for the backward, or nullptr.  Returns loglik on every thread.
__device__ float fwd_tick(const svpf_config_t& c, int n, int np, float* x, float* v, float* work, Shared& sh,
                          const Noise& nz, float y_t, float y_prev, float* rec, int bmax, int objective) {
    const int tid = threadIdx.x;
    TickScalars& ts = sh.ts;
    GState& st = sh.st;
    float* xn = work;                 // next positions
    float* g = work + np;             // transport score (clamped)
    float* curv = work + 2 * np;      // full-Newton curvature
    float* lw = work + 3 * np;        // log-weights of the last gradient pass
    float* muk = work + 4 * np;       // prior means
    float* srt = work + 5 * np;       // prior means scaled and sorted (mix_len floats)
    const bool full = c.use_newton && c.use_full_newton;
    if (tid == 0) {
        ts.y_t = y_t;
        ts.y_prev = y_prev;
        ts.s2 = ts.sz * ts.sz;
        ts.stc = lgammaf((ts.nu + 1.0f) * 0.5f) - lgammaf(ts.nu * 0.5f) - 0.5f * logf(3.14159265358979f * ts.nu);
        ts.off = c.student_t_implied_offset;
        ts.gs = c.guide_strength_base;
        ts.cm = st.h_mean_prev;
        // EKF guide in FP64 (svpf_kernels.cuh:509-541)
        if (c.use_guide) {
            const double mu = ts.mu, rho = ts.rho, sz = ts.sz;
            ts.init_here = st.guide_init ? 0 : 1;
            double m = st.m, P = st.P;
            if (!st.guide_init) {
                m = mu;
                P = sz * sz / (1.0 - rho * rho);
                st.guide_init = 1;
            }
            ts.m_in = m;
            ts.P_in = P;
            ts.m_pred = mu + rho * (m - mu);
            ts.P_pred = rho * rho * P + sz * sz;
            ts.K = ts.P_pred / (ts.P_pred + 6.93 + 1e-8);
            const double ly2 = log((double)y_t * (double)y_t + 1e-8);
            st.m = ts.m_pred + ts.K * (ly2 - (ts.m_pred - (double)ts.off));
            st.P = (1.0 - ts.K) * ts.P_pred;
            ts.gm = (float)st.m;
        }
    }
    __syncthreads();
    // ---- predict and prior means (svpf_opt_kernels.cu:125-206, 384-392), guide
    {
        const float lev_num = ts.gamma * y_prev;
        const float rc = fminf(fmaxf(ts.rho, 0.0f), 0.999f);
        for (int i = tid; i < n; i += kThreads) {
            const float xi = x[i];
            const float z = nz.normal(i, 0);
            const float lev = lev_num / (expf(fminf(xi * 0.5f, 20.0f)) + 1e-8f);
            muk[i] = ts.mu + ts.rho * (xi - ts.mu) + lev_num / (expf(xi * 0.5f) + 1e-8f);
            float hpr;
            if (c.use_mim) {
                const float sel = nz.uniform(i, 0);
                const float scale = sel < c.mim_jump_prob ? c.mim_jump_scale : 1.0f;
                hpr = ts.mu + rc * (xi - ts.mu) + lev + ts.sz * (scale * z);
            } else {
                hpr = ts.mu + ts.rho * (xi - ts.mu) + ts.sz * z + lev;
            }
            const float hp = clamp_h(hpr);
            float hgr = hp;
            if (c.use_guide) {
                if (c.use_guide_preserving) {
                    const float nm = (1.0f - ts.gs) * ts.cm + ts.gs * ts.gm;
                    hgr = nm + (hp - ts.cm);
                } else {
                    hgr = hp + ts.gs * (ts.gm - hp);
                }
            }
            if (rec) {
                rec[XS * np + i] = xi;
                rec[HPR * np + i] = hpr;
                rec[HGR * np + i] = hgr;
                rec[MUK * np + i] = muk[i];
            }
            xn[i] = c.use_guide ? clamp_h(hgr) : hp;
            if (objective == 1) {
                // predictive: Student-t log density of y_t at the predicted particle
                const float A = y_t * y_t / (expf(fminf(hp, 20.0f)) + 1e-8f) / ts.nu;
                lw[i] = ts.stc - 0.5f * hp - (ts.nu + 1.0f) * 0.5f * log1pf(A);
            }
        }
    }
    __syncthreads();
    for (int i = tid; i < n; i += kThreads) x[i] = xn[i];
    float ll_pred = 0.0f;
    if (objective == 1) {
        float mp = -1e10f;
        for (int i = tid; i < n; i += kThreads) mp = fmaxf(mp, lw[i]);
        mp = reduce_max(mp, sh.red);
        float sp[1] = {0.0f};
        for (int i = tid; i < n; i += kThreads) sp[0] += expf(lw[i] - mp);
        reduce_sum<1>(sp, sh.red);
        ll_pred = mp + logf(fmaxf(sp[0] / (float)n, 1e-10f));
        if (tid == 0) {
            ts.mxp = mp;
            ts.sep = sp[0];
        }
    }
    // ---- bandwidth (svpf_opt_kernels.cu:1159-1235)
    {
        float s[2] = {0.0f, 0.0f};
        float mn = 1e10f, mx = -1e10f;
        int imn = 0, imx = 0;
        for (int i = tid; i < n; i += kThreads) {
            const float xi = xn[i];
            s[0] += xi;
            s[1] += xi * xi;
            if (xi < mn) { mn = xi; imn = i; }
            if (xi > mx) { mx = xi; imx = i; }
        }
        reduce_sum<2>(s, sh.red);
        reduce_argminmax(mn, imn, mx, imx, sh.red, sh.ired);
        if (tid == 0) {
            const float inv_n = 1.0f / (float)n;
            ts.mean = s[0] * inv_n;
            ts.var = s[1] * inv_n - ts.mean * ts.mean;
            ts.mn = mn; ts.mx = mx; ts.imn = imn; ts.imx = imx;
            ts.bw2_new_raw = 2.0f * ts.var / logf((float)n + 1.0f);
            const float bw2_new = fmaxf(ts.bw2_new_raw, 1e-6f);
            ts.bw2_prev = st.bw_sq;
            ts.pre = st.bw_sq > 0.0f ? 0.3f * bw2_new + 0.7f * st.bw_sq : bw2_new;
            const float a = fabsf(y_t);
            float ema = st.return_ema, rv = st.return_var;
            ema = ema > 0.0f ? 0.05f * a + 0.95f * ema : a;
            rv = rv > 0.0f ? 0.05f * a * a + 0.95f * rv : a * a;
            st.return_ema = ema;
            st.return_var = rv;
            ts.ratio = a / fmaxf(ema, 1e-8f);
            ts.spread_f = fminf((mx - mn) * 0.5f, 2.0f);
            ts.comb = fmaxf(ts.ratio, ts.spread_f);
            ts.scale_raw = 1.0f - 0.25f * fminf(ts.comb - 1.0f, 2.0f);
            ts.bw2 = ts.pre * clampf(ts.scale_raw, 0.5f, 1.0f);
            ts.bw = clampf(sqrtf(ts.bw2), 0.01f, 2.0f);
            ts.ib = 1.0f / ts.bw;
            st.bw_sq = ts.bw2;
            // Stein budget and beta schedule (svpf_optimized_graph.cu:1057-1138)
            const int na = c.use_annealing ? max(min(c.n_anneal_steps, SVPF_MAX_ANNEAL_STEPS), 1) : 1;
            int budget;
            if (st.timestep < 10) {
                budget = c.stein_max_steps;
            } else {
                float kn01 = (st.ksd_prev - 0.05f) / (0.50f - 0.05f);
                kn01 = fminf(fmaxf(kn01, 0.0f), 1.0f);
                budget = c.stein_min_steps + (int)(kn01 * (float)(c.stein_max_steps - c.stein_min_steps));
            }
            budget = max(min(budget, bmax), 0);
            ts.budget = budget;
            ts.na = na;
            const float eps_step = SVPF_STEIN_STEP_SIZE * (c.use_guide ? 0.5f : 1.0f);
            for (int it = 0; it < budget; ++it) {
                const int ai = stage_of_it(it, budget, na);
                float beta;
                if (!c.use_annealing) beta = 1.0f;
                else if (c.use_adaptive_beta) beta = adaptive_beta(st.ksd_prev, ai, na);
                else beta = (ai % 3 == 0) ? 0.30f : (ai % 3 == 1) ? 0.65f : 1.0f;
                ts.beta[it] = beta;
                ts.es[it] = eps_step * sqrtf(beta);
            }
        }
        __syncthreads();
    }
    // ---- sorted, scaled prior means for the mixture passes
    const float inv2 = 0.5f / ts.s2, inv = 1.0f / ts.s2;
    const float psc = sqrtf(kLog2e * inv2);
    const int nk4 = round_up(n, 4);
    {
        const int ml = mix_len(n, np);
        for (int i = tid; i < ml; i += kThreads) srt[i] = i < n ? muk[i] * psc : kMuPad;
        // far columns of the transport pair loops
        for (int i = n + tid; i < nk4; i += kThreads) x[i] = kHPadRaw;
        __syncthreads();
        bitonic_sort(srt, pow2_at_least(n));
    }
    // ---- Stein loop
    const float sign = c.stein_repulsive_sign == 1 ? 1.0f : -1.0f;
    const float temp = c.use_svld ? c.temperature : 0.0f;
    const float y2 = y_t * y_t;
    const float ib = ts.ib, ib2 = ib * ib;
    const float inv_n = 1.0f / (float)n;
    const int budget = ts.budget;
    int kn = 1;
    float ksd_acc = 0.0f;
    for (int it = 0; it < budget; ++it) {
        const float beta = ts.beta[it];
        const bool last = it == budget - 1;
        float* R = rec ? rec + (size_t)np * (kRecFixed + kRecPerIt * it) : nullptr;
        // gradient pass (svpf_opt_kernels.cu:354-521), two rows per thread
        for (int i = n + tid; i < nk4; i += kThreads) {
            g[i] = 0.0f;
            curv[i] = 0.0f;
        }
        for (int base = 0; base < n; base += 2 * kThreads) {
            const int j0 = base + tid;
            if (j0 >= n) break;
            const bool two = j0 + kThreads < n;
            const int j1 = two ? j0 + kThreads : j0;
            const float2 xs2 = make_float2(x[j0] * psc, x[j1] * psc);
            const float2 dm = make_float2(nearest_d2(srt, n, xs2.x), nearest_d2(srt, n, xs2.y));
            float2 sr2 = f2(0.0f), wg2 = f2(0.0f), m22 = f2(0.0f), m32 = f2(0.0f);
            if (R) mixture_rows<true>(srt, nk4, xs2, make_float2(-dm.x, -dm.y), sr2, wg2, m22, m32);
            else mixture_rows<false>(srt, nk4, xs2, make_float2(-dm.x, -dm.y), sr2, wg2, m22, m32);
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                if (r == 1 && !two) break;
                const int j = r ? j1 : j0;
                const float xj = x[j];
                const float sr = r ? sr2.y : sr2.x;
                // sum_k w d = wg' / psc;  gp = -(sum w d) / s2 / (sum w + 1e-8)
                const float gp = -((r ? wg2.y : wg2.x) / psc) * inv / (sr + 1e-8f);
                const float A = y2 / (expf(fminf(xj, 20.0f)) + 1e-8f) / ts.nu;
                const float opA = 1.0f + A;
                lw[j] = ts.stc - 0.5f * xj - (ts.nu + 1.0f) * 0.5f * log1pf(fmaxf(A, -0.999f));
                float glik;
                if (c.use_exact_gradient) glik = -0.5f + 0.5f * (ts.nu + 1.0f) * A / opA - c.lik_offset;
                else glik = (logf(y2 + 1e-10f) - xj + c.lik_offset) / 1.4f;
                const float gpre = gp + beta * glik;
                g[j] = clampf(gpre, -10.0f, 10.0f);
                if (full) {
                    const float hl = -0.5f * (ts.nu + 1.0f) * A / (opA * opA);
                    curv[j] = clampf(-(hl - inv), 0.1f, 100.0f);
                }
                if (R) {
                    const float dbar = -gp * ts.s2;              // E_w[d]
                    const float i2 = 1.0f / (psc * psc);
                    const float e2 = (r ? m22.y : m22.x) * i2 / sr, e3 = (r ? m32.y : m32.x) * i2 / psc / sr;
                    R[IX * np + j] = xj;
                    R[IV * np + j] = v[j];
                    R[IGPRE * np + j] = gpre;
                    R[IAL * np + j] = A;
                    R[ILMAX * np + j] = r ? dm.y : dm.x;      // nearest scaled distance^2
                    R[IZ * np + j] = sr;
                    R[IDBAR * np + j] = dbar;
                    R[IVARD * np + j] = e2 - dbar * dbar;
                    R[ISKEW * np + j] = e3 - dbar * e2;
                }
            }
        }
        __syncthreads();
        // transport (vanilla :527-599 or full Newton :912-1103), Jacobi
        const float es = ts.es[it];
        for (int base = 0; base < n; base += 2 * kThreads) {
            const int i0 = base + tid;
            if (i0 >= n) break;
            const bool two = i0 + kThreads < n;
            const int i1 = two ? i0 + kThreads : i0;
            const float2 xi2 = make_float2(x[i0] * ib, x[i1] * ib);
            float2 kg = f2(0.0f), gk = f2(0.0f), ks = f2(0.0f), kc = f2(0.0f), nk = f2(0.0f), gdk = f2(0.0f),
                   ht = f2(0.0f);
            if (full) {
                if (last) transport_rows<true, true>(x, g, curv, nk4, xi2, ib, kg, gk, ks, kc, nk, gdk, ht);
                else transport_rows<true, false>(x, g, curv, nk4, xi2, ib, kg, gk, ks, kc, nk, gdk, ht);
            } else {
                if (last) transport_rows<false, true>(x, g, curv, nk4, xi2, ib, kg, gk, ks, kc, nk, gdk, ht);
                else transport_rows<false, false>(x, g, curv, nk4, xi2, ib, kg, gk, ks, kc, nk, gdk, ht);
            }
            {   // the row's own column: u = 0 exactly (self_uk2)
                float2 Ks;
                const float2 s1 = self_uk2(make_float2(x[i0], x[i1]), xi2, ib, Ks);
                gk = fma2(s1, f2(-1.0f), gk);
                if (last) gdk = fma2(make_float2(-g[i0], -g[i1]), s1, gdk);
            }
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                if (r == 1 && !two) break;
                const int i = r ? i1 : i0;
                const float xi = x[i], gi = g[i];
                const float kgr = r ? kg.y : kg.x, gkr = r ? gk.y : gk.x;
                const float phir = (kgr + sign * 2.0f * ib * gkr) * inv_n;
                float phi = phir, hr = 0.0f, hw = 0.0f, kk = 0.0f;
                if (full) {
                    hw = (r ? kc.y : kc.x) + 2.0f * ib2 * (r ? nk.y : nk.x);
                    kk = r ? ks.y : ks.x;
                    hr = hw / fmaxf(kk, 1e-6f);
                    phi = phir / clampf(hr, 0.1f, 100.0f) * 0.7f;
                }
                if (last)
                    ksd_acc += gi * kgr + 2.0f * ib * (gi * gkr - (r ? gdk.y : gdk.x)) + 2.0f * ib2 * (r ? ht.y : ht.x);
                const float rr = c.rmsprop_rho;
                const float vn = rr * v[i] + (1.0f - rr) * phi * phi;
                float diff = 0.0f;
                if (temp > 1e-6f) diff = sqrtf(2.0f * es * temp) * nz.normal(i, kn);
                const float xr = xi + es * phi * rsqrtf(vn + c.rmsprop_eps) + diff;
                xn[i] = clamp_h(xr);
                v[i] = vn;
                if (R) {
                    R[IPHIR * np + i] = phir;
                    R[IHR * np + i] = hr;
                    R[IHW * np + i] = hw;
                    R[IKN * np + i] = kk;
                    R[IXR * np + i] = xr;
                    R[INK * np + i] = full ? (r ? nk.y : nk.x) : 0.0f;
                }
            }
        }
        __syncthreads();
        for (int i = tid; i < n; i += kThreads) x[i] = xn[i];
        __syncthreads();
        if (temp > 1e-6f) ++kn;
    }
    // ---- outputs (svpf_opt_kernels.cu:1109-1153)
    float mxl = -1e10f;
    for (int i = tid; i < n; i += kThreads) mxl = fmaxf(mxl, lw[i]);
    mxl = reduce_max(mxl, sh.red);
    float s[3] = {0.0f, 0.0f, ksd_acc};
    for (int i = tid; i < n; i += kThreads) {
        s[0] += expf(lw[i] - mxl);
        s[1] += x[i];
    }
    reduce_sum<3>(s, sh.red);
    if (rec) {
        float* RB = rec + (size_t)np * (kRecFixed + kRecPerIt * bmax);
        for (int i = tid; i < n; i += kThreads) {
            RB[i] = x[i];
            RB[np + i] = v[i];
        }
    }
    const float ll = mxl + logf(fmaxf(s[0] * inv_n, 1e-10f));
    if (tid == 0) {
        ts.mxl = mxl;
        ts.se = s[0];
        st.h_mean_prev = s[1] * inv_n;
        if (budget > 0) {
            const float k2 = s[2] / ((float)n * (float)n);
            st.ksd_prev = sqrtf(fmaxf(k2, 0.0f));
        }
        st.timestep += 1;
    }
    __syncthreads();
    return objective == 1 ? ll_pred : ll;
}

// Backward of one recorded tick.  xb, vb: adjoints of the tick's output
// positions / moments on entry, of its input positions / moments on exit.
// sa: adjoints of the scalar state (in: outputs of this tick; out: inputs).
__device__ void bwd_tick(const svpf_config_t& c, int n, int np, float* xb, float* vb, float* work,
                         Shared& sh, GAdj& sa, const Noise& nz, const float* rec, int bmax, float wt,
                         int objective) {
    const int tid = threadIdx.x;
    const TickScalars& ts = sh.ts;
    float* xs = work;                 // x^(it)
    float* g = work + np;             // clamped score
    float* a = work + 2 * np;         // dL/dphi_raw / n
    float* cv = work + 3 * np;        // curvature
    float* hwb = work + 4 * np;       // dL/dhw
    float* knb = work + 5 * np;       // dL/dkn
    float* coef = work + 6 * np;      // mixture column coefficients
    float* lmx = work + 7 * np;
    float* dbr = work + 8 * np;
    float* mub = work + 9 * np;       // dL/dmu_k accumulated over iterations
    float* lwb = work + 10 * np;      // dL/dlw of the last gradient pass
    const bool full = c.use_newton && c.use_full_newton;
    const float sign = c.stein_repulsive_sign == 1 ? 1.0f : -1.0f;
    const float s2 = ts.s2, inv = 1.0f / s2;
    const float psc = sqrtf(kLog2e * (0.5f / s2));   // mixture scale of the forward
    const int nk4 = round_up(n, 4);
    const float nu = ts.nu;
    const float ib = ts.ib, ib2 = ib * ib;
    const float inv_n = 1.0f / (float)n;
    const float rr = c.rmsprop_rho;
    const int budget = ts.budget;
    // thread-local partial sums of theta adjoints: mu, rho, sigma_z, nu, s2, bw
    float pmu = 0.0f, prho = 0.0f, psz = 0.0f, pnu = 0.0f, ps2 = 0.0f, pbw = 0.0f;

    // output mean -> next tick's guide reference
    const float hmb = (float)sa.h_mean * inv_n;
    for (int i = tid; i < n; i += kThreads) {
        xb[i] += hmb;
        mub[i] = 0.0f;
        lwb[i] = 0.0f;
    }
    // loglik = mxl + log(se/n): dL/dlw_i = w_t exp(lw_i - mxl) / se
    if (objective == 0 && budget > 0 && ts.se * inv_n > 1e-10f) {
        const float* R = rec + (size_t)np * (kRecFixed + kRecPerIt * (budget - 1));
        for (int i = tid; i < n; i += kThreads) {
            const float xi = R[IX * np + i], A = R[IAL * np + i];
            const float lwi = ts.stc - 0.5f * xi - (nu + 1.0f) * 0.5f * log1pf(fmaxf(A, -0.999f));
            lwb[i] = wt * expf(lwi - ts.mxl) / ts.se;
        }
    }
    __syncthreads();

    for (int it = budget - 1; it >= 0; --it) {
        const float* R = rec + (size_t)np * (kRecFixed + kRecPerIt * it);
        const float beta = ts.beta[it], es = ts.es[it];
        // (a) elementwise: clamp, drift, RMSProp
        for (int i = tid; i < n; i += kThreads) {
            const float xr = R[IXR * np + i];
            const float xi = R[IX * np + i];
            const float vin = R[IV * np + i];
            const float phir = R[IPHIR * np + i];
            xs[i] = xi;
            const float gp = R[IGPRE * np + i];
            g[i] = clampf(gp, -10.0f, 10.0f);
            float Hc = 1.0f, phi = phir;
            if (full) {
                Hc = clampf(R[IHR * np + i], 0.1f, 100.0f);
                phi = phir / Hc * 0.7f;
                const float A = R[IAL * np + i];
                const float opA = 1.0f + A;
                const float hl = -0.5f * (nu + 1.0f) * A / (opA * opA);
                cv[i] = clampf(-(hl - inv), 0.1f, 100.0f);
            }
            const float vn = rr * vin + (1.0f - rr) * phi * phi;
            const float r = rsqrtf(vn + c.rmsprop_eps);
            const float cc = (xr >= SVPF_H_MIN && xr <= SVPF_H_MAX) ? xb[i] : 0.0f;
            const float vbt = vb[i] + cc * es * phi * (-0.5f) * r * r * r;
            const float phib = cc * es * r + vbt * 2.0f * (1.0f - rr) * phi;
            vb[i] = vbt * rr;
            xb[i] = cc;
            float pr = phib;
            if (full) {
                pr = phib * 0.7f / Hc;
                const float hr = R[IHR * np + i];
                const float Hb = (hr >= 0.1f && hr <= 100.0f) ? -phib * 0.7f * phir / (Hc * Hc) : 0.0f;
                const float kk = R[IKN * np + i], hw = R[IHW * np + i];
                const float kkc = fmaxf(kk, 1e-6f);
                hwb[i] = Hb / kkc;
                knb[i] = kk > 1e-6f ? -Hb * hw / (kkc * kkc) : 0.0f;
            }
            a[i] = pr * inv_n;
        }
        __syncthreads();
        // far columns of the pair loops: position pad, zero weights
        for (int i = n + tid; i < nk4; i += kThreads) {
            xs[i] = kHPadRaw;
            g[i] = 0.0f;
            a[i] = 0.0f;
            cv[i] = 0.0f;
            hwb[i] = 0.0f;
            knb[i] = 0.0f;
            coef[i] = 0.0f;
            lmx[i] = 0.0f;
            dbr[i] = 0.0f;
        }
        __syncthreads();
        // (b) transport adjoint: one pass of row sums (row and column terms),
        // two rows per thread; (c) the O(N) gradient adjoint of each row
        for (int base = 0; base < n; base += 2 * kThreads) {
            const int i0 = base + tid;
            if (i0 >= n) break;
            const bool two = i0 + kThreads < n;
            const int i1 = two ? i0 + kThreads : i0;
            float2 acc[kAdjAcc];
#pragma unroll
            for (int q = 0; q < kAdjAcc; ++q) acc[q] = f2(0.0f);
            const float2 xi2 = make_float2(xs[i0] * ib, xs[i1] * ib);
            if (full) adjoint_rows<true>(xs, g, a, cv, hwb, knb, nk4, xi2, ib, acc);
            else adjoint_rows<false>(xs, g, a, cv, hwb, knb, nk4, xi2, ib, acc);
            {   // the row's own column: u = 0 exactly (self_uk2); its terms odd in u leave the sums
                float2 Ks;
                const float2 s1 = self_uk2(make_float2(xs[i0], xs[i1]), xi2, ib, Ks);
                const float2 ns1 = make_float2(-s1.x, -s1.y);
                acc[0] = fma2(make_float2(g[i0], g[i1]), ns1, acc[0]);
                acc[2] = fma2(make_float2(a[i0], a[i1]), ns1, acc[2]);
                acc[5] = add2(acc[5], ns1);
                if (full) {
                    const float2 t = fma2(Ks, f2(-4.0f), f2(3.0f));
                    const float2 f6u = mul2(s1, fma2(Ks, f2(16.0f), f2(-6.0f)));
                    const float2 nf6 = make_float2(-flip_sign(f6u.x, t.x), -flip_sign(f6u.y, t.y));
                    const float2 hb2 = make_float2(hwb[i0], hwb[i1]);
                    acc[6] = fma2(make_float2(cv[i0], cv[i1]), ns1, acc[6]);
                    acc[7] = add2(acc[7], nf6);
                    acc[8] = fma2(hb2, ns1, acc[8]);
                    acc[9] = fma2(hb2, nf6, acc[9]);
                    acc[10] = fma2(make_float2(knb[i0], knb[i1]), ns1, acc[10]);
                }
            }
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                if (r == 1 && !two) break;
                const int i = r ? i1 : i0;
                float v_[kAdjAcc];
#pragma unroll
                for (int q = 0; q < kAdjAcc; ++q) v_[q] = r ? acc[q].y : acc[q].x;
                const float S1 = v_[0], S2 = -v_[1], C1 = v_[2], C2 = -v_[3], C3 = v_[4], R3 = v_[5];
                const float xi = xs[i], gi = g[i], ai = a[i];
                float dx = ib * (ai * (-2.0f * S1 + 2.0f * sign * ib * S2) - 2.0f * gi * C1 - 2.0f * sign * ib * C2);
                // parts of the iteration's objective of degree -1 (repulsion, 2 s uK^2 / bw) and
                // -2 (the Hessian's 2 K^2 |3u^2 - 1| / bw^2) under (x, bw) -> (l x, l bw)
                float gm1 = 2.0f * sign * ib * ai * R3, gm2 = 0.0f;
                float gb = C3;
                if (full) {
                    const float R1 = v_[6], R2 = v_[7], D1 = v_[8], D2 = v_[9], D3 = v_[10], E1 = v_[11];
                    const float hb = hwb[i], kb = knb[i];
                    dx += ib * (hb * (-2.0f * R1 + 2.0f * ib2 * R2) - 2.0f * kb * R3);
                    dx += ib * (-2.0f * cv[i] * D1 + 2.0f * ib2 * D2 - 2.0f * D3);
                    gm2 = 2.0f * ib2 * hb * R[INK * np + i];
                    // bandwidth adjoint by homogeneity, before the curvature path joins dx (below)
                    pbw -= ib * ((xi - ts.mean) * dx + gm1 + 2.0f * gm2);
                    // curvature adjoint E1 -> A and s2 (clamp [0.1, 100])
                    const float A = R[IAL * np + i];
                    const float opA = 1.0f + A;
                    const float craw = 0.5f * (nu + 1.0f) * A / (opA * opA) + inv;
                    if (craw >= 0.1f && craw <= 100.0f) {
                        // curv = 0.5 (nu+1) A / (1+A)^2 + 1/s2
                        const float dcdA = 0.5f * (nu + 1.0f) * (1.0f - A) / (opA * opA * opA);
                        const float dAdx = (xi < 20.0f) ? -A * expf(xi) / (expf(xi) + 1e-8f) : 0.0f;
                        dx += E1 * dcdA * dAdx;
                        pnu += E1 * (0.5f * A / (opA * opA) + dcdA * (-A / nu));
                        ps2 += E1 * (-inv * inv);
                    }
                } else {
                    pbw -= ib * ((xi - ts.mean) * dx + gm1);
                }
                xb[i] += dx;   // rows read a, g, xs of other rows, never xb
                // (c) gradient adjoint, O(N) part (g = clamp(gp + beta glik))
                const float gpre = R[IGPRE * np + i];
                const float gpb = (gpre >= -10.0f && gpre <= 10.0f) ? gb : 0.0f;
                const float A = R[IAL * np + i];
                const float opA = 1.0f + A;
                const float ex = expf(fminf(xi, 20.0f));
                const float dAdx = (xi < 20.0f) ? -A * ex / (ex + 1e-8f) : 0.0f;
                const float dAdnu = -A / nu;
                const float dbar = R[IDBAR * np + i], vard = R[IVARD * np + i], skew = R[ISKEW * np + i];
                float dgdx = -inv + vard * inv * inv;
                float dgdnu = 0.0f;
                if (c.use_exact_gradient) {
                    const float dglA = 0.5f * (nu + 1.0f) / (opA * opA);
                    dgdx += beta * dglA * dAdx;
                    dgdnu = beta * (0.5f * A / opA + dglA * dAdnu);
                } else {
                    dgdx += beta * (-1.0f / 1.4f);
                }
                float dxx = gpb * dgdx;
                pnu += gpb * dgdnu;
                ps2 += gpb * (dbar * inv * inv - skew * 0.5f * inv * inv * inv);
                if (it == budget - 1) {
                    const float lb = lwb[i];
                    const float dlwdA = -(nu + 1.0f) * 0.5f / opA;
                    dxx += lb * (-0.5f + dlwdA * dAdx);
                    pnu += lb * (-0.5f * log1pf(A) + dlwdA * dAdnu);
                }
                xb[i] += dxx;
                coef[i] = gpb * inv / R[IZ * np + i];
                lmx[i] = R[ILMAX * np + i];
                dbr[i] = dbar * psc;
            }
        }
        __syncthreads();
        // (d) mixture column pass: dL/dmu_k, two prior means per thread
        {
            const float* MU = rec + (size_t)np * MUK;
            for (int base = 0; base < n; base += 2 * kThreads) {
                const int k0 = base + tid;
                if (k0 >= n) break;
                const bool two = k0 + kThreads < n;
                const int k1 = two ? k0 + kThreads : k0;
                const float2 acc = mixture_cols(xs, lmx, dbr, coef, nk4, psc, make_float2(MU[k0] * psc, MU[k1] * psc));
                mub[k0] += acc.x;
                if (two) mub[k1] += acc.y;
            }
        }
        __syncthreads();
    }

    // ---- stc(nu) enters every log-weight: dL/dnu += stc'(nu) * sum lwb
    // ---- bandwidth adjoint (needs the total dL/dbw)
    {
        // predictive objective: its weights sum to one, so stc' enters once, times w_t
        const bool pred_on = objective == 1 && ts.sep * inv_n > 1e-10f;
        float s[2] = {pbw, (tid == 0 && pred_on) ? wt : 0.0f};
        for (int i = tid; i < n; i += kThreads) s[1] += lwb[i];
        reduce_sum<2>(s, sh.red);
        if (tid == 0) {
            TickScalars& t = sh.ts;
            const double dstc = 0.5 * digamma_bounded(0.5 * ((double)nu + 1.0)) - 0.5 * digamma_bounded(0.5 * (double)nu) -
                                0.5 / (double)nu;
            sh.acc[3] = dstc * (double)s[1];
            const float bwb = s[0];
            const float sq = sqrtf(t.bw2);
            float bw2b = (sq >= 0.01f && sq <= 2.0f) ? bwb * 0.5f / sq : 0.0f;
            bw2b += (float)sa.bw_sq;
            const float sc = clampf(t.scale_raw, 0.5f, 1.0f);
            const float scb = bw2b * t.pre;
            const float preb = bw2b * sc;
            float spb = 0.0f;
            if (t.scale_raw >= 0.5f && t.scale_raw <= 1.0f && t.comb - 1.0f <= 2.0f) {
                const float combb = -0.25f * scb;
                if (t.spread_f > t.ratio && (t.mx - t.mn) * 0.5f <= 2.0f) spb = 0.5f * combb;
            }
            const float bnb = t.bw2_prev > 0.0f ? 0.3f * preb : preb;
            sa.bw_sq = t.bw2_prev > 0.0f ? 0.7 * (double)preb : 0.0;
            const float varb = t.bw2_new_raw >= 1e-6f ? bnb * 2.0f / logf((float)n + 1.0f) : 0.0f;
            // broadcast through the scratch
            sh.red[0][0] = varb;
            sh.red[0][1] = spb;
        }
        __syncthreads();
        const float varb = sh.red[0][0], spb = sh.red[0][1];
        const float* X0 = rec + (size_t)np * (kRecFixed + 0);   // x^(0) = X of iteration 0
        for (int i = tid; i < n; i += kThreads) {
            float x0;
            if (budget > 0) x0 = X0[IX * np + i];
            else x0 = rec[(size_t)np * (kRecFixed + kRecPerIt * bmax) + i];
            xb[i] += varb * 2.0f * (x0 - ts.mean) * inv_n;
        }
        __syncthreads();
        if (tid == 0) {
            xb[ts.imx] += spb;
            xb[ts.imn] -= spb;
        }
        __syncthreads();
    }
    // ---- guide adjoint, predict adjoint, prior-mean adjoint
    {
        const float rc = fminf(fmaxf(ts.rho, 0.0f), 0.999f);
        const bool rin = ts.rho >= 0.0f && ts.rho <= 0.999f;
        const float lev_num = ts.gamma * ts.y_prev;
        float sc[1] = {0.0f};
        for (int i = tid; i < n; i += kThreads) {
            float hpb;
            if (c.use_guide) {
                const float hgr = rec[HGR * np + i];
                const float cg = (hgr >= SVPF_H_MIN && hgr <= SVPF_H_MAX) ? xb[i] : 0.0f;
                sc[0] += cg;
                hpb = c.use_guide_preserving ? cg : (1.0f - ts.gs) * cg;
            } else {
                hpb = xb[i];
            }
            const float hpr = rec[HPR * np + i];
            if (objective == 1 && ts.sep * inv_n > 1e-10f) {
                // d/dhp and d/dnu of w_t log mean_i p(y_t | hp_i)
                const float hp = clamp_h(hpr);
                const float e = expf(fminf(hp, 20.0f));
                const float A = ts.y_t * ts.y_t / (e + 1e-8f) / nu;
                const float lp = ts.stc - 0.5f * hp - (nu + 1.0f) * 0.5f * log1pf(A);
                const float pw = wt * expf(lp - ts.mxp) / ts.sep;
                const float dlpdA = -(nu + 1.0f) * 0.5f / (1.0f + A);
                const float dAdh = hp < 20.0f ? -A * e / (e + 1e-8f) : 0.0f;
                hpb += pw * (-0.5f + dlpdA * dAdh);
                pnu += pw * (-0.5f * log1pf(A) + dlpdA * (-A / nu));
            }
            const float cp = (hpr >= SVPF_H_MIN && hpr <= SVPF_H_MAX) ? hpb : 0.0f;
            const float xi = rec[XS * np + i];
            const float z = nz.normal(i, 0);
            const float e1 = expf(fminf(xi * 0.5f, 20.0f));
            const float levd = (xi * 0.5f < 20.0f) ? -lev_num * 0.5f * e1 / ((e1 + 1e-8f) * (e1 + 1e-8f)) : 0.0f;
            const float e2 = expf(xi * 0.5f);
            const float mkd = -lev_num * 0.5f * e2 / ((e2 + 1e-8f) * (e2 + 1e-8f));
            const float mb = mub[i];
            float dxin;
            if (c.use_mim) {
                const float sel = nz.uniform(i, 0);
                const float scale = sel < c.mim_jump_prob ? c.mim_jump_scale : 1.0f;
                dxin = cp * (rc + levd);
                pmu += cp * (1.0f - rc);
                if (rin) prho += cp * (xi - ts.mu);
                psz += cp * scale * z;
            } else {
                dxin = cp * (ts.rho + levd);
                pmu += cp * (1.0f - ts.rho);
                prho += cp * (xi - ts.mu);
                psz += cp * z;
            }
            dxin += mb * (ts.rho + mkd);
            pmu += mb * (1.0f - ts.rho);
            prho += mb * (xi - ts.mu);
            xb[i] = dxin;
        }
        reduce_sum<1>(sc, sh.red);
        float s[6] = {pmu, prho, psz, pnu, ps2, 0.0f};
        reduce_sum<6>(s, sh.red);
        if (tid == 0) {
            const double mu = ts.mu, rho = ts.rho, sz = ts.sz;
            double dmu = s[0], drho = s[1], dsz = s[2], dnu = (double)s[3] + sh.acc[3];
            dsz += (double)s[4] * 2.0 * sz;
            double cmb = 0.0;
            if (c.use_guide) {
                const double gmb = (double)ts.gs * (double)sc[0];
                cmb = c.use_guide_preserving ? -(double)ts.gs * (double)sc[0] : 0.0;
                // EKF adjoint (FP64)
                const double mpb0 = sa.m + gmb;
                const double Pb = sa.P;
                const double ly2 = log((double)ts.y_t * (double)ts.y_t + 1e-8);
                const double Kb = mpb0 * (ly2 + (double)ts.off - ts.m_pred) - Pb * ts.P_pred;
                const double mpb = mpb0 * (1.0 - ts.K);
                const double den = ts.P_pred + 6.93 + 1e-8;
                const double Ppb = Pb * (1.0 - ts.K) + Kb * (6.93 + 1e-8) / (den * den);
                dmu += mpb * (1.0 - rho);
                drho += mpb * (ts.m_in - mu) + Ppb * 2.0 * rho * ts.P_in;
                dsz += Ppb * 2.0 * sz;
                double mb = mpb * rho, Pbi = Ppb * rho * rho;
                if (ts.init_here) {
                    dmu += mb;
                    const double q = 1.0 - rho * rho;
                    dsz += Pbi * 2.0 * sz / q;
                    drho += Pbi * sz * sz * 2.0 * rho / (q * q);
                    mb = 0.0;
                    Pbi = 0.0;
                }
                sa.m = mb;
                sa.P = Pbi;
            }
            sa.h_mean = cmb;
            sa.th[0] += dmu;
            sa.th[1] += drho;
            sa.th[2] += dsz;
            sa.th[3] += dnu;
        }
        __syncthreads();
    }
}

__device__ inline Noise make_noise(unsigned long long seed, int f, int tick, int n, int* flag) {
    return Noise{philox_key(seed, f), (uint32_t)tick, nullptr, nullptr, 0, 0, n, flag};
}

__device__ inline void load_theta(const GArgs& a, int f, TickScalars& ts) {
    ts.mu = a.theta[4 * f + 0];
    ts.rho = a.theta[4 * f + 1];
    ts.sz = a.theta[4 * f + 2];
    ts.nu = a.theta[4 * f + 3];
    ts.gamma = a.gamma ? a.gamma[f] : 0.0f;
}

// 1 when filter f's parameters cannot be run (see theta_ok; leverage finite).
__device__ inline int theta_bad(const TickScalars& ts) {
    return !theta_ok(ts.mu, ts.rho, ts.sz, ts.nu) || !(fabsf(ts.gamma) < INFINITY);
}

// svpf_initialize (svpf_optimized_graph.cu:349-451), single factor, Philox draw 0 of stream 2.
__device__ void init_filter(const GArgs& a, int f, int n, float* x, float* v, Shared& sh) {
    const TickScalars& ts = sh.ts;
    const float var = ts.sz * ts.sz / (1.0f - ts.rho * ts.rho + 1e-6f);
    const float sd = sqrtf(var);
    const uint2 key = philox_key(a.seed, f);
    for (int i = threadIdx.x; i < n; i += kThreads) {
        const uint4 r = philox10(key, make_uint4((uint32_t)i, 0u, 0u, 2u));
        const float z = normal_from_bits(r.x, r.y);
        x[i] = clamp_h(ts.mu + sd * z);
        v[i] = 0.0f;
    }
    if (threadIdx.x == 0) {
        GState& s = sh.st;
        s.m = ts.mu;
        s.P = var;
        s.bw_sq = 0.0f;
        s.h_mean_prev = -3.5f;   // :492-494
        s.return_ema = 0.0f;
        s.return_var = 0.0f;
        s.ksd_prev = 1e10f;
        s.guide_init = 0;
        s.timestep = 0;
        s.pad = 0;
    }
    __syncthreads();
}

// adjoint of the initialisation: h_i = clamp(mu + sd z_i), sd^2 = sz^2/(1 - rho^2 + 1e-6)
__device__ void init_adjoint(const GArgs& a, int f, int n, const float* xb, Shared& sh, GAdj& sa) {
    const TickScalars& ts = sh.ts;
    const float q = 1.0f - ts.rho * ts.rho + 1e-6f;
    const float var = ts.sz * ts.sz / q;
    const float sd = sqrtf(var);
    const uint2 key = philox_key(a.seed, f);
    float s[2] = {0.0f, 0.0f};
    for (int i = threadIdx.x; i < n; i += kThreads) {
        const uint4 r = philox10(key, make_uint4((uint32_t)i, 0u, 0u, 2u));
        const float z = normal_from_bits(r.x, r.y);
        const float hr = ts.mu + sd * z;
        if (hr >= SVPF_H_MIN && hr <= SVPF_H_MAX) {
            s[0] += xb[i];
            s[1] += xb[i] * z;
        }
    }
    reduce_sum<2>(s, sh.red);
    if (threadIdx.x == 0) {
        const double varb = (double)s[1] / (2.0 * sd);
        sa.th[0] += s[0];
        sa.th[2] += varb * 2.0 * ts.sz / q;
        sa.th[1] += varb * (double)ts.sz * ts.sz * 2.0 * ts.rho / ((double)q * q);
    }
    __syncthreads();
}

__device__ inline void copy_state_to(GState* dst, const GState& src) {
    if (threadIdx.x == 0) *dst = src;
}

// Truncated backpropagation through time: after the adjoint of tick t, for
// t > 0 with t % trunc == 0, the state carried into tick t (particles,
// RMSProp moments, EKF mean and variance, bandwidth average, previous mean)
// is held constant in theta -- its adjoint is dropped; theta's is kept.
__device__ inline void truncate_after(const GArgs& a, int t, int n, float* xb, float* vb, GAdj& sa) {
    if (a.trunc <= 0 || t == 0 || t % a.trunc != 0) return;
    for (int i = threadIdx.x; i < n; i += kThreads) {
        xb[i] = 0.0f;
        vb[i] = 0.0f;
    }
    if (threadIdx.x == 0) {
        sa.m = 0.0;
        sa.P = 0.0;
        sa.bw_sq = 0.0;
        sa.h_mean = 0.0;
    }
    __syncthreads();
}

// Forward over ticks [t0, t1) for every filter; checkpoint at segment starts.
__global__ void __launch_bounds__(kThreads) grad_forward_kernel(const GArgs a, int t0, int t1) {
    extern __shared__ __align__(16) float smem[];
    __shared__ Shared sh;
    __shared__ svpf_config_t cfg;
    const int np = a.np;
    float* x = smem;
    float* v = smem + np;
    float* work = smem + 2 * np;
    for (int f = blockIdx.x; f < a.F; f += gridDim.x) {
        if (threadIdx.x == 0) {
            cfg = a.cfg[f];
            sh.flag = 0;
            load_theta(a, f, sh.ts);
            sh.bad = theta_bad(sh.ts);
        }
        __syncthreads();
        if (sh.bad) {
            // parameters no filter can run with: report them and leave the filter out
            if (a.loglik)
                for (int t = t0 + threadIdx.x; t < t1; t += kThreads) a.loglik[(size_t)f * a.T + t] = NAN;
            if (threadIdx.x == 0) {
                a.status[f] = SVPF_ERR_INVALID_ARG;
                a.ll_sum[f] = NAN;
            }
            __syncthreads();
            continue;
        }
        const int n = a.n[f];
        if (t0 == 0) {
            init_filter(a, f, n, x, v, sh);
            if (threadIdx.x == 0) a.ll_sum[f] = 0.0;
        } else {
            for (int i = threadIdx.x; i < n; i += kThreads) {
                x[i] = a.fx[(size_t)f * np + i];
                v[i] = a.fv[(size_t)f * np + i];
            }
            if (threadIdx.x == 0) sh.st = a.fs[f];
            __syncthreads();
        }
        for (int t = t0; t < t1; ++t) {
            if (t % a.k == 0) {
                const int sg = t / a.k;
                float* ck = a.ck + ((size_t)f * a.nseg + sg) * 2 * np;
                for (int i = threadIdx.x; i < n; i += kThreads) {
                    ck[i] = x[i];
                    ck[np + i] = v[i];
                }
                copy_state_to(&a.cks[(size_t)f * a.nseg + sg], sh.st);
            }
            const float yt = a.y[(size_t)f * a.T + t];
            const float yp = t > 0 ? a.y[(size_t)f * a.T + t - 1] : 0.0f;
            const Noise nz = make_noise(a.seed, f, sh.st.timestep, n, &sh.flag);
            float* rt = nullptr;
            if (a.run_rec) {   // keep this tick's record: the backward replays none of the forward
                rt = a.run_rec + ((size_t)f * a.T_max + t) * a.rec_floats;
                copy_state_to(&a.run_st[(size_t)f * a.T_max + t], sh.st);
            }
            __syncthreads();
            const float ll = fwd_tick(cfg, n, np, x, v, work, sh, nz, yt, yp, rt, a.bmax, a.objective);
            if (threadIdx.x == 0) {
                if (a.loglik) a.loglik[(size_t)f * a.T + t] = ll;
                a.ll_sum[f] += (double)ll;
                if (a.run_rec) a.run_ts[(size_t)f * a.T_max + t] = sh.ts;
            }
        }
        for (int i = threadIdx.x; i < n; i += kThreads) {
            a.fx[(size_t)f * np + i] = x[i];
            a.fv[(size_t)f * np + i] = v[i];
        }
        if (threadIdx.x == 0) {
            a.fs[f] = sh.st;
            if (sh.flag) a.status[f] = sh.flag;
        }
        __syncthreads();
    }
}

// Backward over segment sg for every filter.
__global__ void __launch_bounds__(kThreads) grad_backward_kernel(const GArgs a, int sg) {
    extern __shared__ __align__(16) float smem[];
    __shared__ Shared sh;
    __shared__ svpf_config_t cfg;
    __shared__ GAdj sa;
    const int np = a.np;
    float* x = smem;
    float* v = smem + np;
    float* xb = smem + 2 * np;
    float* vb = smem + 3 * np;
    float* work = smem + 4 * np;
    float* seg = a.seg + (size_t)blockIdx.x * a.k * 2 * np;
    GState* segs = a.segs + (size_t)blockIdx.x * a.k;
    TickScalars* segts = a.segts + (size_t)blockIdx.x * a.k;
    float* rec = a.rec + (size_t)blockIdx.x * a.rec_floats * (a.seg_rec ? a.k : 1);
    const int t0 = sg * a.k;
    const int t1 = min(a.T, t0 + a.k);
    for (int f = blockIdx.x; f < a.F; f += gridDim.x) {
        const int n = a.n[f];
        if (threadIdx.x == 0) {
            cfg = a.cfg[f];
            sh.flag = 0;
            load_theta(a, f, sh.ts);
            sh.bad = theta_bad(sh.ts);
            sh.st = a.cks[(size_t)f * a.nseg + sg];
            sa = a.as[f];
        }
        __syncthreads();
        if (sh.bad) {
            if (threadIdx.x == 0) {
                for (int q = 0; q < 4; ++q) a.as[f].th[q] = NAN;
                a.status[f] = SVPF_ERR_INVALID_ARG;
            }
            __syncthreads();
            continue;
        }
        const float* ck = a.ck + ((size_t)f * a.nseg + sg) * 2 * np;
        for (int i = threadIdx.x; i < n; i += kThreads) {
            x[i] = ck[i];
            v[i] = ck[np + i];
            xb[i] = a.ax[(size_t)f * np + i];
            vb[i] = a.av[(size_t)f * np + i];
        }
        __syncthreads();
        if (a.run_rec) {
            // the forward kept every tick's record: adjoints in reverse, nothing recomputed
            for (int t = t1 - 1; t >= t0; --t) {
                const float* rt = a.run_rec + ((size_t)f * a.T_max + t) * a.rec_floats;
                if (threadIdx.x == 0) {
                    sh.st = a.run_st[(size_t)f * a.T_max + t];
                    sh.ts = a.run_ts[(size_t)f * a.T_max + t];
                }
                __syncthreads();
                const Noise nz = make_noise(a.seed, f, sh.st.timestep, n, &sh.flag);
                const float wt = a.w ? a.w[(size_t)f * a.T + t] : 1.0f;
                bwd_tick(cfg, n, np, xb, vb, work, sh, sa, nz, rt, a.bmax, wt, a.objective);
                truncate_after(a, t, n, xb, vb, sa);
            }
        } else if (a.seg_rec) {
            // one forward over the segment recording every tick, then the
            // ticks' adjoints in reverse from those records
            for (int t = t0; t < t1; ++t) {
                float* rt = rec + (size_t)(t - t0) * a.rec_floats;
                copy_state_to(&segs[t - t0], sh.st);
                const float yt = a.y[(size_t)f * a.T + t];
                const float yp = t > 0 ? a.y[(size_t)f * a.T + t - 1] : 0.0f;
                const Noise nz = make_noise(a.seed, f, sh.st.timestep, n, &sh.flag);
                __syncthreads();
                fwd_tick(cfg, n, np, x, v, work, sh, nz, yt, yp, rt, a.bmax, a.objective);
                if (threadIdx.x == 0) segts[t - t0] = sh.ts;
            }
            for (int t = t1 - 1; t >= t0; --t) {
                const float* rt = rec + (size_t)(t - t0) * a.rec_floats;
                if (threadIdx.x == 0) {
                    sh.st = segs[t - t0];
                    sh.ts = segts[t - t0];
                }
                __syncthreads();
                const Noise nz = make_noise(a.seed, f, sh.st.timestep, n, &sh.flag);
                const float wt = a.w ? a.w[(size_t)f * a.T + t] : 1.0f;
                bwd_tick(cfg, n, np, xb, vb, work, sh, sa, nz, rt, a.bmax, wt, a.objective);
                truncate_after(a, t, n, xb, vb, sa);
            }
        } else {
        // recompute the segment, keeping every tick's input state
        for (int t = t0; t < t1; ++t) {
            float* sx = seg + (size_t)(t - t0) * 2 * np;
            for (int i = threadIdx.x; i < n; i += kThreads) {
                sx[i] = x[i];
                sx[np + i] = v[i];
            }
            copy_state_to(&segs[t - t0], sh.st);
            const float yt = a.y[(size_t)f * a.T + t];
            const float yp = t > 0 ? a.y[(size_t)f * a.T + t - 1] : 0.0f;
            const Noise nz = make_noise(a.seed, f, sh.st.timestep, n, &sh.flag);
            __syncthreads();
            if (t + 1 < t1) fwd_tick(cfg, n, np, x, v, work, sh, nz, yt, yp, nullptr, a.bmax, a.objective);
        }
        // reverse over the segment's ticks, re-recording each
        for (int t = t1 - 1; t >= t0; --t) {
            const float* sx = seg + (size_t)(t - t0) * 2 * np;
            for (int i = threadIdx.x; i < n; i += kThreads) {
                x[i] = sx[i];
                v[i] = sx[np + i];
            }
            if (threadIdx.x == 0) {
                sh.st = segs[t - t0];
                load_theta(a, f, sh.ts);
            }
            const float yt = a.y[(size_t)f * a.T + t];
            const float yp = t > 0 ? a.y[(size_t)f * a.T + t - 1] : 0.0f;
            __syncthreads();
            const Noise nz = make_noise(a.seed, f, sh.st.timestep, n, &sh.flag);
            fwd_tick(cfg, n, np, x, v, work, sh, nz, yt, yp, rec, a.bmax, a.objective);
            const float wt = a.w ? a.w[(size_t)f * a.T + t] : 1.0f;
            bwd_tick(cfg, n, np, xb, vb, work, sh, sa, nz, rec, a.bmax, wt, a.objective);
            truncate_after(a, t, n, xb, vb, sa);
        }
        }
        if (t0 == 0) init_adjoint(a, f, n, xb, sh, sa);
        for (int i = threadIdx.x; i < n; i += kThreads) {
            a.ax[(size_t)f * np + i] = xb[i];
            a.av[(size_t)f * np + i] = vb[i];
        }
        if (threadIdx.x == 0) {
            a.as[f] = sa;
            if (sh.flag) a.status[f] = sh.flag;
            // an exact gradient can grow exponentially with the run's length: report overflow
            if (t0 == 0 && !(isfinite(sa.th[0]) && isfinite(sa.th[1]) && isfinite(sa.th[2]) && isfinite(sa.th[3])))
                a.status[f] = SVPF_ERR_NONFINITE;
        }
        __syncthreads();
    }
}

}  // namespace grad
}  // namespace svpf

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using namespace svpf;
using namespace svpf::grad;

struct svpf_grad {
    int F = 0, n_max = 0, np = 0, T_max = 0, k = 64, nseg = 0, bmax = 1, grid = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    size_t smem = 0, rec_floats = 0;
    std::vector<int> ns;
    std::vector<svpf_config_t> cfgs;
    int T = 0;
    unsigned long long seed = 0;
    bool forward_done = false;
    int trunc = 0;                    // truncated backpropagation every trunc ticks (0: off)
    int objective = 0;
    // device
    int* d_n = nullptr;
    svpf_config_t* d_cfg = nullptr;
    float* d_theta = nullptr;
    float* d_gamma = nullptr;
    float* d_y = nullptr;
    float* d_w = nullptr;
    float* d_loglik = nullptr;
    double* d_llsum = nullptr;
    float* d_fx = nullptr;
    float* d_fv = nullptr;
    GState* d_fs = nullptr;
    float* d_ck = nullptr;
    GState* d_cks = nullptr;
    float* d_ax = nullptr;
    float* d_av = nullptr;
    GAdj* d_as = nullptr;
    float* d_seg = nullptr;
    GState* d_segs = nullptr;
    float* d_rec = nullptr;
    TickScalars* d_segts = nullptr;
    bool seg_rec = false;             // records of a whole segment (k ticks per CTA)
    float* d_run_rec = nullptr;       // run records: every tick's record kept by the forward
    GState* d_run_st = nullptr;
    TickScalars* d_run_ts = nullptr;
    int* d_status = nullptr;
    const float* u_theta = nullptr;   // the arrays the last forward used
    const float* u_gamma = nullptr;
    const float* u_y = nullptr;
};

namespace {

template <class T>
bool galloc(T** p, size_t count) {
    return cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T)) == cudaSuccess;
}

size_t run_record_bytes(const svpf_grad* g) {
    return (size_t)g->F * g->T_max * (g->rec_floats * sizeof(float) + sizeof(GState) + sizeof(TickScalars));
}

void free_run_records(svpf_grad* g) {
    cudaFree(g->d_run_rec);
    cudaFree(g->d_run_st);
    cudaFree(g->d_run_ts);
    g->d_run_rec = nullptr;
    g->d_run_st = nullptr;
    g->d_run_ts = nullptr;
}

bool alloc_run_records(svpf_grad* g) {
    const size_t FT = (size_t)g->F * g->T_max;
    if (galloc(&g->d_run_rec, FT * g->rec_floats) && galloc(&g->d_run_st, FT) && galloc(&g->d_run_ts, FT))
        return true;
    free_run_records(g);
    cudaGetLastError();
    return false;
}

GArgs make_gargs(const svpf_grad* g, const float* theta, const float* gamma, const float* y, const float* w,
                 float* loglik) {
    GArgs a;
    std::memset(&a, 0, sizeof(a));
    a.F = g->F;
    a.T = g->T;
    a.k = g->k;
    a.np = g->np;
    a.bmax = g->bmax;
    a.n = g->d_n;
    a.cfg = g->d_cfg;
    a.theta = theta;
    a.gamma = gamma;
    a.y = y;
    a.w = w;
    a.loglik = loglik;
    a.ll_sum = g->d_llsum;
    a.seed = g->seed;
    a.fx = g->d_fx;
    a.fv = g->d_fv;
    a.fs = g->d_fs;
    a.ck = g->d_ck;
    a.cks = g->d_cks;
    a.ax = g->d_ax;
    a.av = g->d_av;
    a.as = g->d_as;
    a.seg = g->d_seg;
    a.segs = g->d_segs;
    a.rec = g->d_rec;
    a.rec_floats = g->rec_floats;
    a.segts = g->d_segts;
    a.seg_rec = g->seg_rec ? 1 : 0;
    a.run_rec = g->d_run_rec;
    a.run_st = g->d_run_st;
    a.run_ts = g->d_run_ts;
    a.T_max = g->T_max;
    a.trunc = g->trunc;
    a.nseg = g->nseg;
    a.status = g->d_status;
    a.objective = g->objective;
    return a;
}

}  // namespace

extern "C" {

int svpf_grad_supported(const svpf_config_t* c) {
    if (!c) return 0;
    if (c->use_two_factor || c->use_heun || c->use_student_t_state || c->use_fan_mode) return 0;
    if (c->use_adaptive_mu || c->use_adaptive_sigma || c->use_adaptive_guide) return 0;
    if (c->use_asymmetric_rho || c->use_local_params || c->use_guided || c->use_rejuvenation) return 0;
    if (c->use_newton && !c->use_full_newton) return 0;
    if (c->stein_min_steps < 1 || c->stein_max_steps < 1) return 0;
    // adaptive beta is a continuous function of the previous tick's KSD, which
    // the adjoint does not differentiate
    if (c->use_annealing && c->use_adaptive_beta) return 0;
    return 1;
}

svpf_grad_t* svpf_grad_create(int F, const int* ns, const svpf_config_t* cfgs, int T_max, int k,
                              cudaStream_t stream) {
    SVPF_TRACE();
    if (F < 1 || !ns || !cfgs || T_max < 1 || k < 1) return nullptr;
    int n_max = 0, bmax = 1;
    for (int f = 0; f < F; ++f) {
        if (ns[f] < 1 || ns[f] > SVPF_MAX_PARTICLES || !svpf_grad_supported(&cfgs[f])) return nullptr;
        n_max = std::max(n_max, ns[f]);
        bmax = std::max(bmax, std::max(cfgs[f].stein_max_steps, cfgs[f].stein_min_steps));
    }
    if (bmax > 64) return nullptr;
    svpf_grad* g = new svpf_grad();
    g->F = F;
    g->n_max = n_max;
    g->np = round_up(n_max, 64);
    g->T_max = T_max;
    g->k = k;
    g->nseg = (T_max + k - 1) / k;
    g->bmax = bmax;
    g->ns.assign(ns, ns + F);
    g->cfgs.assign(cfgs, cfgs + F);
    if (stream) {
        g->stream = stream;
    } else {
        cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
        g->own_stream = true;
    }
    const size_t np = (size_t)g->np;
    g->smem = (size_t)(4 + 11) * np * sizeof(float);
    int dev = 0, optin = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t static_bytes = sizeof(Shared) + sizeof(svpf_config_t) + sizeof(GAdj) + 64;
    if (g->smem + static_bytes > (size_t)optin) {
        delete g;
        return nullptr;
    }
    // the opt-in is the device's whole limit (engines of different sizes share the kernels)
    if (configure_kernel((const void*)grad_forward_kernel, (int)kernel_smem_cap((const void*)grad_forward_kernel),
                         false) != cudaSuccess ||
        configure_kernel((const void*)grad_backward_kernel, (int)kernel_smem_cap((const void*)grad_backward_kernel),
                         false) != cudaSuccess) {
        cudaGetLastError();
        delete g;
        return nullptr;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grad_backward_kernel, kThreads, g->smem);
    g->grid = std::min(F, std::max(1, per_sm) * sms);
    g->rec_floats = rec_floats_for(g->np, bmax);
    const size_t G = (size_t)g->grid;
    bool ok = galloc(&g->d_n, F) && galloc(&g->d_cfg, F) && galloc(&g->d_theta, 4 * (size_t)F) &&
              galloc(&g->d_gamma, F) && galloc(&g->d_y, (size_t)F * T_max) && galloc(&g->d_w, (size_t)F * T_max) &&
              galloc(&g->d_loglik, (size_t)F * T_max) && galloc(&g->d_llsum, F) && galloc(&g->d_fx, F * np) &&
              galloc(&g->d_fv, F * np) && galloc(&g->d_fs, F) && galloc(&g->d_ck, F * g->nseg * 2 * np) &&
              galloc(&g->d_cks, (size_t)F * g->nseg) && galloc(&g->d_ax, F * np) && galloc(&g->d_av, F * np) &&
              galloc(&g->d_as, F) && galloc(&g->d_seg, G * k * 2 * np) && galloc(&g->d_segs, G * k) &&
              galloc(&g->d_segts, G * k) && galloc(&g->d_status, F);
    // Records, in order of preference: every tick's record kept by the forward
    // (run records: the backward recomputes nothing) when they take at most
    // half of the free device memory (and 96 GiB); else the records of whole
    // segments, recomputed once per segment from its checkpoint, when they take
    // at most a quarter (and 16 GiB); else one tick's record per CTA.
    if (ok) {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const size_t run_bytes = run_record_bytes(g);
        if (run_bytes <= std::min(free_b / 2, (size_t)96 << 30)) alloc_run_records(g);
        if (g->d_run_rec) {
            ok = galloc(&g->d_rec, G * g->rec_floats);
        } else {
            const size_t seg_bytes = G * (size_t)k * g->rec_floats * sizeof(float);
            g->seg_rec = seg_bytes <= std::min(free_b / 4, (size_t)16 << 30) &&
                         galloc(&g->d_rec, G * k * g->rec_floats);
            if (!g->seg_rec) ok = galloc(&g->d_rec, G * g->rec_floats);
        }
    }
    ok = ok && cudaMemcpy(g->d_n, ns, F * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(g->d_cfg, cfgs, F * sizeof(svpf_config_t), cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) {
        svpf_grad_destroy(g);
        return nullptr;
    }
    return g;
}

void svpf_grad_destroy(svpf_grad_t* g) {
    if (!g) return;
    if (g->stream) cudaStreamSynchronize(g->stream);
    void* ptrs[] = {g->d_n, g->d_cfg, g->d_theta, g->d_gamma, g->d_y, g->d_w, g->d_loglik, g->d_llsum,
                    g->d_fx, g->d_fv, g->d_fs, g->d_ck, g->d_cks, g->d_ax, g->d_av, g->d_as, g->d_seg,
                    g->d_segs, g->d_rec, g->d_segts, g->d_status};
    for (void* p : ptrs) cudaFree(p);
    free_run_records(g);
    if (g->own_stream) cudaStreamDestroy(g->stream);
    delete g;
}

int svpf_grad_forward_device(svpf_grad_t* g, const float* d_theta, const float* d_gamma, const float* d_y, int T,
                             unsigned long long seed, float* d_loglik) {
    SVPF_TRACE();
    if (!g || !d_theta || !d_y || T < 1 || T > g->T_max) return SVPF_ERR_INVALID_ARG;
    g->T = T;
    g->seed = seed;
    g->u_theta = d_theta;
    g->u_gamma = d_gamma;
    g->u_y = d_y;
    if (cudaMemsetAsync(g->d_status, 0, g->F * sizeof(int), g->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    const GArgs a = make_gargs(g, d_theta, d_gamma, d_y, nullptr, d_loglik ? d_loglik : g->d_loglik);
    for (int t0 = 0; t0 < T; t0 += g->k) {
        grad_forward_kernel<<<g->grid, kThreads, g->smem, g->stream>>>(a, t0, std::min(T, t0 + g->k));
        if (cudaGetLastError() != cudaSuccess) return SVPF_ERR_CUDA;
    }
    g->forward_done = true;
    return SVPF_OK;
}

int svpf_grad_backward_device(svpf_grad_t* g, const float* d_w, double* d_grad) {
    SVPF_TRACE();
    if (!g || !g->forward_done) return SVPF_ERR_NOT_INITIALIZED;
    // statuses are the backward's own from here (parameter domain, overflow)
    if (cudaMemsetAsync(g->d_status, 0, g->F * sizeof(int), g->stream) != cudaSuccess ||
        cudaMemsetAsync(g->d_ax, 0, (size_t)g->F * g->np * sizeof(float), g->stream) != cudaSuccess ||
        cudaMemsetAsync(g->d_av, 0, (size_t)g->F * g->np * sizeof(float), g->stream) != cudaSuccess ||
        cudaMemsetAsync(g->d_as, 0, (size_t)g->F * sizeof(GAdj), g->stream) != cudaSuccess)
        return SVPF_ERR_CUDA;
    const GArgs a = make_gargs(g, g->u_theta, g->u_gamma, g->u_y, d_w, nullptr);
    const int nseg = (g->T + g->k - 1) / g->k;
    for (int sg = nseg - 1; sg >= 0; --sg) {
        grad_backward_kernel<<<g->grid, kThreads, g->smem, g->stream>>>(a, sg);
        if (cudaGetLastError() != cudaSuccess) return SVPF_ERR_CUDA;
    }
    if (d_grad) {
        // gather th[4] of every filter (strided copy)
        if (cudaMemcpy2DAsync(d_grad, 4 * sizeof(double), reinterpret_cast<const char*>(g->d_as) + offsetof(GAdj, th),
                              sizeof(GAdj), 4 * sizeof(double), g->F, cudaMemcpyDeviceToDevice,
                              g->stream) != cudaSuccess)
            return SVPF_ERR_CUDA;
    }
    return SVPF_OK;
}

int svpf_grad_forward(svpf_grad_t* g, const float* theta, const float* gamma, const float* y, int T,
                      unsigned long long seed, float* loglik, double* loglik_sum) {
    SVPF_TRACE();
    if (!g || !theta || !y || T < 1 || T > g->T_max) return SVPF_ERR_INVALID_ARG;
    const size_t F = (size_t)g->F;
    for (size_t f = 0; f < F; ++f) {
        if (!theta_ok(theta[4 * f], theta[4 * f + 1], theta[4 * f + 2], theta[4 * f + 3])) return SVPF_ERR_INVALID_ARG;
        if (gamma && !(std::fabs(gamma[f]) < INFINITY)) return SVPF_ERR_INVALID_ARG;
    }
    if (cudaMemcpyAsync(g->d_theta, theta, 4 * F * sizeof(float), cudaMemcpyHostToDevice, g->stream) != cudaSuccess)
        return SVPF_ERR_CUDA;
    if (gamma && cudaMemcpyAsync(g->d_gamma, gamma, F * sizeof(float), cudaMemcpyHostToDevice, g->stream) != cudaSuccess)
        return SVPF_ERR_CUDA;
    // y: [F][T] from the host, packed with row stride T
    if (cudaMemcpyAsync(g->d_y, y, F * T * sizeof(float), cudaMemcpyHostToDevice, g->stream) != cudaSuccess)
        return SVPF_ERR_CUDA;
    int rc = svpf_grad_forward_device(g, g->d_theta, gamma ? g->d_gamma : nullptr, g->d_y, T, seed, g->d_loglik);
    if (rc != SVPF_OK) return rc;
    if (loglik && cudaMemcpyAsync(loglik, g->d_loglik, F * T * sizeof(float), cudaMemcpyDeviceToHost, g->stream) != cudaSuccess)
        return SVPF_ERR_CUDA;
    if (loglik_sum && cudaMemcpyAsync(loglik_sum, g->d_llsum, F * sizeof(double), cudaMemcpyDeviceToHost, g->stream) != cudaSuccess)
        return SVPF_ERR_CUDA;
    if (cudaStreamSynchronize(g->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    std::vector<int> st(F);
    if (cudaMemcpy(st.data(), g->d_status, F * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SVPF_ERR_CUDA;
    for (int s : st)
        if (s) return s;
    return SVPF_OK;
}

int svpf_grad_backward(svpf_grad_t* g, const float* w, double* grad) {
    SVPF_TRACE();
    if (!g || !grad) return SVPF_ERR_INVALID_ARG;
    if (!g->forward_done) return SVPF_ERR_NOT_INITIALIZED;
    const size_t F = (size_t)g->F;
    const float* dw = nullptr;
    if (w) {
        if (cudaMemcpyAsync(g->d_w, w, F * g->T * sizeof(float), cudaMemcpyHostToDevice, g->stream) != cudaSuccess)
            return SVPF_ERR_CUDA;
        dw = g->d_w;
    }
    double* d_grad = nullptr;
    if (!galloc(&d_grad, 4 * F)) return SVPF_ERR_CUDA;
    int rc = svpf_grad_backward_device(g, dw, d_grad);
    if (rc == SVPF_OK &&
        cudaMemcpyAsync(grad, d_grad, 4 * F * sizeof(double), cudaMemcpyDeviceToHost, g->stream) != cudaSuccess)
        rc = SVPF_ERR_CUDA;
    if (rc == SVPF_OK && cudaStreamSynchronize(g->stream) != cudaSuccess) rc = SVPF_ERR_CUDA;
    cudaFree(d_grad);
    return rc;
}

int svpf_grad_get_status(svpf_grad_t* g, int* status) {
    if (!g || !status) return SVPF_ERR_INVALID_ARG;
    if (cudaStreamSynchronize(g->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    return cudaMemcpy(status, g->d_status, (size_t)g->F * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess
               ? SVPF_OK : SVPF_ERR_CUDA;
}

int svpf_grad_checkpoint_every(const svpf_grad_t* g) { return g ? g->k : 0; }

int svpf_grad_segment_records(const svpf_grad_t* g) { return g && g->seg_rec ? 1 : 0; }

int svpf_grad_set_segment_records(svpf_grad_t* g, int on) {
    if (!g) return SVPF_ERR_INVALID_ARG;
    if ((on != 0) == g->seg_rec) return SVPF_OK;
    if (cudaStreamSynchronize(g->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    float* r = nullptr;
    const size_t per = (size_t)g->grid * g->rec_floats;
    if (!galloc(&r, on ? per * g->k : per)) return SVPF_ERR_CUDA;
    cudaFree(g->d_rec);
    g->d_rec = r;
    g->seg_rec = on != 0;
    return SVPF_OK;
}

int svpf_grad_set_truncation(svpf_grad_t* g, int every) {
    if (!g || every < 0) return SVPF_ERR_INVALID_ARG;
    g->trunc = every;
    return SVPF_OK;
}

int svpf_grad_truncation(const svpf_grad_t* g) { return g ? g->trunc : 0; }

int svpf_grad_run_records(const svpf_grad_t* g) { return g && g->d_run_rec ? 1 : 0; }

int svpf_grad_set_run_records(svpf_grad_t* g, int on) {
    if (!g) return SVPF_ERR_INVALID_ARG;
    if ((on != 0) == (g->d_run_rec != nullptr)) return SVPF_OK;
    if (cudaStreamSynchronize(g->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    g->forward_done = false;   // the records come from a forward made in this mode
    if (!on) {
        free_run_records(g);
        // the backward recomputes from now on: segment records when they fit (as at create)
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const size_t seg_bytes = (size_t)g->grid * g->k * g->rec_floats * sizeof(float);
        if (!g->seg_rec && seg_bytes <= std::min(free_b / 4, (size_t)16 << 30)) svpf_grad_set_segment_records(g, 1);
        cudaGetLastError();
        return SVPF_OK;
    }
    return alloc_run_records(g) ? SVPF_OK : SVPF_ERR_CUDA;
}

int svpf_grad_set_objective(svpf_grad_t* g, int objective) {
    if (!g || (objective != SVPF_GRAD_TICK_LOGLIK && objective != SVPF_GRAD_PREDICTIVE)) return SVPF_ERR_INVALID_ARG;
    g->objective = objective;
    g->forward_done = false;
    return SVPF_OK;
}

}  // extern "C"
