/*
 * svpf_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Plain CPU restatement of one SVPF tick of the reference, written for
 * clarity, not speed: every stage is a direct O(N) or O(N^2) loop in index
 * order.  R = double is the FP64 oracle; R = float is the FP32 CPU baseline.
 * Each function cites the reference file:line whose behaviour it restates.
 *
 * Not linked into, imported by, or called from the product library.
 */
#include "svpf_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11, "Parallel random        */
/* numbers: as easy as 1, 2, 3").  Written from the paper's round function.  */
/* ------------------------------------------------------------------------ */
struct Block { uint32_t v[4]; };

Block philox(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)M0 * c0;
        uint64_t p1 = (uint64_t)M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += W0; k1 += W1;
    }
    return Block{{c0, c1, c2, c3}};
}

/* Project RNG convention (also implemented, independently, on the GPU):
 * key  = (seed_lo, seed_hi + 0x9E3779B9 * filter)
 * ctr  = (particle, draw index, tick_lo, stream) with stream 0 = normals,
 *        1 = uniforms, 2 = initial draw.
 * normal  = sqrt(-2 ln u1) cos(2 pi u2), u1 = (x0>>8 + 1) 2^-24, u2 = (x1>>8) 2^-24
 * uniform = (x0>>8 + 1) 2^-24  in (0, 1]                                      */
struct PhiloxKey { uint32_t k0, k1; };
PhiloxKey make_key(uint64_t seed, int filter) {
    return PhiloxKey{(uint32_t)seed, (uint32_t)(seed >> 32) + 0x9E3779B9u * (uint32_t)filter};
}
template <typename R>
R philox_normal(PhiloxKey k, uint32_t particle, uint32_t draw, uint32_t tick, uint32_t stream) {
    Block b = philox(k.k0, k.k1, particle, draw, tick, stream);
    R u1 = (R)((b.v[0] >> 8) + 1u) * (R)(1.0 / 16777216.0);
    R u2 = (R)(b.v[1] >> 8) * (R)(1.0 / 16777216.0);
    return std::sqrt((R)-2 * std::log(u1)) * std::cos((R)(2.0 * kPi) * u2);
}
template <typename R>
R philox_uniform(PhiloxKey k, uint32_t particle, uint32_t draw, uint32_t tick, uint32_t stream) {
    Block b = philox(k.k0, k.k1, particle, draw, tick, stream);
    return (R)((b.v[0] >> 8) + 1u) * (R)(1.0 / 16777216.0);
}

/* Noise source with one normal counter and one uniform counter per tick.  The
 * draw order per particle matches the reference's curand call order:
 * predict normal(s) then predict uniform (svpf_opt_kernels.cu:187-193), one
 * normal per Stein transport (:594 etc.), rejuvenation uniform then normal
 * (:1261-1265). */
template <typename R>
struct Noise {
    const oracle_noise* src;
    PhiloxKey key;
    int n;
    int bad = 0;
    Noise(const oracle_noise* s, int n_) : src(s), n(n_) {
        key = make_key(s->seed, s->filter_id);
    }
    R normal(int i, int k) {
        if (src->mode == 0) {
            if (k >= src->n_normal_slots) { bad = 1; return 0; }
            return (R)src->normals[(size_t)k * n + i];
        }
        return philox_normal<R>(key, (uint32_t)i, (uint32_t)k, (uint32_t)src->tick, 0u);
    }
    R uniform(int i, int k) {
        if (src->mode == 0) {
            if (k >= src->n_uniform_slots) { bad = 1; return 1; }
            return (R)src->uniforms[(size_t)k * n + i];
        }
        return philox_uniform<R>(key, (uint32_t)i, (uint32_t)k, (uint32_t)src->tick, 1u);
    }
};

template <typename R> R clampv(R x, R lo, R hi) { return std::min(std::max(x, lo), hi); }
/* clamp_logvol, svpf_opt_kernels.cu:20-22 */
template <typename R> R clamp_h(R h) { return clampv<R>(h, (R)-15, (R)5); }
/* safe_exp, svpf_opt_kernels.cu:24-26 */
template <typename R> R safe_exp(R x) { return std::exp(std::min(x, (R)20)); }

/* Student-t state noise, svpf_opt_kernels.cu:31-53.  Returns draws used. */
template <typename R>
R student_t_noise(Noise<R>& nz, int i, int& kn, R nu_state) {
    if (nu_state > (R)30) return nz.normal(i, kn++);
    R z = nz.normal(i, kn++);
    int nu_int = std::max((int)(nu_state + (R)0.5), 3);
    R chi2 = 0;
    for (int m = 0; m < nu_int; ++m) { R u = nz.normal(i, kn++); chi2 += u * u; }
    return z * std::sqrt((R)nu_int / (chi2 + (R)1e-8));
}

template <typename R>
struct Tick {
    const oracle_config& c;
    const oracle_params& p;
    oracle_ctl& s;
    int n;
    std::vector<R> h, hp, v, lw, g, curv, precond, ksd_part;
    R y_t, y_prev;

    Tick(const oracle_config& c_, const oracle_params& p_, oracle_ctl& s_, int n_)
        : c(c_), p(p_), s(s_), n(n_) {}

    /* Student-t normaliser, svpf_optimized_graph.cu:951-953 */
    R student_t_const() const {
        R nu = (R)c.nu;
        return std::lgamma((nu + 1) / 2) - std::lgamma(nu / 2) - (R)0.5 * std::log((R)kPi * nu);
    }
    /* student_t_implied_offset is fixed when the filter is created
     * (svpf_optimized_graph.cu:127-138) and read from the state afterwards. */
    R implied_offset() const { return (R)c.student_t_implied_offset; }

    /* EKF guide update, include/svpf_kernels.cuh:509-541 (FP64 here). */
    void ekf(R mu, R rho, R sigma_z, R offset) {
        double m = s.guide_mean, P = s.guide_var;
        if (!s.guide_initialized) {
            m = (double)mu;
            P = (double)sigma_z * (double)sigma_z / (1.0 - (double)rho * (double)rho);
            s.guide_initialized = 1;
        }
        double m_pred = (double)mu + (double)rho * (m - (double)mu);
        double P_pred = (double)rho * (double)rho * P + (double)sigma_z * (double)sigma_z;
        double log_y2 = std::log((double)y_t * (double)y_t + 1e-8);
        double Rn = 4.93 + 2.0;
        double S = P_pred + Rn;
        double K = P_pred / (S + 1e-8);
        double innov = log_y2 - (m_pred - (double)offset);
        s.guide_mean = m_pred + K * innov;
        s.guide_var = (1.0 - K) * P_pred;
        s.guide_K = K;
    }

    /* svpf_fused_bandwidth_kernel, svpf_opt_kernels.cu:1159-1235 */
    void bandwidth() {
        R sum = 0, sum2 = 0, mn = (R)1e10, mx = (R)-1e10;
        for (int i = 0; i < n; ++i) {
            sum += h[i]; sum2 += h[i] * h[i];
            mn = std::min(mn, h[i]); mx = std::max(mx, h[i]);
        }
        R mean = sum / (R)n;
        R var = sum2 / (R)n - mean * mean;
        R spread = mx - mn;
        R bw2_new = std::max((R)2 * var / std::log((R)n + 1), (R)1e-6);
        R bw2_prev = (R)s.bw_sq;
        R bw2 = bw2_prev > 0 ? (R)0.3 * bw2_new + (R)0.7 * bw2_prev : bw2_new;
        R a = std::fabs(y_t);
        R ema = (R)s.return_ema, rv = (R)s.return_var;
        ema = ema > 0 ? (R)0.05 * a + (R)0.95 * ema : a;
        rv = rv > 0 ? (R)0.05 * a * a + (R)0.95 * rv : a * a;
        s.return_ema = (float)ema;
        s.return_var = (float)rv;
        R ratio = a / std::max(ema, (R)1e-8);
        R spread_f = std::min(spread * (R)0.5, (R)2);
        R comb = std::max(ratio, spread_f);
        R scale = clampv<R>((R)1 - (R)0.25 * std::min(comb - 1, (R)2), (R)0.5, (R)1);
        bw2 *= scale;
        R bw = clampv<R>(std::sqrt(bw2), (R)0.01, (R)2);
        s.bw_sq = (float)bw2;
        s.bw = (float)bw;
    }

    /* svpf_fused_gradient_kernel, svpf_opt_kernels.cu:354-521 */
    void gradient(R beta, R rho, R sigma_z, R mu, R stc) {
        R lev_num = (R)p.gamma * y_prev;
        std::vector<R> mu_k(n);
        for (int k = 0; k < n; ++k) {
            R volk = std::exp(hp[k] * (R)0.5);
            mu_k[k] = mu + rho * (hp[k] - mu) + lev_num / (volk + (R)1e-8);
        }
        R s2 = sigma_z * sigma_z;
        R nu = (R)c.nu;
        for (int j = 0; j < n; ++j) {
            R hj = h[j];
            R grad_prior, hess_prior;
            if (c.use_student_t_state) {
                /* :406-447 */
                R nus = (R)c.nu_state, nus2 = nus * s2, np1 = nus + 1;
                R lmax = (R)-1e10;
                for (int k = 0; k < n; ++k) {
                    R d = hj - mu_k[k];
                    lmax = std::max(lmax, -(R)0.5 * np1 * std::log(1 + d * d / nus2));
                }
                R sr = 0, wg = 0, wh = 0;
                for (int k = 0; k < n; ++k) {
                    R d = hj - mu_k[k], d2 = d * d, den = nus2 + d2;
                    R r = std::exp(-(R)0.5 * np1 * std::log(1 + d2 / nus2) - lmax);
                    sr += r;
                    wg -= r * np1 * d / den;
                    wh += r * (-np1 * (nus2 - d2) / (den * den));
                }
                grad_prior = wg / (sr + (R)1e-8);
                hess_prior = wh / (sr + (R)1e-8);
            } else {
                /* :449-473 */
                R inv2 = (R)0.5 / s2, inv = (R)1 / s2;
                R lmax = (R)-1e10;
                for (int k = 0; k < n; ++k) {
                    R d = hj - mu_k[k];
                    lmax = std::max(lmax, -d * d * inv2);
                }
                R sr = 0, wg = 0;
                for (int k = 0; k < n; ++k) {
                    R d = hj - mu_k[k];
                    R r = std::exp(-d * d * inv2 - lmax);
                    sr += r;
                    wg -= r * d * inv;
                }
                grad_prior = wg / (sr + (R)1e-8);
                hess_prior = -inv;
            }
            /* likelihood, :475-499 */
            R vol = safe_exp(hj);
            R y2 = y_t * y_t;
            R A = y2 / (vol + (R)1e-8) / nu;
            R opA = 1 + A;
            if (c.use_fan_mode) lw[j] = 0;
            else lw[j] = stc - (R)0.5 * hj - (nu + 1) * (R)0.5 * std::log1p(std::max(A, (R)-0.999));
            R glik;
            if (c.use_exact_gradient) glik = (R)-0.5 + (R)0.5 * (nu + 1) * A / opA - (R)c.lik_offset;
            else glik = (std::log(y2 + (R)1e-10) - hj + (R)c.lik_offset) / (R)1.4;
            /* combine, :504-507 */
            R eb = c.use_fan_mode ? (R)1 : beta;
            R gg = clampv<R>(grad_prior + eb * glik, (R)-10, (R)10);
            g[j] = gg;
            /* curvature, :510-520 */
            if (c.use_newton) {
                R hl = (R)-0.5 * (nu + 1) * A / (opA * opA);
                R cv = clampv<R>(-(hl + hess_prior), (R)0.1, (R)100);
                curv[j] = cv;
                precond[j] = (R)0.7 * gg / cv;
            }
        }
    }

    /* Stein operator phi_i plus the optional per-row KSD sum.  Variants:
     * vanilla :527-599 / :618-709, Newton :742-906, full Newton :912-1103. */
    R phi_row(int i, R bw, bool want_ksd, R& ksd_row) {
        R inv_bw2 = 1 / (bw * bw);
        R sign = c.stein_repulsive_sign == 1 ? (R)1 : (R)-1;
        bool newton = c.use_newton != 0, full = newton && c.use_full_newton;
        const std::vector<R>& score = (newton && !full) ? precond : g;
        R hi = h[i], si = score[i];
        R ks = 0, gk = 0, hw = 0, kn = 0, ksd = 0;
        for (int j = 0; j < n; ++j) {
            R d = hi - h[j];
            R dist2 = d * d * inv_bw2;
            R K = 1 / (1 + dist2);
            R K2 = K * K;
            ks += K * score[j];
            R rep = sign * 2 * d * inv_bw2 * K2;
            if (newton && !full) rep /= curv[j];
            gk += rep;
            if (full) {
                hw += curv[j] * K + 2 * inv_bw2 * K2 * std::fabs(3 * dist2 - 1);
                kn += K;
            }
            if (want_ksd) {
                R gxk = -2 * d * inv_bw2 * K2;
                R hxy = 2 * inv_bw2 * K2 * (4 * dist2 * K - 1);
                ksd += K * si * score[j] + si * (-gxk) + score[j] * gxk + hxy;
            }
        }
        ksd_row = ksd;
        R phi = (ks + gk) / (R)n;
        if (full) {
            R H = clampv<R>(hw / std::max(kn, (R)1e-6), (R)0.1, (R)100);
            phi = phi / H * (R)0.7;
        }
        return phi;
    }

    /* Transport: RMSProp + drift + SVLD diffusion + clamp (Jacobi: all rows
     * read the pre-iteration h), e.g. svpf_opt_kernels.cu:1078-1102. */
    R transport(R eps_step, R bf, R temp, bool want_ksd, Noise<R>& nz, int kn) {
        R bw = (R)s.bw;
        std::vector<R> hn(n);
        R ksd_sum = 0;
        for (int i = 0; i < n; ++i) {
            R kr = 0;
            R phi = phi_row(i, bw, want_ksd, kr);
            ksd_sum += kr;
            R rr = (R)c.rmsprop_rho;
            R vn = rr * v[i] + (1 - rr) * phi * phi;
            v[i] = vn;
            R es = eps_step * bf;
            R drift = es * phi / std::sqrt(vn + (R)c.rmsprop_eps);
            R diff = 0;
            if (temp > (R)1e-6) diff = std::sqrt(2 * es * temp) * nz.normal(i, kn);
            hn[i] = clamp_h(h[i] + drift + diff);
        }
        h.swap(hn);
        return ksd_sum;
    }

    /* Heun (use_heun), svpf_optimized_graph.cu:1147-1232 with kernels
     * svpf_opt_kernels.cu:1293-1566. */
    R heun(R beta, R bf, R temp, R eps_step, bool last, Noise<R>& nz, int kn,
           R rho, R sz, R mu, R stc) {
        std::vector<R> h0 = h;
        gradient(beta, rho, sz, mu, stc);
        R bw = (R)s.bw, dummy;
        bool full = c.use_newton && c.use_full_newton;
        auto op = [&](int i) -> R {
            /* svpf_stein_operator[_full_newton]_kernel: raw score, no Newton
             * (non-full) variant. */
            R inv_bw2 = 1 / (bw * bw);
            R sign = c.stein_repulsive_sign == 1 ? (R)1 : (R)-1;
            R ks = 0, gk = 0, hw = 0, kn2 = 0;
            for (int j = 0; j < n; ++j) {
                R d = h[i] - h[j];
                R dist2 = d * d * inv_bw2;
                R K = 1 / (1 + dist2), K2 = K * K;
                if (full) { hw += curv[j] * K + 2 * inv_bw2 * K2 * std::fabs(3 * dist2 - 1); kn2 += K; }
                ks += K * g[j];
                gk += sign * 2 * d * inv_bw2 * K2;
            }
            R phi = (ks + gk) / (R)n;
            if (full) {
                R H = clampv<R>(hw / std::max(kn2, (R)1e-6), (R)0.1, (R)100);
                phi = phi / H * (R)0.7;
            }
            return phi;
        };
        (void)dummy;
        std::vector<R> phi0(n), phi1(n);
        for (int i = 0; i < n; ++i) phi0[i] = op(i);
        R es = eps_step * bf;
        for (int i = 0; i < n; ++i)
            h[i] = clamp_h(h0[i] + es * phi0[i] / std::sqrt(v[i] + (R)c.rmsprop_eps));
        std::vector<R> g0 = g;  /* grad at h0 kept for the KSD below */
        gradient(beta, rho, sz, mu, stc);
        for (int i = 0; i < n; ++i) phi1[i] = op(i);
        R ksd_sum = 0;
        if (last) {
            /* svpf_heun_corrector_ksd_kernel uses h_orig with the grad buffer,
             * which at this point holds the gradient at the predicted h. */
            R inv_bw2 = 1 / (bw * bw);
            for (int i = 0; i < n; ++i) {
                R si = g[i], acc = 0;
                for (int j = 0; j < n; ++j) {
                    R d = h0[i] - h0[j];
                    R dist2 = d * d * inv_bw2;
                    R K = 1 / (1 + dist2), K2 = K * K;
                    R gxk = -2 * d * inv_bw2 * K2;
                    R hxy = 2 * inv_bw2 * K2 * (4 * dist2 * K - 1);
                    acc += K * si * g[j] + si * (-gxk) + g[j] * gxk + hxy;
                }
                ksd_sum += acc;
            }
        }
        for (int i = 0; i < n; ++i) {
            R pa = (R)0.5 * (phi0[i] + phi1[i]);
            R rr = (R)c.rmsprop_rho;
            R vn = rr * v[i] + (1 - rr) * pa * pa;
            v[i] = vn;
            R diff = 0;
            if (temp > (R)1e-6) diff = std::sqrt(2 * es * temp) * nz.normal(i, kn);
            h[i] = clamp_h(h0[i] + es * pa / std::sqrt(vn + (R)c.rmsprop_eps) + diff);
        }
        (void)g0;
        return ksd_sum;
    }

    /* Adaptive beta, svpf_optimized_graph.cu:1066-1092 */
    static R adaptive_beta(R ksd_prev, int ai, int na) {
        if (ai == na - 1) return 1;
        R b;
        if (ksd_prev > (R)0.5) b = (R)0.3;
        else if (ksd_prev < (R)0.05) b = (R)0.8;
        else b = (R)0.3 + ((R)0.5 - ksd_prev) / (R)0.45 * (R)0.5;
        b *= (R)0.5 + (R)0.5 * ((R)(ai + 1) / (R)na);
        return clampv<R>(b, (R)0.1, (R)1);
    }

    /* Smoother, svpf_optimized_graph.cu:658-737 */
    R smooth(R hm, R hvar) {
        if (!c.use_smoothing) return hm;
        int k = std::min(std::max(c.smooth_lag, 1), ORACLE_SMOOTH_MAX_LAG);
        int head = s.smooth_head;
        s.smooth_h_mean[head] = (float)hm;
        s.smooth_h_var[head] = (float)hvar;
        s.smooth_y[head] = (float)y_t;
        s.smooth_head = (head + 1) % k;
        if (s.timestep >= k) {
            R rho = (R)p.rho;
            R mu = c.use_adaptive_mu ? (R)s.mu_state : (R)p.mu;
            R q = (R)p.sigma_z * (R)p.sigma_z;
            for (int lag = 1; lag < k; ++lag) {
                int ic = (s.smooth_head - lag - 1 + k) % k;
                int inx = (s.smooth_head - lag + k) % k;
                R hc = s.smooth_h_mean[ic], hn = s.smooth_h_mean[inx], vc = s.smooth_h_var[ic];
                R pv = rho * rho * vc + q;
                R J = rho * vc / (pv + (R)1e-8);
                s.smooth_h_mean[ic] = (float)(hc + J * (hn - (mu + rho * (hc - mu))));
                s.smooth_h_var[ic] = (float)(vc * (1 - J * rho));
            }
        }
        /* svpf_get_smoothed_output :720-737 (k not re-floored at 1 there) */
        int k2 = std::min(c.smooth_lag, ORACLE_SMOOTH_MAX_LAG);
        if (k2 < 1 || s.timestep < k2) return hm;
        int ol = c.smooth_output_lag;
        if (ol <= 0) return hm;
        if (ol >= k2) ol = k2 - 1;
        int idx = (s.smooth_head - ol - 1 + k2) % k2;
        return (R)s.smooth_h_mean[idx];
    }

    /* Two-factor tick: svpf_step_two_factor, svpf_optimized_graph.cu:744-897,
     * kernels src/svpf_two_factor.cu, host EKF include/svpf_two_factor.cuh:245-300.
     * h/hp/v hold [fast (n) ; slow (n)]. */
    int run2f(R yt, R yp, Noise<R>& nz, oracle_out* out) {
        y_t = yt; y_prev = yp;
        const R rf = (R)c.rho_fast, sf = (R)c.sigma_fast, rs = (R)c.rho_slow, ss = (R)c.sigma_slow;
        const R mu = (R)p.mu, nu = (R)c.nu;
        /* predict, svpf_two_factor.cu:55-90 */
        for (int i = 0; i < n; ++i) {
            R hf = h[i], hs = h[n + i];
            hp[i] = hf; hp[n + i] = hs;
            R zf = nz.normal(i, 0), zs = nz.normal(i, 1);
            if (c.use_mim) {
                R u = nz.uniform(i, 0);
                if (u < (R)c.mim_jump_prob) zf *= (R)c.mim_jump_scale;
            }
            h[i] = clamp_h(rf * hf + sf * zf);
            h[n + i] = clamp_h(rs * hs + ss * zs);
        }
        /* EKF with innovation split (FP64 here) + guide, :781-807 */
        if (c.use_guide) {
            double gmf = s.guide_mean_fast, gms = s.guide_mean_slow, gvf = s.guide_var_fast, gvs = s.guide_var_slow;
            if (!s.guide_2f_initialized) {
                gmf = 0.0; gms = 0.0;
                gvf = (double)sf * sf / (1.0 - (double)rf * rf);
                gvs = (double)ss * ss / (1.0 - (double)rs * rs);
                s.guide_2f_initialized = 1;
            }
            const double pf = (double)rf * gmf, ps = (double)rs * gms;
            const double Pf = (double)rf * rf * gvf + (double)sf * sf;
            const double Ps = (double)rs * rs * gvs + (double)ss * ss;
            const double implied = std::log((double)y_t * y_t + 1e-8) + (double)c.student_t_implied_offset;
            const double innov = implied - ((double)mu + pf + ps);
            const double S = Pf + Ps + (4.93 + 2.0);
            const double Kf = Pf / (S + 1e-8), Ks = Ps / (S + 1e-8);
            s.guide_mean_fast = pf + Kf * innov;
            s.guide_mean_slow = ps + Ks * innov;
            s.guide_var_fast = std::max((1.0 - Kf) * Pf, 1e-6);
            s.guide_var_slow = std::max((1.0 - Ks) * Ps, 1e-6);
            const R g = (R)c.guide_strength;
            const R cmf = (R)s.h_fast_mean, cms = (R)s.h_slow_mean;
            const R gf = (R)s.guide_mean_fast, gsl = (R)s.guide_mean_slow;
            for (int i = 0; i < n; ++i) {
                if (c.use_guide_preserving) {
                    h[i] = clamp_h(((1 - g) * cmf + g * gf) + (h[i] - cmf));
                    h[n + i] = clamp_h(((1 - g) * cms + g * gsl) + (h[n + i] - cms));
                } else {
                    h[i] = clamp_h((1 - g) * h[i] + g * gf);
                    h[n + i] = clamp_h((1 - g) * h[n + i] + g * gsl);
                }
            }
        }
        /* Silverman bandwidth per factor, svpf_two_factor.cu:256-318 */
        R bw2[2];
        for (int k = 0; k < 2; ++k) {
            R sum = 0, sum2 = 0;
            for (int i = 0; i < n; ++i) { R x = h[k * n + i]; sum += x; sum2 += x * x; }
            R mean = sum / (R)n, var = sum2 / (R)n - mean * mean;
            R sd = std::sqrt(std::max(var, (R)1e-8));
            R bw = (R)1.06 * sd * std::pow((R)n, (R)-0.2);
            bw2[k] = std::max(bw, k == 0 ? (R)c.bw_floor_fast : (R)c.bw_floor_slow);
        }
        /* Stein loop: n_stein_steps per stage, beta = (a+1)/na, step 0.5/n_stein */
        const int na = c.use_annealing ? c.n_anneal_steps : 1;   /* 0 stages: no Stein step */
        const R base_step = (R)0.5 / (R)c.n_stein_steps;
        const R stc = student_t_const();
        const R sign = c.stein_repulsive_sign == 1 ? (R)1 : (R)-1;
        std::vector<R> gfa(n), gsa(n), hn(2 * n);
        int kn = 2;
        for (int a = 0; a < na; ++a) {
            const R beta = (R)(a + 1) / (R)na;
            const R temp = c.use_svld ? (R)c.temperature : (R)0;
            for (int st = 0; st < c.n_stein_steps; ++st) {
                /* gradient, svpf_two_factor.cu:166-243 */
                const R sf2 = sf * sf + (R)1e-8, ss2 = ss * ss + (R)1e-8;
                const R wf = sf2 / (sf2 + ss2), ws = 1 - wf;
                for (int i = 0; i < n; ++i) {
                    const R hf = h[i], hs = h[n + i];
                    const R hc = mu + hf + hs;
                    const R y2 = y_t * y_t;
                    const R ratio = y2 / (nu * std::exp(hc) + (R)1e-8);
                    lw[i] = stc - (R)0.5 * hc - (R)0.5 * (nu + 1) * std::log(1 + ratio);
                    R lg;
                    if (c.use_exact_gradient) lg = (R)-0.5 + (R)0.5 * (nu + 1) * ratio / (1 + ratio + (R)1e-8);
                    else lg = (R)0.5 * (std::log(y2 + (R)1e-8) - hc);
                    gfa[i] = -(hf - rf * hp[i]) / sf2 + beta * wf * lg;
                    gsa[i] = -(hs - rs * hp[n + i]) / ss2 + beta * ws * lg;
                }
                /* two vanilla transports, svpf_opt_kernels.cu:527-599 (fast, then slow) */
                for (int k = 0; k < 2; ++k) {
                    const R* hh = &h[k * n];
                    const std::vector<R>& gg = k == 0 ? gfa : gsa;
                    const R inv_bw2 = 1 / (bw2[k] * bw2[k]);
                    for (int i = 0; i < n; ++i) {
                        R ks = 0, gk = 0;
                        for (int j = 0; j < n; ++j) {
                            const R d = hh[i] - hh[j];
                            const R K = 1 / (1 + d * d * inv_bw2);
                            ks += K * gg[j];
                            gk += sign * 2 * d * inv_bw2 * K * K;
                        }
                        const R phi = (ks + gk) / (R)n;
                        const R rr = (R)c.rmsprop_rho;
                        R& vv = v[k * n + i];
                        vv = rr * vv + (1 - rr) * phi * phi;
                        const R es = base_step * beta;
                        R diff = 0;
                        if (temp > (R)1e-6) diff = std::sqrt(2 * es * temp) * nz.normal(i, kn + k);
                        hn[k * n + i] = clamp_h(hh[i] + es * phi / std::sqrt(vv + (R)c.rmsprop_eps) + diff);
                    }
                }
                for (int i = 0; i < 2 * n; ++i) h[i] = hn[i];
                if (temp > (R)1e-6) kn += 2;
            }
        }
        /* outputs, svpf_two_factor.cu:368-470 */
        R mx = (R)-1e30, sfm = 0, ssm = 0, svol = 0;
        for (int i = 0; i < n; ++i) {
            mx = std::max(mx, lw[i]);
            sfm += h[i]; ssm += h[n + i];
            svol += std::exp((R)0.5 * (mu + h[i] + h[n + i]));
        }
        R se = 0;
        for (int i = 0; i < n; ++i) se += std::exp(lw[i] - mx);
        const R ll = mx + std::log(std::max(se / (R)n, (R)1e-10));
        const R mf = sfm / (R)n, ms = ssm / (R)n;
        const R hm = mu + mf + ms, vol = svol / (R)n;
        s.h_fast_mean = (float)mf;
        s.h_slow_mean = (float)ms;
        s.h_mean_prev = (float)hm;
        s.vol_prev = (float)vol;
        s.loglik_sum += (double)ll;
        s.timestep += 1;
        out->loglik = (float)ll;
        out->vol = (float)vol;
        out->h_mean = (float)hm;
        out->h_mean_raw = (float)hm;
        /* the single-factor bandwidth, KSD and step counter are left as they were */
        out->bw = (float)bw2[0];
        out->ksd = s.ksd_last;
        out->steps_used = std::max(na, 0) * c.n_stein_steps;
        out->rejuv_fired = 0;
        return nz.bad ? -3 : 0;
    }

    int run(R yt, R yp, Noise<R>& nz, oracle_out* out) {
        y_t = yt; y_prev = yp;
        const int t = s.timestep;
        /* effective parameters, svpf_optimized_graph.cu:933-948 */
        R mu_eff = c.use_adaptive_mu ? (R)s.mu_state : (R)p.mu;
        R sz_eff = (R)p.sigma_z;
        if (c.use_adaptive_sigma && t > 0) {
            R ve = std::max((R)s.vol_prev, (R)1e-4);
            R z = std::fabs(y_t) / ve;
            R boost = 1;
            if (z > (R)c.sigma_boost_threshold) {
                R sev = std::min((z - (R)c.sigma_boost_threshold) / 3, (R)1);
                boost = 1 + ((R)c.sigma_boost_max - 1) * sev;
            }
            sz_eff = (R)p.sigma_z * boost;
            s.sigma_z_effective = (float)sz_eff;
        }
        R stc = student_t_const();
        R off = implied_offset();
        R rho_up = c.use_asymmetric_rho ? (R)c.rho_up : (R)p.rho;
        R rho_dn = c.use_asymmetric_rho ? (R)c.rho_down : (R)p.rho;
        R drho = c.use_local_params ? (R)c.delta_rho : 0;
        R dsig = c.use_local_params ? (R)c.delta_sigma : 0;

        int kn = 0, ku = 0;
        /* predict, svpf_opt_kernels.cu:125-276 */
        {
            R hbar = (R)s.h_mean_prev;
            for (int i = 0; i < n; ++i) {
                R hi = h[i], hpi = hp[i];
                hp[i] = hi;
                int kk = 0;
                R noise = c.use_student_t_state ? student_t_noise<R>(nz, i, kk, (R)c.nu_state)
                                                : nz.normal(i, kk++);
                if (i == 0) kn = kk;
                R lev = (R)p.gamma * y_prev / (safe_exp(hi / 2) + (R)1e-8);
                if (c.use_guided || c.use_mim) {
                    R dev = hi - hbar;
                    R rho_adj = drho * std::tanh(dev);
                    R sscale = 1 + dsig * std::fabs(dev);
                    R sel = nz.uniform(i, 0);
                    R scale = sel < (R)c.mim_jump_prob ? (R)c.mim_jump_scale : (R)1;
                    R br = hi > hpi ? rho_up : rho_dn;
                    R rho = clampv<R>(br + rho_adj, (R)0, (R)0.999);
                    R sl = sz_eff * sscale;
                    R mprior = mu_eff + rho * (hi - mu_eff) + lev;
                    if (c.use_guided) {
                        R ly2 = std::log(y_t * y_t + (R)1e-10);
                        R mimp = std::max(ly2 + off, (R)-5);
                        R z = (mimp - mprior) / (R)2.5;
                        R act = z > (R)c.guided_innovation_threshold
                                    ? std::tanh(z - (R)c.guided_innovation_threshold) : (R)0;
                        R ga = (R)c.guided_alpha_base + ((R)c.guided_alpha_shock - (R)c.guided_alpha_base) * act;
                        mprior = (1 - ga) * mprior + ga * mimp;
                    }
                    h[i] = clamp_h(mprior + sl * scale * noise);
                } else {
                    h[i] = clamp_h(mu_eff + (R)p.rho * (hi - mu_eff) + sz_eff * noise + lev);
                }
            }
            if (c.use_guided || c.use_mim) ku = 1;
        }

        /* guide, svpf_optimized_graph.cu:1006-1039 */
        R gs = (R)c.guide_strength_base;
        if (c.use_guide && c.use_adaptive_guide && t > 0) {
            R ve = std::max((R)s.vol_prev, (R)1e-4);
            R z = std::fabs(y_t) / ve;
            R ih = std::log(y_t * y_t + (R)1e-8) + off;
            R he = std::log(ve * ve + (R)1e-8);
            if (ih - he > 0 && z > (R)c.guide_innovation_threshold) {
                R sev = std::min((z - (R)c.guide_innovation_threshold) / 3, (R)1);
                gs = (R)c.guide_strength_base + ((R)c.guide_strength_max - (R)c.guide_strength_base) * sev;
            }
        }
        if (c.use_guide) {
            ekf(mu_eff, (R)p.rho, (R)p.sigma_z, off);
            R gm = (R)s.guide_mean;
            if (c.use_guide_preserving) {
                R cm = (R)s.h_mean_prev;
                R nm = (1 - gs) * cm + gs * gm;
                for (int i = 0; i < n; ++i) h[i] = clamp_h(nm + (h[i] - cm));
            } else {
                for (int i = 0; i < n; ++i) h[i] = clamp_h(h[i] + gs * (gm - h[i]));
            }
        }

        bandwidth();

        /* Stein budget / beta schedule, svpf_optimized_graph.cu:1057-1138 */
        int na = c.use_annealing ? std::max(c.n_anneal_steps, 1) : 1;
        R eps_step = (R)0.1 * (c.use_guide ? (R)0.5 : (R)1);
        int budget;
        if (t < 10) budget = c.stein_max_steps;
        else {
            /* a discrete decision: evaluated in float exactly as the host does */
            float kn01 = (s.ksd_prev - 0.05f) / (0.50f - 0.05f);
            kn01 = std::min(std::max(kn01, 0.0f), 1.0f);
            budget = c.stein_min_steps + (int)(kn01 * (float)(c.stein_max_steps - c.stein_min_steps));
        }
        if (budget < 0) budget = 0;
        int total = 0;
        for (int ai = 0; ai < na; ++ai) {
            R beta;
            if (!c.use_annealing) beta = 1;
            else if (c.use_adaptive_beta) beta = adaptive_beta((R)s.ksd_prev, ai, na);
            else { static const double sch[3] = {0.3, 0.65, 1.0}; beta = (R)sch[ai % 3]; }
            R bf = std::sqrt(beta);
            R temp = c.use_svld ? (R)c.temperature : (R)0;
            int si = budget / na;
            if (ai == na - 1) si = budget - si * (na - 1);
            for (int st = 0; st < si; ++st) {
                ++total;
                bool last = (ai == na - 1) && (st == si - 1);
                R ksd_sum;
                if (c.use_heun) {
                    ksd_sum = heun(beta, bf, temp, eps_step, last, nz, kn, (R)p.rho, sz_eff, mu_eff, stc);
                } else {
                    gradient(beta, (R)p.rho, sz_eff, mu_eff, stc);
                    ksd_sum = transport(eps_step, bf, temp, last, nz, kn);
                }
                if (temp > (R)1e-6) ++kn;
                if (last) {
                    R k2 = ksd_sum / ((R)n * (R)n);
                    s.ksd_last = (float)std::sqrt(std::max(k2, (R)0));
                }
            }
        }
        s.stein_steps_used = total;

        /* rejuvenation, svpf_optimized_graph.cu:1328-1341 + kernel :1248-1275 */
        int fired = 0;
        if (c.use_rejuvenation && c.use_guide && t > 10 && (R)s.ksd_prev > (R)c.rejuv_ksd_threshold) {
            fired = 1;
            R gstd = std::sqrt(std::max((R)s.guide_var, (R)1e-6));
            R gm = (R)s.guide_mean;
            R b = (R)c.rejuv_blend;
            for (int i = 0; i < n; ++i) {
                R u = nz.uniform(i, ku);
                if (u < (R)c.rejuv_prob) {
                    R z = nz.normal(i, kn);
                    h[i] = clamp_h((1 - b) * h[i] + b * (gm + gstd * z));
                }
            }
        }

        /* outputs, svpf_opt_kernels.cu:1109-1153 */
        R mx = (R)-1e10;
        for (int i = 0; i < n; ++i) mx = std::max(mx, lw[i]);
        R se = 0, sv = 0, sh = 0;
        for (int i = 0; i < n; ++i) {
            se += std::exp(lw[i] - mx);
            sv += safe_exp(h[i] * (R)0.5);
            sh += h[i];
        }
        R ll = mx + std::log(std::max(se / (R)n, (R)1e-10));
        R vol = sv / (R)n;
        R hm = sh / (R)n;
        s.h_mean_prev = (float)hm;

        /* host tail, svpf_optimized_graph.cu:1361-1388 */
        R bwl = (R)s.bw;
        R hm_out = smooth(hm, bwl * bwl);
        s.vol_prev = (float)vol;
        s.ksd_prev = s.ksd_last;
        if (c.use_adaptive_mu && t > 10) {
            /* svpf_adaptive_mu_update :619-642 */
            R mp = (R)s.mu_state, Pp = (R)s.mu_var + (R)c.mu_process_var;
            R Rm = (R)c.mu_obs_var_scale * bwl * bwl;
            R K = Pp / (Pp + Rm + (R)1e-8);
            s.mu_state = (float)clampv<R>(mp + K * (hm - mp), (R)c.mu_min, (R)c.mu_max);
            s.mu_var = (float)((1 - K) * Pp);
        }
        s.loglik_sum += (double)ll;
        s.timestep = t + 1;

        out->loglik = (float)ll;
        out->vol = (float)vol;
        out->h_mean = (float)hm_out;
        out->h_mean_raw = (float)hm;
        out->bw = s.bw;
        out->ksd = s.ksd_last;
        out->steps_used = total;
        out->rejuv_fired = fired;
        return nz.bad ? -3 : 0;
    }
};

template <typename R>
int tick_impl(const oracle_config* cfg, const oracle_params* p, oracle_ctl* ctl, int n,
              double* h, double* hp, double* v, double* lw, float yt, float yp,
              const oracle_noise* noise, oracle_out* out) {
    Tick<R> tk(*cfg, *p, *ctl, n);
    const int m = cfg->use_two_factor ? 2 * n : n;   /* two-factor: [fast; slow] */
    tk.h.assign(h, h + m); tk.hp.assign(hp, hp + m); tk.v.assign(v, v + m);
    tk.lw.assign(lw, lw + n);
    tk.g.assign(n, 0); tk.curv.assign(n, 1); tk.precond.assign(n, 0);
    Noise<R> nz(noise, n);
    int rc = cfg->use_two_factor ? tk.run2f((R)yt, (R)yp, nz, out) : tk.run((R)yt, (R)yp, nz, out);
    for (int i = 0; i < m; ++i) { h[i] = tk.h[i]; hp[i] = tk.hp[i]; v[i] = tk.v[i]; }
    for (int i = 0; i < n; ++i) lw[i] = tk.lw[i];
    return rc;
}

}  // namespace

/* ======================================================================== */
/* Gradient oracle: d(sum_t w_t loglik_t) / d(mu, rho, sigma_z, nu) of a     */
/* whole run (initialisation included) under common random numbers, by       */
/* forward-mode automatic differentiation in FP64 (a value plus four          */
/* tangents carried through every operation).  It restates the single-factor  */
/* tick for the differentiable configuration (see svpf_oracle_grad_supported) */
/* with the same formulas and reference citations as Tick::run above, but     */
/* keeps every quantity in FP64 (no float rounding of the stored bandwidth).  */
/* Decisions that are piecewise constant in theta (the Stein budget, adaptive */
/* beta, clamps, the MIM jump selection) are taken on the primal values.      */
/* ======================================================================== */
namespace {

struct Dual {
    double v;
    double d[4];
    Dual() : v(0), d{0, 0, 0, 0} {}
    Dual(double x) : v(x), d{0, 0, 0, 0} {}  // NOLINT: implicit from constants
    static Dual var(double x, int k) { Dual r(x); r.d[k] = 1; return r; }
};
inline Dual mk(double v, const Dual& a, double da) {   /* f(a) with f'(a) = da */
    Dual r(v);
    for (int k = 0; k < 4; ++k) r.d[k] = da * a.d[k];
    return r;
}
inline Dual operator+(const Dual& a, const Dual& b) { Dual r(a.v + b.v); for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] + b.d[k]; return r; }
inline Dual operator-(const Dual& a, const Dual& b) { Dual r(a.v - b.v); for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] - b.d[k]; return r; }
inline Dual operator-(const Dual& a) { Dual r(-a.v); for (int k = 0; k < 4; ++k) r.d[k] = -a.d[k]; return r; }
inline Dual operator*(const Dual& a, const Dual& b) { Dual r(a.v * b.v); for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k]; return r; }
inline Dual operator/(const Dual& a, const Dual& b) {
    Dual r(a.v / b.v);
    for (int k = 0; k < 4; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
    return r;
}
inline Dual& operator+=(Dual& a, const Dual& b) { a = a + b; return a; }
inline Dual& operator-=(Dual& a, const Dual& b) { a = a - b; return a; }
inline Dual& operator*=(Dual& a, const Dual& b) { a = a * b; return a; }
inline bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
inline bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
inline double val(const Dual& a) { return a.v; }
inline double val(double a) { return a; }

/* psi(x), x > 0: recurrence psi(x) = psi(x+1) - 1/x up to x >= 8 (at most
 * eight shifts), then the asymptotic series (Abramowitz & Stegun 6.3.18);
 * NaN for x <= 0 or NaN. */
double digamma(double x) {
    if (!(x > 0)) return std::nan("");
    double acc = 0;
    for (int k = 0; k < 8 && x < 8; ++k) { acc -= 1 / x; x += 1; }
    double r = 1 / x, r2 = r * r;
    return acc + std::log(x) - 0.5 * r -
           r2 * (1.0 / 12 - r2 * (1.0 / 120 - r2 * (1.0 / 252 - r2 * (1.0 / 240 - r2 * (1.0 / 132)))));
}

inline Dual dexp(const Dual& a) { double e = std::exp(a.v); return mk(e, a, e); }
inline Dual dlog(const Dual& a) { return mk(std::log(a.v), a, 1 / a.v); }
inline Dual dlog1p(const Dual& a) { return mk(std::log1p(a.v), a, 1 / (1 + a.v)); }
inline Dual dsqrt(const Dual& a) { double s = std::sqrt(a.v); return mk(s, a, 0.5 / s); }
inline Dual dlgamma(const Dual& a) { return mk(std::lgamma(a.v), a, digamma(a.v)); }
inline Dual dmin(const Dual& a, const Dual& b) { return b.v < a.v ? b : a; }
inline Dual dmax(const Dual& a, const Dual& b) { return b.v > a.v ? b : a; }
inline Dual dclamp(const Dual& x, double lo, double hi) { return dmin(dmax(x, Dual(lo)), Dual(hi)); }
inline Dual dclamp_h(const Dual& x) { return dclamp(x, -15, 5); }
inline Dual dsafe_exp(const Dual& x) { return dexp(dmin(x, Dual(20))); }

/* One filter of the differentiable configuration.  State carried between
 * ticks that depends on theta is Dual; the return EMAs depend on y only. */
struct GradFilter {
    const oracle_config& c;
    int n;
    double gamma;
    int predictive = 0;              /* 1: log mean_i p(y_t | predicted h_i) instead of the tick loglik */
    Dual mu, rho, sz, nu;            /* theta */
    std::vector<Dual> h, v, lw, g, curv;
    Dual bw_sq, h_mean_prev, gm, gP; /* bandwidth EMA, previous mean, EKF mean/variance */
    int guide_initialized = 0, timestep = 0;
    double return_ema = 0, return_var = 0, ksd_prev = 1e10;
    Dual bw;

    GradFilter(const oracle_config& c_, int n_, const double* theta, double gamma_)
        : c(c_), n(n_), gamma(gamma_) {
        mu = Dual::var(theta[0], 0);
        rho = Dual::var(theta[1], 1);
        sz = Dual::var(theta[2], 2);
        nu = Dual::var(theta[3], 3);
        h.assign(n, Dual()); v.assign(n, Dual()); lw.assign(n, Dual()); g.assign(n, Dual()); curv.assign(n, Dual(1));
        bw_sq = Dual(0);
        h_mean_prev = Dual(-3.5);   /* svpf_optimized_graph.cu:492-494 */
    }

    /* Truncation: the carried state keeps its values and loses its tangents. */
    void hold_state() {
        for (int i = 0; i < n; ++i) {
            h[i] = Dual(h[i].v);
            v[i] = Dual(v[i].v);
        }
        bw_sq = Dual(bw_sq.v);
        h_mean_prev = Dual(h_mean_prev.v);
        gm = Dual(gm.v);
        gP = Dual(gP.v);
    }

    /* svpf_initialize, svpf_optimized_graph.cu:349-451 (single-factor part) */
    void initialize(Noise<double>& nz_init, const float* init_normals, PhiloxKey key) {
        Dual var = sz * sz / (Dual(1) - rho * rho + Dual(1e-6));
        Dual sd = dsqrt(var);
        for (int i = 0; i < n; ++i) {
            double z = init_normals ? (double)init_normals[i] : philox_normal<double>(key, (uint32_t)i, 0u, 0u, 2u);
            h[i] = dclamp_h(mu + sd * Dual(z));
            v[i] = Dual(0);
        }
        (void)nz_init;
        guide_initialized = 0;
        gm = mu;
        gP = var;
        ksd_prev = 1e10;
        timestep = 0;
    }

    Dual stc() const {   /* svpf_optimized_graph.cu:951-953 */
        return dlgamma((nu + Dual(1)) * Dual(0.5)) - dlgamma(nu * Dual(0.5)) - Dual(0.5) * dlog(Dual(kPi) * nu);
    }

    /* one tick; returns loglik_t.  Citations as in Tick::run. */
    Dual tick(double y_t, double y_prev, Noise<double>& nz) {
        const int t = timestep;
        const double off = c.student_t_implied_offset;
        const Dual st = stc();
        /* predict (:125-276) and prior means (:384-392) from tick-start positions */
        std::vector<Dual> mu_k(n);
        for (int i = 0; i < n; ++i) {
            const Dual hi = h[i];
            const double z = nz.normal(i, 0);
            const Dual lev = Dual(gamma * y_prev) / (dsafe_exp(hi * Dual(0.5)) + Dual(1e-8));
            mu_k[i] = mu + rho * (hi - mu) + Dual(gamma * y_prev) / (dexp(hi * Dual(0.5)) + Dual(1e-8));
            if (c.use_mim) {
                const double sel = nz.uniform(i, 0);
                const double scale = sel < (double)c.mim_jump_prob ? (double)c.mim_jump_scale : 1.0;
                const Dual r = dclamp(rho, 0, 0.999);
                h[i] = dclamp_h(mu + r * (hi - mu) + lev + sz * Dual(scale * z));
            } else {
                h[i] = dclamp_h(mu + rho * (hi - mu) + sz * Dual(z) + lev);
            }
        }
        /* predictive log-likelihood log p(y_t | y_1:t-1): Student-t log density
         * of y_t averaged over the predicted particles (before guide and Stein) */
        Dual ll_pred(0);
        if (predictive) {
            const Dual st0 = stc();
            std::vector<Dual> lp(n);
            Dual mxp(-1e10);
            for (int i = 0; i < n; ++i) {
                const Dual A = Dual(y_t * y_t) / (dsafe_exp(h[i]) + Dual(1e-8)) / nu;
                lp[i] = st0 - Dual(0.5) * h[i] - (nu + Dual(1)) * Dual(0.5) * dlog1p(A);
                mxp = dmax(mxp, lp[i]);
            }
            Dual sp(0);
            for (int i = 0; i < n; ++i) sp += dexp(lp[i] - mxp);
            ll_pred = mxp + dlog(dmax(sp / Dual(n), Dual(1e-10)));
        }
        /* EKF guide (svpf_kernels.cuh:509-541) and the preserving shift (:1006-1039) */
        if (c.use_guide) {
            if (!guide_initialized) {
                gm = mu;
                gP = sz * sz / (Dual(1) - rho * rho);
                guide_initialized = 1;
            }
            const Dual m_pred = mu + rho * (gm - mu);
            const Dual P_pred = rho * rho * gP + sz * sz;
            const double log_y2 = std::log(y_t * y_t + 1e-8);
            const Dual K = P_pred / (P_pred + Dual(4.93 + 2.0) + Dual(1e-8));
            gm = m_pred + K * (Dual(log_y2) - (m_pred - Dual(off)));
            gP = (Dual(1) - K) * P_pred;
            const double gs = c.guide_strength_base;
            if (c.use_guide_preserving) {
                const Dual cm = h_mean_prev;
                const Dual nm = Dual(1 - gs) * cm + Dual(gs) * gm;
                for (int i = 0; i < n; ++i) h[i] = dclamp_h(nm + (h[i] - cm));
            } else {
                for (int i = 0; i < n; ++i) h[i] = dclamp_h(h[i] + Dual(gs) * (gm - h[i]));
            }
        }
        /* bandwidth (:1159-1235) */
        {
            Dual sum(0), sum2(0), mn(1e10), mx(-1e10);
            for (int i = 0; i < n; ++i) {
                sum += h[i]; sum2 += h[i] * h[i];
                mn = dmin(mn, h[i]); mx = dmax(mx, h[i]);
            }
            const Dual mean = sum / Dual(n);
            const Dual var = sum2 / Dual(n) - mean * mean;
            const Dual bw2_new = dmax(Dual(2) * var / Dual(std::log((double)n + 1)), Dual(1e-6));
            Dual bw2 = bw_sq.v > 0 ? Dual(0.3) * bw2_new + Dual(0.7) * bw_sq : bw2_new;
            const double a = std::fabs(y_t);
            return_ema = return_ema > 0 ? 0.05 * a + 0.95 * return_ema : a;
            return_var = return_var > 0 ? 0.05 * a * a + 0.95 * return_var : a * a;
            const double ratio = a / std::max(return_ema, 1e-8);
            const Dual spread_f = dmin((mx - mn) * Dual(0.5), Dual(2));
            const Dual comb = dmax(Dual(ratio), spread_f);
            const Dual scale = dclamp(Dual(1) - Dual(0.25) * dmin(comb - Dual(1), Dual(2)), 0.5, 1);
            bw2 = bw2 * scale;
            bw_sq = bw2;
            bw = dclamp(dsqrt(bw2), 0.01, 2);
        }
        /* budget and beta schedule (:1057-1138) */
        const int na = c.use_annealing ? std::max(c.n_anneal_steps, 1) : 1;
        const double eps_step = 0.1 * (c.use_guide ? 0.5 : 1.0);
        int budget;
        if (t < 10) budget = c.stein_max_steps;
        else {
            float kn01 = ((float)ksd_prev - 0.05f) / (0.50f - 0.05f);
            kn01 = std::min(std::max(kn01, 0.0f), 1.0f);
            budget = c.stein_min_steps + (int)(kn01 * (float)(c.stein_max_steps - c.stein_min_steps));
        }
        if (budget < 0) budget = 0;
        const bool full = c.use_newton && c.use_full_newton;
        const double temp = c.use_svld ? c.temperature : 0.0;
        int kn = 1;
        double ksd_last = 0;
        for (int ai = 0; ai < na; ++ai) {
            double beta;
            if (!c.use_annealing) beta = 1;
            else if (c.use_adaptive_beta) beta = Tick<double>::adaptive_beta(ksd_prev, ai, na);
            else { static const double sch[3] = {0.3, 0.65, 1.0}; beta = sch[ai % 3]; }
            const double bf = std::sqrt(beta);
            int si = budget / na;
            if (ai == na - 1) si = budget - si * (na - 1);
            for (int s = 0; s < si; ++s) {
                const bool last = (ai == na - 1) && (s == si - 1);
                gradient(beta, mu_k, st, y_t);
                ksd_last = transport(eps_step * bf, temp, last, nz, kn, full, ksd_last);
                if (temp > 1e-6) ++kn;
            }
        }
        /* outputs (:1109-1153) */
        Dual mxl(-1e10);
        for (int i = 0; i < n; ++i) mxl = dmax(mxl, lw[i]);
        Dual se(0), sh(0);
        for (int i = 0; i < n; ++i) { se += dexp(lw[i] - mxl); sh += h[i]; }
        const Dual ll = mxl + dlog(dmax(se / Dual(n), Dual(1e-10)));
        h_mean_prev = sh / Dual(n);
        ksd_prev = ksd_last;
        timestep = t + 1;
        return predictive ? ll_pred : ll;
    }

    /* gradient pass, Gaussian mixture prior + Student-t likelihood (:354-521) */
    void gradient(double beta, const std::vector<Dual>& mu_k, const Dual& st, double y_t) {
        const Dual s2 = sz * sz;
        const Dual inv2 = Dual(0.5) / s2, inv = Dual(1) / s2;
        const double y2 = y_t * y_t;
        for (int j = 0; j < n; ++j) {
            const Dual hj = h[j];
            Dual lmax(-1e10);
            for (int k = 0; k < n; ++k) {
                const Dual d = hj - mu_k[k];
                lmax = dmax(lmax, -d * d * inv2);
            }
            Dual sr(0), wg(0);
            for (int k = 0; k < n; ++k) {
                const Dual d = hj - mu_k[k];
                const Dual r = dexp(-d * d * inv2 - lmax);
                sr += r;
                wg -= r * d * inv;
            }
            const Dual gp = wg / (sr + Dual(1e-8));
            const Dual A = Dual(y2) / (dsafe_exp(hj) + Dual(1e-8)) / nu;
            const Dual opA = Dual(1) + A;
            lw[j] = st - Dual(0.5) * hj - (nu + Dual(1)) * Dual(0.5) * dlog1p(dmax(A, Dual(-0.999)));
            Dual glik;
            if (c.use_exact_gradient) glik = Dual(-0.5) + Dual(0.5) * (nu + Dual(1)) * A / opA - Dual(c.lik_offset);
            else glik = (Dual(std::log(y2 + 1e-10)) - hj + Dual(c.lik_offset)) / Dual(1.4);
            g[j] = dclamp(gp + Dual(beta) * glik, -10, 10);
            if (c.use_newton) {
                const Dual hl = Dual(-0.5) * (nu + Dual(1)) * A / (opA * opA);
                curv[j] = dclamp(-(hl - inv), 0.1, 100);
            }
        }
    }

    /* vanilla or full-Newton transport with RMSProp, SVLD and clamp (Jacobi) */
    double transport(double es, double temp, bool want_ksd, Noise<double>& nz, int kn, bool full, double ksd_keep) {
        const Dual inv_bw2 = Dual(1) / (bw * bw);
        const double sign = c.stein_repulsive_sign == 1 ? 1.0 : -1.0;
        std::vector<Dual> hn(n);
        double ksd_sum = 0;
        for (int i = 0; i < n; ++i) {
            Dual ks(0), gk(0), hw(0), knn(0);
            for (int j = 0; j < n; ++j) {
                const Dual d = h[i] - h[j];
                const Dual dist2 = d * d * inv_bw2;
                const Dual K = Dual(1) / (Dual(1) + dist2);
                const Dual K2 = K * K;
                ks += K * g[j];
                gk += Dual(sign * 2) * d * inv_bw2 * K2;
                if (full) {
                    const Dual w = Dual(3) * dist2 - Dual(1);
                    hw += curv[j] * K + Dual(2) * inv_bw2 * K2 * (w.v < 0 ? -w : w);
                    knn += K;
                }
                if (want_ksd) {
                    const double dd = d.v, ib = inv_bw2.v, dd2 = dist2.v, k1 = K.v, k2 = K2.v;
                    const double gxk = -2 * dd * ib * k2;
                    const double hxy = 2 * ib * k2 * (4 * dd2 * k1 - 1);
                    ksd_sum += k1 * g[i].v * g[j].v + g[i].v * (-gxk) + g[j].v * gxk + hxy;
                }
            }
            Dual phi = (ks + gk) / Dual(n);
            if (full) {
                const Dual H = dclamp(hw / dmax(knn, Dual(1e-6)), 0.1, 100);
                phi = phi / H * Dual(0.7);
            }
            const double rr = c.rmsprop_rho;
            const Dual vn = Dual(rr) * v[i] + Dual(1 - rr) * phi * phi;
            v[i] = vn;
            const Dual drift = Dual(es) * phi / dsqrt(vn + Dual((double)c.rmsprop_eps));
            double diff = 0;
            if (temp > 1e-6) diff = std::sqrt(2 * es * temp) * nz.normal(i, kn);
            hn[i] = dclamp_h(h[i] + drift + Dual(diff));
        }
        h.swap(hn);
        if (!want_ksd) return ksd_keep;
        return std::sqrt(std::max(ksd_sum / ((double)n * (double)n), 0.0));
    }
};

}  // namespace

extern "C" {

void svpf_oracle_philox(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1,
                        uint32_t c2, uint32_t c3, uint32_t* out) {
    Block b = philox(k0, k1, c0, c1, c2, c3);
    for (int i = 0; i < 4; ++i) out[i] = b.v[i];
}

/* Defaults of svpf_create, svpf_optimized_graph.cu:116-283. */
void svpf_oracle_config_defaults(oracle_config* c, int n_stein_steps, float nu) {
    std::memset(c, 0, sizeof(*c));
    c->n_stein_steps = n_stein_steps;
    c->nu = nu;
    {
        /* svpf_optimized_graph.cu:127-138, evaluated in float like svpf_create */
        const float psi_half = -1.9635100260214235f;
        float nh = nu / 2.0f, psi;
        if (nh >= 1.0f) psi = std::log(nh) - 1.0f / (2.0f * nh) - 1.0f / (12.0f * nh * nh);
        else psi = -0.5772156649f - 1.0f / nh;
        c->student_t_implied_offset = -(std::log(nu) + psi_half - psi);
    }
    c->lik_offset = 0.45f;
    c->use_exact_gradient = 0;
    c->use_svld = 1; c->use_annealing = 1; c->use_adaptive_beta = 1; c->n_anneal_steps = 3;
    c->temperature = 1.0f; c->rmsprop_rho = 0.9f; c->rmsprop_eps = 1e-6f;
    c->use_mim = 1; c->mim_jump_prob = 0.05f; c->mim_jump_scale = 5.0f;
    c->use_asymmetric_rho = 1; c->rho_up = 0.98f; c->rho_down = 0.93f;
    c->use_guide = 1; c->use_guide_preserving = 1; c->guide_strength = 0.05f;
    c->use_adaptive_guide = 0; c->guide_strength_base = 0.05f; c->guide_strength_max = 0.30f;
    c->guide_innovation_threshold = 1.0f;
    c->use_rejuvenation = 1; c->rejuv_ksd_threshold = 0.30f; c->rejuv_prob = 0.30f; c->rejuv_blend = 0.30f;
    c->use_newton = 0; c->use_full_newton = 0;
    c->use_guided = 0; c->guided_alpha_base = 0.0f; c->guided_alpha_shock = 0.5f;
    c->guided_innovation_threshold = 1.5f;
    c->use_local_params = 0; c->delta_rho = 0.02f; c->delta_sigma = 0.1f;
    c->use_adaptive_mu = 0; c->mu_process_var = 0.001f; c->mu_obs_var_scale = 10.0f;
    c->mu_min = -6.0f; c->mu_max = -1.0f;
    c->use_adaptive_sigma = 0; c->sigma_boost_threshold = 1.0f; c->sigma_boost_max = 3.0f;
    c->stein_repulsive_sign = 0; c->use_fan_mode = 0;
    c->stein_min_steps = 4; c->stein_max_steps = 12; c->ksd_improvement_threshold = 0.05f;
    c->use_student_t_state = 0; c->nu_state = 5.0f;
    c->use_smoothing = 0; c->smooth_lag = 3; c->smooth_output_lag = 1;
    c->use_heun = 0;
    c->use_two_factor = 0;   /* :257-266 */
    c->rho_fast = 0.90f; c->sigma_fast = 0.15f; c->rho_slow = 0.99f; c->sigma_slow = 0.05f;
    c->bw_floor_fast = 0.01f; c->bw_floor_slow = 0.05f;
}

void svpf_oracle_ctl_defaults(oracle_ctl* s) {
    std::memset(s, 0, sizeof(*s));
    s->ksd_prev = 1e10f;
    s->ksd_last = 0.0f;
    s->vol_prev = 0.05f;
    s->h_mean_prev = -3.5f;   /* svpf_optimized_graph.cu:492-494 */
    s->bw_sq = 0.0f;          /* :483-484 */
    s->return_ema = 0.0f;     /* :158-165 */
    s->return_var = 0.0f;
    s->sigma_z_effective = 0.10f;
    s->mu_state = -3.5f;
    s->mu_var = 1.0f;
    for (int i = 0; i < ORACLE_SMOOTH_MAX_LAG; ++i) s->smooth_h_var[i] = 1.0f;
}

int svpf_oracle_initialize(oracle_config* cfg, const oracle_params* p, oracle_ctl* s, int n,
                           double* h, double* hp, double* v, const float* init_normals,
                           uint64_t seed, int filter_id) {
    if (n <= 0) return -1;
    s->timestep = 0;
    s->y_prev = 0.0f;
    cfg->nu_state = std::max(cfg->nu_state, 2.5f);
    float rho = p->rho, sz = p->sigma_z;
    float base_var = (sz * sz) / (1.0f - rho * rho + 1e-6f);
    float var = cfg->use_student_t_state ? cfg->nu_state / (cfg->nu_state - 2.0f) * base_var : base_var;
    double sd = std::sqrt((double)var);
    PhiloxKey key = make_key(seed, filter_id);
    for (int i = 0; i < n; ++i) {
        double z = init_normals ? (double)init_normals[i]
                                : philox_normal<double>(key, (uint32_t)i, 0u, 0u, 2u);
        double hv = std::min(std::max((double)p->mu + sd * z, -15.0), 5.0);
        h[i] = hv; hp[i] = hv; v[i] = 0.0;
    }
    s->guide_initialized = 0;
    s->guide_mean = p->mu;
    s->guide_var = var;
    if (cfg->use_two_factor) {
        /* svpf_optimized_graph.cu:414-447, svpf_init_two_factor_kernel (svpf_two_factor.cu:29-48):
         * draws 1 (fast) and 2 (slow) after the single-factor draw 0; h/hp/v are [fast; slow] */
        const float rf = cfg->rho_fast, sf = cfg->sigma_fast, rs = cfg->rho_slow, ss = cfg->sigma_slow;
        const double sdf = sf / std::sqrt((double)(1.0f - rf * rf + 1e-8f));
        const double sds = ss / std::sqrt((double)(1.0f - rs * rs + 1e-8f));
        for (int i = 0; i < n; ++i) {
            double zf = init_normals ? (double)init_normals[(size_t)n + i]
                                     : philox_normal<double>(key, (uint32_t)i, 1u, 0u, 2u);
            double zs = init_normals ? (double)init_normals[2 * (size_t)n + i]
                                     : philox_normal<double>(key, (uint32_t)i, 2u, 0u, 2u);
            h[i] = std::min(std::max(sdf * zf, -15.0), 5.0);
            h[n + i] = std::min(std::max(sds * zs, -15.0), 5.0);
            hp[i] = h[i]; hp[n + i] = h[n + i];
            v[i] = 0.0; v[n + i] = 0.0;
        }
        s->guide_2f_initialized = 0;
        s->guide_mean_fast = 0.0;
        s->guide_mean_slow = 0.0;
        s->guide_var_fast = (double)(sf * sf / (1.0f - rf * rf + 1e-6f));
        s->guide_var_slow = (double)(ss * ss / (1.0f - rs * rs + 1e-6f));
    }
    if (cfg->use_adaptive_mu) { s->mu_state = p->mu; s->mu_var = 1.0f; }
    if (cfg->use_adaptive_sigma) s->sigma_z_effective = p->sigma_z;
    s->ksd_prev = 1e10f;
    s->stein_steps_used = cfg->n_stein_steps;
    return 0;
}

int svpf_oracle_tick(const oracle_config* cfg, const oracle_params* p, oracle_ctl* ctl, int n,
                     double* h, double* hp, double* v, double* lw, float yt, float yp,
                     const oracle_noise* noise, oracle_out* out, int precision) {
    if (n <= 0 || !cfg || !p || !ctl || !noise || !out) return -1;
    if (precision == 0) return tick_impl<double>(cfg, p, ctl, n, h, hp, v, lw, yt, yp, noise, out);
    return tick_impl<float>(cfg, p, ctl, n, h, hp, v, lw, yt, yp, noise, out);
}

int svpf_oracle_batch_tick_f32(int nf, const oracle_config* cfgs, const oracle_params* ps,
                               oracle_ctl* ctls, const int* ns, int n_max,
                               float* h, float* hp, float* v, float* lw,
                               const float* yt, const float* yp, uint64_t seed, uint64_t tick,
                               int n_threads, oracle_out* outs) {
    int bad = 0;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
#endif
    for (int f = 0; f < nf; ++f) {
        int n = ns[f];
        size_t off = (size_t)f * n_max;
        Tick<float> tk(cfgs[f], ps[f], ctls[f], n);
        tk.h.assign(h + off, h + off + n); tk.hp.assign(hp + off, hp + off + n);
        tk.v.assign(v + off, v + off + n); tk.lw.assign(lw + off, lw + off + n);
        tk.g.assign(n, 0); tk.curv.assign(n, 1); tk.precond.assign(n, 0);
        oracle_noise nzs;
        std::memset(&nzs, 0, sizeof(nzs));
        nzs.mode = 1; nzs.seed = seed; nzs.tick = tick; nzs.filter_id = f;
        Noise<float> nz(&nzs, n);
        bad |= tk.run(yt[f], yp[f], nz, &outs[f]) != 0;
        for (int i = 0; i < n; ++i) {
            h[off + i] = tk.h[i]; hp[off + i] = tk.hp[i]; v[off + i] = tk.v[i]; lw[off + i] = tk.lw[i];
        }
    }
    return bad ? -3 : 0;
}

}  // extern "C"

/* ---- gradient oracle entry points ---------------------------------------- */
extern "C" {

double svpf_oracle_digamma(double x) { return digamma(x); }

/* 1 if the configuration is inside the differentiable set: single factor,
 * plain or MIM predict with the model's rho, preserving or blending EKF guide
 * with a fixed strength, Gaussian mixture prior, vanilla or full-Newton
 * transport, fixed beta schedule, no rejuvenation, no adaptive mu / sigma /
 * guide.  The Stein budget may follow the KSD: it is piecewise constant. */
int svpf_oracle_grad_supported(const oracle_config* c) {
    if (c->use_two_factor || c->use_heun || c->use_student_t_state || c->use_fan_mode) return 0;
    if (c->use_adaptive_mu || c->use_adaptive_sigma || c->use_adaptive_guide) return 0;
    if (c->use_asymmetric_rho || c->use_local_params || c->use_guided || c->use_rejuvenation) return 0;
    if (c->use_newton && !c->use_full_newton) return 0;
    if (c->stein_min_steps < 1 || c->stein_max_steps < 1) return 0;
    /* adaptive beta is a continuous function of the previous tick's KSD, which
     * the adjoint does not differentiate */
    if (c->use_annealing && c->use_adaptive_beta) return 0;
    return 1;
}

/* A whole run of one filter: initialisation from theta = (mu, rho, sigma_z,
 * nu) with the project's Philox draws keyed by (seed, filter_id), then T ticks
 * of ys (y_prev = 0 before the first).  Writes loglik[T] and
 * grad[4] = d(sum_t w_t loglik_t)/d theta (w = NULL: all ones); h_final[n]
 * optional.  Returns 0, or -2 for a configuration outside the
 * differentiable set. */
int svpf_oracle_grad_run2(const oracle_config* cfg_in, int n, int T, const double* theta, double gamma,
                          const float* ys, const double* w, uint64_t seed, int filter_id,
                          double* loglik, double* grad, double* h_final, int objective);
int svpf_oracle_grad_run3(const oracle_config* cfg_in, int n, int T, const double* theta, double gamma,
                          const float* ys, const double* w, uint64_t seed, int filter_id,
                          double* loglik, double* grad, double* h_final, int objective, int truncate_every);

int svpf_oracle_grad_run(const oracle_config* cfg_in, int n, int T, const double* theta, double gamma,
                         const float* ys, const double* w, uint64_t seed, int filter_id,
                         double* loglik, double* grad, double* h_final) {
    return svpf_oracle_grad_run2(cfg_in, n, T, theta, gamma, ys, w, seed, filter_id, loglik, grad, h_final, 0);
}

/* objective 0: the tick's log-likelihood (log-weights of its last gradient
 * pass, the reference's output); 1: the predictive log-likelihood
 * log p(y_t | y_1:t-1), averaged over the predicted particles. */
int svpf_oracle_grad_run2(const oracle_config* cfg_in, int n, int T, const double* theta, double gamma,
                          const float* ys, const double* w, uint64_t seed, int filter_id,
                          double* loglik, double* grad, double* h_final, int objective) {
    return svpf_oracle_grad_run3(cfg_in, n, T, theta, gamma, ys, w, seed, filter_id, loglik, grad, h_final,
                                 objective, 0);
}

int svpf_oracle_grad_run3(const oracle_config* cfg_in, int n, int T, const double* theta, double gamma,
                          const float* ys, const double* w, uint64_t seed, int filter_id,
                          double* loglik, double* grad, double* h_final, int objective, int truncate_every) {
    if (!svpf_oracle_grad_supported(cfg_in)) return -2;
    if (n < 1 || T < 0) return -1;
    oracle_config cfg = *cfg_in;
    cfg.nu = (float)theta[3];
    GradFilter f(cfg, n, theta, gamma);
    f.predictive = objective == 1;
    oracle_noise nzs;
    std::memset(&nzs, 0, sizeof(nzs));
    nzs.mode = 1;
    nzs.seed = seed;
    nzs.filter_id = filter_id;
    Noise<double> nz0(&nzs, n);
    f.initialize(nz0, nullptr, make_key(seed, filter_id));
    for (int k = 0; k < 4; ++k) grad[k] = 0;
    double y_prev = 0;
    for (int t = 0; t < T; ++t) {
        if (truncate_every > 0 && t > 0 && t % truncate_every == 0) f.hold_state();
        nzs.tick = (uint64_t)t;
        Noise<double> nz(&nzs, n);
        const Dual ll = f.tick((double)ys[t], y_prev, nz);
        y_prev = (double)ys[t];
        if (loglik) loglik[t] = ll.v;
        const double wt = w ? w[t] : 1.0;
        for (int k = 0; k < 4; ++k) grad[k] += wt * ll.d[k];
    }
    if (h_final)
        for (int i = 0; i < n; ++i) h_final[i] = f.h[i].v;
    return 0;
}

}  // extern "C"

/* ======================================================================== */
/* svpf_fully_fused_step_v2 restated (src/svpf_fully_fused_v2.cu:90-745).   */
/* ======================================================================== */
namespace {

template <typename R>
int v2_tick(const oracle_v2_params& P, int n, double* hd, double* hpd, double* gd, double* lwd, double* vd,
            double* ihd, float yt, float yp, float hmp, float volp, float ksdp, int timestep,
            double* gmean, double* gvar, double* mustate, const oracle_noise* noise, oracle_v2_out* out) {
    Noise<R> nz(noise, n);
    const R y_t = yt, y_prev = yp, h_mean_prev = hmp;
    const R rho = P.rho, sz = P.sigma_z, mu = P.mu, nu = P.nu;
    /* phase 0 (:190-267) */
    R eff_mu = P.use_adaptive_mu ? (R)*mustate : mu;
    R prev_gm = (R)*gmean, gv = (R)*gvar;
    if (gv < (R)1e-6) {
        prev_gm = mu;
        gv = sz * sz / (1 - rho * rho);
    }
    R boost = 1;
    if (P.use_adaptive_sigma && timestep > 0) {
        R ve = std::max((R)volp, (R)1e-4);
        R rz = std::fabs(y_t) / ve;
        if (rz > (R)P.sigma_boost_threshold) {
            R sev = std::min((rz - (R)P.sigma_boost_threshold) / 3, (R)1);
            boost = 1 + ((R)P.sigma_boost_max - 1) * sev;
        }
    }
    const R eff_sigma = sz * boost;
    R gm, gs;
    if (P.use_guide) {
        R m_pred = eff_mu + rho * (prev_gm - eff_mu);
        R P_pred = rho * rho * gv + sz * sz;
        R ly2 = std::log(y_t * y_t + (R)1e-8);
        R obs_offset = -(R)P.student_t_implied_offset;
        R S = P_pred + (R)(4.93 + 2.0);
        R K = P_pred / (S + (R)1e-8);
        R innov = ly2 - (m_pred + obs_offset);
        gm = m_pred + K * innov;
        gv = (1 - K) * P_pred;
        *gmean = (double)gm;
        *gvar = (double)gv;
        R ve = std::max((R)volp, (R)1e-4);
        R rz = std::fabs(y_t) / ve;
        if (rz > (R)P.guide_innovation_threshold) {
            R sev = std::min((rz - (R)P.guide_innovation_threshold) / 3, (R)1);
            gs = (R)P.guide_strength_base + ((R)P.guide_strength_max - (R)P.guide_strength_base) * sev;
        } else {
            gs = (R)P.guide_strength_base;
        }
    } else {
        gm = h_mean_prev;
        gv = 1;
        gs = 0;
    }
    const R inv_s2 = 1 / (eff_sigma * eff_sigma), inv_2s2 = (R)0.5 * inv_s2;
    /* phase 1: predict (:274-357) */
    std::vector<R> h(n), muk(n), zd(n), lw(n), g(n), sg(n), sh(n), v(n), ksd_i(n, 0);
    std::vector<int> kn(n, 4);
    for (int i = 0; i < n; ++i) {
        R h_old = (R)hd[i];
        muk[i] = eff_mu + rho * (h_old - eff_mu) + (R)P.gamma * y_prev / (std::exp(h_old * (R)0.5) + (R)1e-8);
        R lrho = rho, lsig = eff_sigma;
        if (P.delta_rho > 0 || P.delta_sigma > 0) {
            R dev = h_old - h_mean_prev;
            lrho = std::min(std::max(rho + (R)P.delta_rho * std::tanh(dev), (R)0), (R)0.999);
            lsig = eff_sigma * (1 + (R)P.delta_sigma * std::fabs(dev));
        }
        R lev = 0;
        if (std::fabs(P.gamma) > 1e-6f) lev = (R)P.gamma * y_prev / (std::exp(h_old * (R)0.5) + (R)1e-8);
        R prior = eff_mu + lrho * (h_old - eff_mu) + lev;
        R z_state = nz.normal(i, 0);
        zd[i] = nz.normal(i, 1);
        R jump = nz.uniform(i, 0) < (R)P.mim_jump_prob ? (R)1 : (R)0;
        R msig = lsig * (1 + jump * ((R)P.mim_jump_scale - 1));
        R hi;
        if (P.use_guided_predict) {
            R ly2 = std::log(y_t * y_t + (R)1e-10);
            R implied = std::max(ly2 + (R)P.student_t_implied_offset, (R)-5);
            R zs = (implied - prior) / (R)2.5;
            R act = zs > (R)P.guided_innovation_thresh_predict ? std::tanh(zs - (R)P.guided_innovation_thresh_predict) : (R)0;
            R alpha = (R)P.guided_alpha_base + ((R)P.guided_alpha_shock - (R)P.guided_alpha_base) * act;
            hi = (1 - alpha) * prior + alpha * implied + msig * z_state;
        } else {
            hi = prior + msig * z_state;
        }
        hpd[i] = (double)h_old;
        h[i] = clamp_h(hi);
    }
    /* phase 2: guide (:363-378) */
    if (P.use_guide && gs > 0) {
        for (int i = 0; i < n; ++i) {
            R hi = P.use_guide_preserving ? h[i] + gs * (gm - h_mean_prev) : (1 - gs) * h[i] + gs * gm;
            h[i] = clamp_h(hi);
        }
    }
    /* phase 3: Silverman bandwidth (:384-410) */
    R sum = 0;
    for (int i = 0; i < n; ++i) sum += h[i];
    const R mean = sum / (R)n;
    R ss = 0;
    for (int i = 0; i < n; ++i) ss += (h[i] - mean) * (h[i] - mean);
    const R sd = std::sqrt(std::max(ss / (R)n, (R)1e-6));
    const R bw = std::min(std::max((R)1.06 * sd * (R)std::pow((double)n, -0.2), (R)0.05), (R)2);
    const R inv_bw2 = 1 / (bw * bw);
    /* phase 4: Stein loop (:416-640) */
    for (int i = 0; i < n; ++i) v[i] = (R)vd[i];
    const int na = P.n_anneal_steps < 1 ? 1 : P.n_anneal_steps;
    const int ns = P.n_stein_steps < 1 ? 1 : P.n_stein_steps;
    const int spa = ns / na, rem = ns - spa * na;
    const R sign = P.stein_sign_mode == 1 ? (R)1 : (R)-1;
    const R hess_prior = -inv_s2;
    const R nu1 = nu + 1;
    int gstep = 0;
    for (int ai = 0; ai < na; ++ai) {
        R beta;
        if (na <= 1) beta = 1;
        else if (ai == na - 1) beta = 1;
        else beta = (R)0.3 + ((R)ai / (R)(na - 1)) * (R)0.5;
        const int si = spa + (ai == na - 1 ? rem : 0);
        for (int s = 0; s < si; ++s) {
            ++gstep;
            const bool last = gstep == ns;
            for (int i = 0; i < n; ++i) {
                const R hi = h[i];
                R lmax = (R)-1e10;
                for (int k = 0; k < n; ++k) { R d = hi - muk[k]; lmax = std::max(lmax, -d * d * inv_2s2); }
                R sr = 0, wg = 0;
                for (int k = 0; k < n; ++k) {
                    R d = hi - muk[k];
                    R r = std::exp(-d * d * inv_2s2 - lmax);
                    sr += r;
                    wg -= r * d * inv_s2;
                }
                R gp = std::min(std::max(wg / (sr + (R)1e-8), (R)-10), (R)10);
                R vol = std::exp(hi * (R)0.5);
                R A = y_t * y_t / (vol * vol + (R)1e-8) / nu;
                R opA = 1 + A;
                lw[i] = (R)P.student_t_const - (R)0.5 * hi - (R)0.5 * nu1 * std::log(opA);
                R gl = (R)-0.5 + (R)0.5 * nu1 * A / opA - (R)P.lik_offset;
                R gg = std::min(std::max(gp + beta * gl, (R)-10), (R)10);
                g[i] = gg;
                R hl = (R)-0.5 * nu1 * A / (opA * opA);
                R curv = std::min(std::max(-(hl + hess_prior), (R)0.1), (R)100);
                R invH = 1 / curv;
                if (P.use_newton || P.use_full_newton) ihd[i] = (double)curv;
                if (P.use_full_newton) { sg[i] = gg; sh[i] = curv; }
                else if (P.use_newton) { sg[i] = (R)0.7 * gg * invH; sh[i] = invH; }
                else { sg[i] = gg; sh[i] = 1; }
            }
            std::vector<R> hn(n);
            const R es = (R)P.step_size * std::sqrt(beta);
            for (int i = 0; i < n; ++i) {
                const R hi = h[i];
                R ks = 0, gk = 0, Hw = 0, Ks = 0, kq = 0;
                for (int j = 0; j < n; ++j) {
                    R diff = hi - h[j];
                    R dist2 = diff * diff * inv_bw2;
                    R K = 1 / (1 + dist2), K2 = K * K;
                    ks += K * sg[j];
                    if (P.use_newton) gk += sign * 2 * diff * inv_bw2 * K2 * sh[j];
                    else gk += sign * 2 * diff * inv_bw2 * K2;
                    if (P.use_full_newton) {
                        Hw += sh[j] * K;
                        Hw += 2 * inv_bw2 * K2 * std::fabs(3 * dist2 - 1);
                        Ks += K;
                    }
                    if (last) {
                        R raw_i = g[i];
                        R raw_j = P.use_newton ? sg[j] / ((R)0.7 * sh[j] + (R)1e-8) : sg[j];
                        R gxk = -2 * diff * inv_bw2 * K2;
                        R hxy = 2 * inv_bw2 * K2 * (4 * dist2 * K - 1);
                        kq += K * raw_i * raw_j + raw_i * (-gxk) + raw_j * gxk + hxy;
                    }
                }
                R phi;
                if (P.use_full_newton) {
                    R H = std::min(std::max(Hw / std::max(Ks, (R)1e-6), (R)0.1), (R)100);
                    phi = (ks + gk) / (R)n / H * (R)0.7;
                } else {
                    phi = (ks + gk) / (R)n;
                }
                R vn = (R)P.rmsprop_rho * v[i] + (1 - (R)P.rmsprop_rho) * phi * phi;
                v[i] = vn;
                R drift = es * phi / std::sqrt(vn + (R)P.rmsprop_eps);
                R diffu = 0;
                if (P.temperature > 1e-6f) {
                    diffu = std::sqrt(2 * es * (R)P.temperature) * zd[i];
                    zd[i] = nz.normal(i, kn[i]++);
                }
                hn[i] = clamp_h(hi + drift + diffu);
                if (last) ksd_i[i] = kq;
            }
            h.swap(hn);
        }
    }
    /* phase 5: rejuvenation (:646-658) */
    if (P.use_rejuvenation && ksdp > P.rejuv_ksd_threshold && timestep > 10) {
        for (int i = 0; i < n; ++i) {
            R u = nz.uniform(i, 1);
            if (u < (R)P.rejuv_prob) {
                R gstd = std::sqrt(std::max(gv, (R)1e-6));
                R target = gm + gstd * nz.normal(i, kn[i]++);
                h[i] = clamp_h((1 - (R)P.rejuv_blend) * h[i] + (R)P.rejuv_blend * target);
            }
        }
    }
    /* phase 6: outputs (:664-706) */
    R ks2 = 0, sh_ = 0, sv = 0, mx = (R)-1e10;
    for (int i = 0; i < n; ++i) {
        ks2 += ksd_i[i];
        sh_ += h[i];
        sv += std::exp(h[i] * (R)0.5);
        mx = std::max(mx, lw[i]);
    }
    R sw = 0;
    for (int i = 0; i < n; ++i) sw += std::exp(lw[i] - mx);
    const R hm = sh_ / (R)n;
    out->ksd = (float)std::sqrt(std::max(ks2 / (R)n / (R)n, (R)0));
    out->h_mean = (float)hm;
    out->vol = (float)(sv / (R)n);
    out->loglik = (float)(mx + std::log(std::max(sw, (R)1e-10) / (R)n));
    out->bandwidth = (float)bw;
    if (P.use_adaptive_mu && timestep > 10) {
        R mo = (R)*mustate;
        R mn = (R)P.mu_ema_alpha * hm + (1 - (R)P.mu_ema_alpha) * mo;
        *mustate = (double)std::min(std::max(mn, (R)-10), (R)0);
    }
    for (int i = 0; i < n; ++i) {
        hd[i] = (double)h[i];
        gd[i] = (double)g[i];
        lwd[i] = (double)lw[i];
        vd[i] = (double)v[i];
    }
    return nz.bad ? -3 : 0;
}

}  // namespace

extern "C" int svpf_oracle_v2_tick(const oracle_v2_params* p, int n, double* h, double* h_prev, double* grad,
                                   double* lw, double* v, double* inv_hess, float y_t, float y_prev,
                                   float h_mean_prev, float vol_prev, float ksd_prev, int timestep,
                                   double* guide_mean, double* guide_var, double* mu_state,
                                   const oracle_noise* noise, oracle_v2_out* out, int precision) {
    if (n < 1) return -1;
    if (precision == 1)
        return v2_tick<float>(*p, n, h, h_prev, grad, lw, v, inv_hess, y_t, y_prev, h_mean_prev, vol_prev,
                              ksd_prev, timestep, guide_mean, guide_var, mu_state, noise, out);
    return v2_tick<double>(*p, n, h, h_prev, grad, lw, v, inv_hess, y_t, y_prev, h_mean_prev, vol_prev,
                           ksd_prev, timestep, guide_mean, guide_var, mu_state, noise, out);
}

/* ======================================================================== */
/* The reference's differentiable torch model, SVPFParamEstimator            */
/* (py-torch/diff_svpf_torch.py:147-217), restated in FP64 with forward-mode */
/* tangents for (mu, rho, sigma_z, nu):                                      */
/*   init   h = mu + sigma_z / sqrt(1 - rho^2 + 1e-6) z               (:168-170) */
/*   tick   h_pred = mu + rho (h - mu) + sigma_z eps, eps antithetic  (:183-189) */
/*          loglik_t = logsumexp_i log t_nu(y_t; scale e^{h_pred/2}) - log N   */
/*                     (before the transport, :192-198)                       */
/*          bw = std(h_pred) + 0.1, no derivative through it          (:201)    */
/*          n_stein times: g = clamp(prior AR score + lik score, +-10),          */
/*          h += lr (K g / N + sum_j grad K / N), IMQ^(-1/2)   (:204-211, :127-145) */
/*   TBPTT  the tangents of h are cut at t % truncate_every == 0, t > 0 (:177-179) */
/* ======================================================================== */
namespace {

Dual student_t_const(const Dual& nu) {
    /* lgamma((nu+1)/2) - lgamma(nu/2) - 0.5 log(nu pi)  (:75-80) */
    return dlgamma((nu + Dual(1.0)) * Dual(0.5)) - dlgamma(nu * Dual(0.5)) - Dual(0.5) * dlog(nu * Dual(kPi));
}

}  // namespace

extern "C" int svpf_oracle_estimator_run2(int n, int n_stein, double stein_lr, int T, const float* ys,
                                          const float* tape_init, const float* tape_ticks, const double* theta,
                                          int truncate_every, const double* w, double* loglik, double* vol,
                                          double* grad, const double* bw_fixed, double* bw_out) {
    if (n < 2 || (n & 1) || n_stein < 0 || T < 0 || !ys || !tape_init || !tape_ticks || !theta) return -1;
    const Dual mu = Dual::var(theta[0], 0), rho = Dual::var(theta[1], 1), sz = Dual::var(theta[2], 2),
               nu = Dual::var(theta[3], 3);
    const Dual C = student_t_const(nu);
    const int half = n / 2;
    std::vector<Dual> h(n), hp(n), tm(n), g(n), hn(n), lp(n);
    /* :168-170 */
    const Dual hstd = sz / dsqrt(Dual(1.0) - rho * rho + Dual(1e-6));
    for (int i = 0; i < n; ++i) h[i] = mu + hstd * Dual((double)tape_init[i]);
    if (grad)
        for (int k = 0; k < 4; ++k) grad[k] = 0;
    const Dual s2e = sz * sz + Dual(1e-8);
    for (int t = 0; t < T; ++t) {
        if (truncate_every > 0 && t > 0 && t % truncate_every == 0)
            for (int i = 0; i < n; ++i) h[i] = Dual(h[i].v);   /* h.detach() */
        const float* e = tape_ticks + (size_t)t * half;
        const Dual y((double)ys[t]);
        for (int i = 0; i < n; ++i) {
            const double eps = i < half ? (double)e[i] : -(double)e[i - half];
            tm[i] = mu + rho * (h[i] - mu);
            hp[i] = mu + rho * (h[i] - mu) + sz * Dual(eps);
        }
        /* predictive log-likelihood (:192-198, _student_t_log_prob :112-119) */
        double mx = -1e300;
        for (int i = 0; i < n; ++i) {
            const Dual sc = dexp(hp[i] * Dual(0.5));
            const Dual z = y / (sc + Dual(1e-8));
            lp[i] = C - dlog(sc + Dual(1e-8)) - (nu + Dual(1.0)) * Dual(0.5) * dlog1p(z * z / nu);
            mx = std::max(mx, lp[i].v);
        }
        Dual se(0.0);
        for (int i = 0; i < n; ++i) se += dexp(lp[i] - Dual(mx));
        const Dual ll = Dual(mx) + dlog(se) - Dual(std::log((double)n));
        if (loglik) loglik[t] = ll.v;
        const double wt = w ? w[t] : 1.0;
        if (grad)
            for (int k = 0; k < 4; ++k) grad[k] += wt * ll.d[k];
        /* bandwidth of the predicted particles, detached (:201) */
        double m = 0;
        for (int i = 0; i < n; ++i) m += hp[i].v;
        m /= n;
        double var = 0;
        for (int i = 0; i < n; ++i) var += (hp[i].v - m) * (hp[i].v - m);
        const double bw = bw_fixed ? bw_fixed[t] : std::sqrt(var / n) + 0.1;
        if (bw_out) bw_out[t] = bw;
        const double b = bw * bw + 1e-8;
        h = hp;
        for (int s = 0; s < n_stein; ++s) {
            for (int i = 0; i < n; ++i) {
                /* :205-209 */
                const Dual v = dexp(h[i] * Dual(0.5));
                const Dual A = y * y / (v * v * nu + Dual(1e-8));
                const Dual gl = Dual(-0.5) + Dual(0.5) * (nu + Dual(1.0)) * A / (Dual(1.0) + A);
                const Dual gpr = -(h[i] - tm[i]) / s2e;
                g[i] = dclamp(gpr + gl, -10, 10);
            }
            /* _stein_step / _imq_kernel (:127-145) */
            for (int i = 0; i < n; ++i) {
                Dual acc(0.0), rep(0.0);
                for (int j = 0; j < n; ++j) {
                    const Dual d = h[i] - h[j];
                    const Dual base = Dual(1.0) + d * d / Dual(b);
                    const Dual sq = dsqrt(base);
                    acc += g[j] / sq;
                    rep += -d / (Dual(b) * base * sq);
                }
                hn[i] = h[i] + Dual(stein_lr) * (acc / Dual((double)n) + rep / Dual((double)n));
            }
            h.swap(hn);
        }
        if (vol) {
            double sv = 0;
            for (int i = 0; i < n; ++i) sv += std::exp(h[i].v * 0.5);
            vol[t] = sv / n;
        }
    }
    return 0;
}

extern "C" int svpf_oracle_estimator_run(int n, int n_stein, double stein_lr, int T, const float* ys,
                                         const float* tape_init, const float* tape_ticks, const double* theta,
                                         int truncate_every, const double* w, double* loglik, double* vol,
                                         double* grad) {
    return svpf_oracle_estimator_run2(n, n_stein, stein_lr, T, ys, tape_init, tape_ticks, theta, truncate_every, w,
                                      loglik, vol, grad, nullptr, nullptr);
}
