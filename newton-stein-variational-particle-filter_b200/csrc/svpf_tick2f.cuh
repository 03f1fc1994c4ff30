// svpf_tick2f.cuh -- one two-factor SVPF tick (h = mu + h_fast + h_slow) of
// one filter on a team (CTA or cluster), both factors resident in shared
// memory from predict to outputs.
//
// Stage order and semantics follow the reference's two-factor driver
// src/svpf_optimized_graph.cu:744-897 and its kernels src/svpf_two_factor.cu;
// the EKF innovation split is include/svpf_two_factor.cuh:245-300.  The
// coordinate-wise transport is the single-factor IMQ transport
// (svpf_opt_kernels.cu:527-599) run once per factor per Stein step.
//
// Global arrays of a two-factor filter hold 2n values: fast (n) then slow (n).
#pragma once

#include "svpf_tick.cuh"

namespace svpf {

// Scalar control of a two-factor tick (one thread): the innovation-split EKF
// in FP64 and the per-factor constants.  Bandwidths come later, from the
// predicted particles.
__device__ inline void make_plan_2f(const svpf_config_t& c, const SVPFParams& p, svpf_ctl_t& s, float y_t,
                                    float y_prev, Plan& pl) {
    pl.y_t = y_t;
    pl.y_prev = y_prev;
    pl.mu_eff = p.mu;
    pl.stc = lgammaf((c.nu + 1.0f) * 0.5f) - lgammaf(c.nu * 0.5f) - 0.5f * logf(3.14159265358979f * c.nu);
    pl.off = c.student_t_implied_offset;
    pl.gs = c.guide_strength;   // the two-factor guide uses guide_strength (:799-806)
    pl.fmean[0] = s.h_fast_mean;
    pl.fmean[1] = s.h_slow_mean;
    if (c.use_guide) {
        const double rf = c.rho_fast, sf = c.sigma_fast, rs = c.rho_slow, ss = c.sigma_slow;
        double mf = s.guide_mean_fast, ms = s.guide_mean_slow;
        double vf = s.guide_var_fast, vs = s.guide_var_slow;
        if (!s.guide_2f_initialized) {
            mf = 0.0;
            ms = 0.0;
            vf = sf * sf / (1.0 - rf * rf);
            vs = ss * ss / (1.0 - rs * rs);
            s.guide_2f_initialized = 1;
        }
        const double pf = rf * mf, ps = rs * ms;
        const double Pf = rf * rf * vf + sf * sf;
        const double Ps = rs * rs * vs + ss * ss;
        const double implied = log((double)y_t * (double)y_t + 1e-8) + (double)pl.off;
        const double innov = implied - ((double)p.mu + pf + ps);
        const double S = Pf + Ps + (4.93 + 2.0);
        const double Kf = Pf / (S + 1e-8), Ks = Ps / (S + 1e-8);
        s.guide_mean_fast = pf + Kf * innov;
        s.guide_mean_slow = ps + Ks * innov;
        s.guide_var_fast = fmax((1.0 - Kf) * Pf, 1e-6);
        s.guide_var_slow = fmax((1.0 - Ks) * Ps, 1e-6);
    }
    pl.gmean2[0] = (float)s.guide_mean_fast;
    pl.gmean2[1] = (float)s.guide_mean_slow;
    // fixed schedule: beta = (a+1)/n_anneal, n_stein_steps per stage (:822-871)
    const int na = c.use_annealing ? c.n_anneal_steps : 1;
    pl.na = max(na, 0);
    pl.budget = pl.na * max(c.n_stein_steps, 0);
    pl.temp = c.use_svld ? c.temperature : 0.0f;
    for (int k = 0; k < 2; ++k) {
        pl.fac[k].eps_step = 0.5f / (float)c.n_stein_steps;
        pl.fac[k].temp = pl.temp;
    }
}

// Two-factor gradient (svpf_gradient_two_factor_kernel, svpf_two_factor.cu:166-243)
// for all n particles on every team member (O(N): no exchange needed).
__device__ inline void grad_pass_2f(const Smem2& sm, int cur, const Plan& pl, const svpf_config_t& cfg,
                                    const SVPFParams& prm, float beta, float* __restrict__ lw_out) {
    const int n = sm.f[0].n;
    const float mu = prm.mu, nu = cfg.nu;
    const float rf = cfg.rho_fast, rs = cfg.rho_slow;
    const float sf2 = cfg.sigma_fast * cfg.sigma_fast + 1e-8f;
    const float ss2 = cfg.sigma_slow * cfg.sigma_slow + 1e-8f;
    const float wf = sf2 / (sf2 + ss2), ws = 1.0f - wf;
    const float y2 = pl.y_t * pl.y_t;
    const float ly2 = logf(y2 + 1e-8f);
    const float half_np1 = 0.5f * (nu + 1.0f);
    const float* xf = sm.f[0].h[cur];
    const float* xs = sm.f[1].h[cur];
    for (int i = threadIdx.x; i < n; i += kThreads) {
        const float hf = xf[i];
        const float hs = xs[i];
        const float hc = mu + hf + hs;
        const float ratio = y2 / (nu * expf(hc) + 1e-8f);
        float lg;
        if (cfg.use_exact_gradient) lg = -0.5f + half_np1 * ratio / (1.0f + ratio + 1e-8f);
        else lg = 0.5f * (ly2 - hc);
        sm.f[0].g[i] = -(hf - rf * sm.prev[0][i]) / sf2 + beta * wf * lg;
        sm.f[1].g[i] = -(hs - rs * sm.prev[1][i]) / ss2 + beta * ws * lg;
        if (lw_out != nullptr) lw_out[i] = pl.stc - 0.5f * hc - half_np1 * logf(1.0f + ratio);
    }
}

template <int R, int S>
__device__ void run_tick_2f(const svpf_config_t& cfg, const SVPFParams& prm, svpf_ctl_t& ctl, float y_t,
                            float y_prev, const FilterIO& io, const Noise& nz, const Smem2& sm, Plan& pl,
                            const Team& team, svpf_out_t& out) {
    const int tid = threadIdx.x;
    const int n = io.n;
    const int np = sm.f[0].np;
    if (tid == 0) {
        pl.flag = 0;
        make_plan_2f(cfg, prm, ctl, y_t, y_prev, pl);
    }
    for (int i = n + tid; i < np; i += kThreads) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            sm.f[k].h[0][i] = kHPadRaw;
            sm.f[k].h[1][i] = kHPadRaw;
            sm.f[k].g[i] = 0.0f;
        }
    }
    __syncthreads();

    // ---- predict (svpf_predict_two_factor_kernel, svpf_two_factor.cu:55-90) and
    //      guide (svpf_apply_guide_two_factor_kernel, :321-362); every member
    //      does all rows.
    float st[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    {
        const float rf = cfg.rho_fast, sf = cfg.sigma_fast, rs = cfg.rho_slow, ss = cfg.sigma_slow;
        const float gs = pl.gs;
        const float cmf = pl.fmean[0], cms = pl.fmean[1];
        const float nmf = (1.0f - gs) * cmf + gs * pl.gmean2[0];
        const float nms = (1.0f - gs) * cms + gs * pl.gmean2[1];
        for (int i = tid; i < n; i += kThreads) {
            const float hf0 = io.h[i], hs0 = io.h[n + i];
            sm.prev[0][i] = hf0;
            sm.prev[1][i] = hs0;
            float zf = nz.normal(i, 0);
            const float zs = nz.normal(i, 1);
            if (cfg.use_mim) {
                const float u = nz.uniform(i, 0);
                if (u < cfg.mim_jump_prob) zf *= cfg.mim_jump_scale;
            }
            float hf = clamp_h(rf * hf0 + sf * zf);
            float hs = clamp_h(rs * hs0 + ss * zs);
            if (cfg.use_guide) {
                if (cfg.use_guide_preserving) {
                    hf = clamp_h(nmf + (hf - cmf));
                    hs = clamp_h(nms + (hs - cms));
                } else {
                    hf = clamp_h((1.0f - gs) * hf + gs * pl.gmean2[0]);
                    hs = clamp_h((1.0f - gs) * hs + gs * pl.gmean2[1]);
                }
            }
            sm.f[0].h[0][i] = hf;
            sm.f[1].h[0][i] = hs;
            st[0] += hf;
            st[1] += hf * hf;
            st[2] += hs;
            st[3] += hs * hs;
        }
    }
    {
        const int op[4] = {0, 0, 0, 0};
        block_reduce<4>(st, op, pl);
    }
    // ---- Silverman bandwidth per factor (svpf_bandwidth_two_factor_kernel, :256-318)
    if (tid == 0) {
        const float inv_n = 1.0f / (float)n;
        const float nf = powf((float)n, -0.2f);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const float mean = st[2 * k] * inv_n;
            const float var = st[2 * k + 1] * inv_n - mean * mean;
            const float sd = sqrtf(fmaxf(var, 1e-8f));
            const float bw = fmaxf(1.06f * sd * nf, k == 0 ? cfg.bw_floor_fast : cfg.bw_floor_slow);
            FactorPlan& fp = pl.fac[k];
            fp.bw = bw;
            fp.inv_bw = 1.0f / bw;
            fp.inv_bw2 = 1.0f / (bw * bw);
            fp.center = mean;
        }
    }
    __syncthreads();
    // ---- own rows' RMSProp state (positions stay in log-volatility units)
    const int row0 = sm.f[0].row0, nloc = sm.f[0].row1 - row0;
    for (int li = tid; li < nloc; li += kThreads) {
        sm.f[0].v[li] = io.v[row0 + li];
        sm.f[1].v[li] = io.v[n + row0 + li];
    }
    team.sync();

    // ---- Stein loop (:822-871): per step one O(N) gradient of both factors on
    //      every member, then both factors' transports of the member's rows,
    //      which write the next positions into every member; one team barrier.
    int cur = 0;
    int kn = 2;
    int it = 0;
    for (int a = 0; a < pl.na; ++a) {
        const float beta = (float)(a + 1) / (float)pl.na;
        for (int s = 0; s < cfg.n_stein_steps; ++s, ++it) {
            const bool last = it == pl.budget - 1;
            grad_pass_2f(sm, cur, pl, cfg, prm, beta, (last && team.rank == 0) ? io.lw : nullptr);
            __syncthreads();
            transport_pass<R, S, 0, false, kTransport>(sm.f[0], cur, pl.fac[0], cfg, beta, nz, kn, team);
            transport_pass<R, S, 0, false, kTransport>(sm.f[1], cur, pl.fac[1], cfg, beta, nz, kn + 1, team);
            team.sync();
            cur ^= 1;
            if (pl.temp > 1e-6f) kn += 2;
        }
    }

    for (int li = tid; li < nloc; li += kThreads) {
        io.v[row0 + li] = sm.f[0].v[li];
        io.v[n + row0 + li] = sm.f[1].v[li];
    }
    if (team.rank != 0) return;

    // ---- outputs (svpf_outputs_two_factor_kernel, svpf_two_factor.cu:368-470)
    const float* hf = sm.f[0].h[cur];
    const float* hs = sm.f[1].h[cur];
    float mx[1] = {-1e30f};
    for (int i = tid; i < n; i += kThreads) mx[0] = fmaxf(mx[0], io.lw[i]);
    {
        const int op[1] = {1};
        block_reduce<1>(mx, op, pl);
    }
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int i = tid; i < n; i += kThreads) {
        acc[0] += expf(io.lw[i] - mx[0]);
        acc[1] += hf[i];
        acc[2] += hs[i];
        acc[3] += expf(0.5f * (prm.mu + hf[i] + hs[i]));
    }
    {
        const int op[4] = {0, 0, 0, 0};
        block_reduce<4>(acc, op, pl);
    }
    for (int i = tid; i < n; i += kThreads) {
        io.h_prev[i] = sm.prev[0][i];
        io.h_prev[n + i] = sm.prev[1][i];
        io.h[i] = hf[i];
        io.h[n + i] = hs[i];
    }
    if (tid == 0) {
        const float inv_n = 1.0f / (float)n;
        const float ll = mx[0] + logf(fmaxf(acc[0] * inv_n, 1e-10f));
        const float mf = acc[1] * inv_n, ms = acc[2] * inv_n;
        const float hm = prm.mu + mf + ms;
        const float vol = acc[3] * inv_n;
        ctl.h_fast_mean = mf;
        ctl.h_slow_mean = ms;
        ctl.h_mean_prev = hm;
        ctl.vol_prev = vol;
        ctl.loglik_sum += (double)ll;
        ctl.timestep += 1;
        int status = pl.flag;
        if (status == SVPF_OK && !(isfinite(y_t) && isfinite(y_prev) && isfinite(ll) && isfinite(vol) && isfinite(hm)))
            status = SVPF_ERR_NONFINITE;
        ctl.status = status;
        out.loglik = ll;
        out.vol = vol;
        out.h_mean = hm;
        out.h_mean_raw = hm;
        out.bw = pl.fac[0].bw;
        out.ksd = ctl.ksd_last;
        out.steps_used = pl.budget;
        out.rejuv_fired = 0;
    }
}

}  // namespace svpf
