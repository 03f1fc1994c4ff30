// svpf_tick.cuh -- one complete SVPF tick of one filter on a team (CTA or
// cluster), particles resident in shared memory from predict to outputs.
//
// Stage order and semantics follow the reference driver
// src/svpf_optimized_graph.cu:915-1389; each stage cites its kernel.
#pragma once

#include "svpf_device.cuh"

namespace svpf {

// Global-memory arrays of one filter.
struct FilterIO {
    float* h;       // [n] positions (read at start, written at end)
    float* h_prev;  // [n] positions of the previous tick
    float* v;       // [n] RMSProp second moment
    float* lw;      // [n] log-weights of the last gradient pass
    int n;
};

template <int R, int S, int KIND, bool KSD, int MODE, int U = 0>
__device__ __forceinline__ float stein_rows(const Smem& sm, int cur, const Plan& pl,
                                            const svpf_config_t& cfg, float bf, const Noise& nz,
                                            int kn, const Team& team, float* phi_out,
                                            const float* pre = nullptr) {
    return transport_pass<R, S, KIND, KSD, MODE, Plan, U>(sm, cur, pl, cfg, bf, nz, kn, team, phi_out, pre);
}

template <int R, int S, int MODE>
__device__ float stein_dispatch(int kind, bool ksd, const Smem& sm, int cur, const Plan& pl,
                                const svpf_config_t& cfg, float bf, const Noise& nz, int kn,
                                const Team& team, float* phi_out = nullptr, const float* pre = nullptr) {
    if (kind == 2) {
        return ksd ? stein_rows<R, S, 2, true, MODE>(sm, cur, pl, cfg, bf, nz, kn, team, phi_out, pre)
                   : stein_rows<R, S, 2, false, MODE>(sm, cur, pl, cfg, bf, nz, kn, team, phi_out, pre);
    } else if (kind == 1) {
        return ksd ? stein_rows<R, S, 1, true, MODE>(sm, cur, pl, cfg, bf, nz, kn, team, phi_out, pre)
                   : stein_rows<R, S, 1, false, MODE>(sm, cur, pl, cfg, bf, nz, kn, team, phi_out, pre);
    }
    return ksd ? stein_rows<R, S, 0, true, MODE>(sm, cur, pl, cfg, bf, nz, kn, team, phi_out, pre)
               : stein_rows<R, S, 0, false, MODE>(sm, cur, pl, cfg, bf, nz, kn, team, phi_out, pre);
}

template <int R, int S, bool SCAN>
__device__ __forceinline__ void grad_dispatch(bool student, const Smem& sm, int cur, const Plan& pl,
                                              const svpf_config_t& cfg, float beta, float* lw,
                                              const Team& team) {
    if (student) grad_pass<R, S, true, SCAN>(sm, cur, pl, cfg, beta, lw, team);
    else grad_pass<R, S, false, SCAN>(sm, cur, pl, cfg, beta, lw, team);
}

// KSD of the last iteration: block sum, then member partials into rank 0.
__device__ __forceinline__ void ksd_publish(float ksd_thread, Plan& pl, const Team& team) {
    float v[1] = {ksd_thread};
    const int op[1] = {0};
    block_reduce<1>(v, op, pl);
    if (threadIdx.x == 0) team.at(pl.ksd_slot, 0)[team.rank] = v[0];
}

// A non-finite observation is refused: the tick leaves the filter's state as
// it was (particles, moments, control record, log-likelihood sum, timestep)
// and reports SVPF_ERR_NONFINITE with NaN outputs.  The reference runs such a
// tick: its fminf/fmaxf clamps pin the particles to a bound and the EKF and
// bandwidth EMAs carry the NaN, so its later ticks report finite nonsense.
// The kernels call it before the tick; every member of a team sees the same
// y_t, so all members skip the tick together.
__device__ __forceinline__ bool refuse_nonfinite(float y_t, svpf_ctl_t& ctl, svpf_out_t& out) {
    if (isfinite(y_t)) return false;
    if (threadIdx.x == 0) {
        const float qnan = __int_as_float(0x7fc00000);
        ctl.status = SVPF_ERR_NONFINITE;
        out.loglik = out.vol = out.h_mean = out.h_mean_raw = qnan;
        out.bw = ctl.bw;
        out.ksd = ctl.ksd_last;
        out.steps_used = 0;
        out.rejuv_fired = 0;
    }
    return true;
}

// A non-finite previous observation is read as 0 (no leverage): the kernels
// pass the returned value to the tick and then flag the tick's status.
__device__ __forceinline__ float readable_y_prev(float y_prev) { return isfinite(y_prev) ? y_prev : 0.0f; }
__device__ __forceinline__ void flag_y_prev(float y_prev, svpf_ctl_t& ctl) {
    if (threadIdx.x == 0 && !isfinite(y_prev) && ctl.status == SVPF_OK) ctl.status = SVPF_ERR_NONFINITE;
}

// The tick.  cfg/prm/ctl are shared-memory copies owned by the caller; only
// thread 0 of rank 0 mutates ctl after make_plan.  Returns on every member; the
// caller stores ctl/out from rank 0 thread 0.  SCAN: the mixture's row
// maximum comes from a min pass over the unsorted prior means instead of the
// means sorted once per tick (the single-filter latency kernel).  PROD: the
// caller guarantees full-Newton transport, Gaussian state noise and no Heun
// step (the production configuration), so only those code paths are compiled
// and the kernel body stays small (instruction fetch bounds the latency kernel).
template <int R, int S, bool SCAN = false, bool PROD = false, int U = 0>
__device__ void run_tick(const svpf_config_t& cfg, const SVPFParams& prm, svpf_ctl_t& ctl, float y_t,
                         float y_prev, const FilterIO& io, const Noise& nz, const Smem& sm, Plan& pl,
                         const Team& team, svpf_out_t& out) {
    const int tid = threadIdx.x;
    const int n = sm.n;
    if (tid == 0) {
        pl.flag = 0;
        make_plan(cfg, prm, ctl, y_t, y_prev, pl);
        if (cfg.use_heun) pl.transport = (cfg.use_newton && cfg.use_full_newton) ? 2 : 0;
    }
    // pads: particle columns [n, np) and prior slots [n, m_len)
    for (int i = n + tid; i < sm.np; i += kThreads) {
        sm.h[0][i] = kHPad; sm.h[1][i] = kHPad; sm.g[i] = 0.0f; sm.c[i] = 0.0f;
    }
    for (int i = n + tid; i < sm.m_len; i += kThreads) sm.mu[i] = kMuPad;
    __syncthreads();

    // ---- predict (svpf_opt_kernels.cu:125-276), guide (:282-327), prior means
    //      (:384-392); every team member does all N rows, no exchange needed.
    float st[4] = {0.0f, 0.0f, 1e10f, -1e10f};
    {
        const float hbar = ctl.h_mean_prev;
        const bool mim = cfg.use_mim || cfg.use_guided;
        const float gmean = pl.guide_mean;
        const float gsn = pl.gs;
        const float nm_pres = (1.0f - gsn) * hbar + gsn * gmean;
        const float ly2 = logf(y_t * y_t + 1e-10f);
        const float mimp = fmaxf(ly2 + pl.off, -5.0f);
        for (int i = tid; i < n; i += kThreads) {
            const float hi = io.h[i];
            const float hpi = io.h_prev[i];
            float z;
            if (cfg.use_student_t_state && cfg.nu_state <= 30.0f) {
                const float z0 = nz.normal(i, 0);
                const int nu_int = max((int)(cfg.nu_state + 0.5f), 3);
                float chi2 = 0.0f;
                for (int m = 0; m < nu_int; ++m) { const float u = nz.normal(i, 1 + m); chi2 += u * u; }
                z = z0 * sqrtf((float)nu_int / (chi2 + 1e-8f));
            } else {
                z = nz.normal(i, 0);
            }
            const float lev = prm.gamma * y_prev / (expf(fminf(hi * 0.5f, 20.0f)) + 1e-8f);
            float hp;
            if (mim) {
                const float dev = hi - hbar;
                const float rho_adj = pl.drho * tanhf(dev);
                const float sscale = 1.0f + pl.dsig * fabsf(dev);
                const float sel = nz.uniform(i, 0);
                const float scale = sel < cfg.mim_jump_prob ? cfg.mim_jump_scale : 1.0f;
                const float br = hi > hpi ? pl.rho_up : pl.rho_dn;
                const float rho = clampf(br + rho_adj, 0.0f, 0.999f);
                float mp = pl.mu_eff + rho * (hi - pl.mu_eff) + lev;
                if (cfg.use_guided) {
                    const float zz = (mimp - mp) / 2.5f;
                    const float act = zz > cfg.guided_innovation_threshold
                                          ? tanhf(zz - cfg.guided_innovation_threshold) : 0.0f;
                    const float ga = cfg.guided_alpha_base + (cfg.guided_alpha_shock - cfg.guided_alpha_base) * act;
                    mp = (1.0f - ga) * mp + ga * mimp;
                }
                hp = clamp_h(mp + pl.sz_eff * sscale * scale * z);
            } else {
                hp = clamp_h(pl.mu_eff + prm.rho * (hi - pl.mu_eff) + pl.sz_eff * z + lev);
            }
            if (cfg.use_guide) {
                hp = cfg.use_guide_preserving ? clamp_h(nm_pres + (hp - hbar)) : clamp_h(hp + gsn * (gmean - hp));
            }
            sm.h[0][i] = hp;
            sm.mu[i] = pl.mu_eff + prm.rho * (hi - pl.mu_eff) + prm.gamma * y_prev / (expf(hi * 0.5f) + 1e-8f);
            st[0] += hp;
            st[1] += hp * hp;
            st[2] = fminf(st[2], hp);
            st[3] = fmaxf(st[3], hp);
        }
    }
    {
        const int op[4] = {0, 0, 2, 1};
        block_reduce<4>(st, op, pl);
    }
    // ---- bandwidth (svpf_fused_bandwidth_kernel, svpf_opt_kernels.cu:1159-1235)
    if (tid == 0) {
        const float inv_n = 1.0f / (float)n;
        const float mean = st[0] * inv_n;
        const float var = st[1] * inv_n - mean * mean;
        const float spread = st[3] - st[2];
        const float bw2_new = fmaxf(2.0f * var / logf((float)n + 1.0f), 1e-6f);
        float bw2 = ctl.bw_sq > 0.0f ? 0.3f * bw2_new + 0.7f * ctl.bw_sq : bw2_new;
        const float a = fabsf(y_t);
        float ema = ctl.return_ema, rv = ctl.return_var;
        ema = ema > 0.0f ? 0.05f * a + 0.95f * ema : a;
        rv = rv > 0.0f ? 0.05f * a * a + 0.95f * rv : a * a;
        ctl.return_ema = ema;
        ctl.return_var = rv;
        const float ratio = a / fmaxf(ema, 1e-8f);
        const float comb = fmaxf(ratio, fminf(spread * 0.5f, 2.0f));
        const float scale = clampf(1.0f - 0.25f * fminf(comb - 1.0f, 2.0f), 0.5f, 1.0f);
        bw2 *= scale;
        const float bw = clampf(sqrtf(bw2), 0.01f, 2.0f);
        ctl.bw_sq = bw2;
        ctl.bw = bw;
        pl.bw = bw;
        pl.inv_bw = 1.0f / bw;
        pl.inv_bw2 = 1.0f / (bw * bw);
        pl.center = mean;
        pl.mu_center = pl.mu_eff;
        pl.prior_scale = sqrtf(kLog2e * 0.5f / (pl.sz_eff * pl.sz_eff));
    }
    // ---- sort prior means once per tick (used for the per-row maximum)
    if constexpr (!SCAN) bitonic_sort(sm.mu, sm.p2);
    else __syncthreads();   // plan scalars of thread 0 visible to all
    // ---- Stein-loop coordinates: positions (h - center) / bw, Gaussian prior
    //      means (mu - mu_center) * prior_scale (order preserving)
    const bool student = PROD ? false : cfg.use_student_t_state != 0;
    if (pl.budget > 0) {
        for (int i = tid; i < n; i += kThreads) {
            sm.h[0][i] = (sm.h[0][i] - pl.center) * pl.inv_bw;
            if (!student) sm.mu[i] = (sm.mu[i] - pl.mu_center) * pl.prior_scale;
        }
    }
    // ---- own rows' RMSProp state
    for (int li = tid; li < sm.row1 - sm.row0; li += kThreads) sm.v[li] = io.v[sm.row0 + li];
    // ---- SVLD normals of own rows for the first Stein iterations, drawn in
    //      parallel (same draws, in the same slots, as the per-row epilogue takes)
    if (sm.pre != nullptr && pl.temp > 1e-6f && (PROD || !cfg.use_heun)) {
        const int nloc = sm.row1 - sm.row0;
        const int iters = min(pl.budget, kPreIters);
        for (int k = tid; k < iters * nloc; k += kThreads) {
            const int it = k / nloc, li = k - it * nloc;
            sm.pre[it * sm.Lp + li] = nz.normal(sm.row0 + li, pl.kn_pred + it);
        }
    }
    team.sync();   // every member has read io.h / io.h_prev; smem ready

    // ---- annealed Stein loop (svpf_optimized_graph.cu:1120-1317)
    int cur = 0;
    int kn = pl.kn_pred;
    const int budget = pl.budget;
    for (int it = 0; it < budget; ++it) {
        const int ai = stage_of(pl, it);
        const float beta = pl.beta[ai];
        const float bf = sqrtf(beta);
        const bool last = it == budget - 1;
        if (PROD || !cfg.use_heun) {
            const float* pre = (sm.pre != nullptr && it < kPreIters) ? sm.pre + it * sm.Lp : nullptr;
            float kt;
            if constexpr (PROD) {
                grad_pass<R, S, false, SCAN, U>(sm, cur, pl, cfg, beta, io.lw, team);
                team.sync();
                kt = last ? stein_rows<R, S, 2, true, kTransport, U>(sm, cur, pl, cfg, bf, nz, kn, team, nullptr, pre)
                          : stein_rows<R, S, 2, false, kTransport, U>(sm, cur, pl, cfg, bf, nz, kn, team, nullptr, pre);
            } else {
                grad_dispatch<R, S, SCAN>(student, sm, cur, pl, cfg, beta, io.lw, team);
                team.sync();
                kt = stein_dispatch<R, S, kTransport>(pl.transport, last, sm, cur, pl, cfg, bf, nz, kn, team,
                                                      nullptr, pre);
            }
            if (last) ksd_publish(kt, pl, team);
            team.sync();
            cur ^= 1;
        } else if constexpr (!PROD) {
            // Heun predictor-corrector (svpf_optimized_graph.cu:1147-1232,
            // kernels svpf_opt_kernels.cu:1293-1566)
            const int nloc = sm.row1 - sm.row0;
            const float es = pl.eps_step * bf;
            grad_dispatch<R, S, SCAN>(student, sm, cur, pl, cfg, beta, io.lw, team);
            team.sync();
            stein_dispatch<R, S, kPhiOnly>(pl.transport, false, sm, cur, pl, cfg, bf, nz, kn, team, sm.phi0);
            __syncthreads();
            for (int li = tid; li < nloc; li += kThreads) {
                const int i = sm.row0 + li;
                const float h0 = fmaf(sm.h[cur][i], pl.bw, pl.center);
                const float hpred = clamp_h(h0 + es * sm.phi0[li] * rsqrtf(sm.v[li] + cfg.rmsprop_eps));
                const float hs = (hpred - pl.center) * pl.inv_bw;
                for (int rk = 0; rk < team.size; ++rk) team.at(sm.h[cur ^ 1], rk)[i] = hs;
            }
            team.sync();
            grad_dispatch<R, S, SCAN>(student, sm, cur ^ 1, pl, cfg, beta, io.lw, team);
            team.sync();
            stein_dispatch<R, S, kPhiOnly>(pl.transport, false, sm, cur ^ 1, pl, cfg, bf, nz, kn, team, sm.phi1);
            if (last) {
                // KSD at the start point with the gradient at the predicted point
                const float kt = stein_dispatch<R, S, kKsdOnly>(0, true, sm, cur, pl, cfg, bf, nz, kn, team);
                ksd_publish(kt, pl, team);
            }
            team.sync();   // all members done reading the predicted positions
            for (int li = tid; li < nloc; li += kThreads) {
                const int i = sm.row0 + li;
                const float pa = 0.5f * (sm.phi0[li] + sm.phi1[li]);
                const float vn = cfg.rmsprop_rho * sm.v[li] + (1.0f - cfg.rmsprop_rho) * pa * pa;
                sm.v[li] = vn;
                float diff = 0.0f;
                if (pl.temp > 1e-6f) diff = sqrtf(2.0f * es * pl.temp) * nz.normal(i, kn);
                const float h0 = fmaf(sm.h[cur][i], pl.bw, pl.center);
                const float hn = clamp_h(h0 + es * pa * rsqrtf(vn + cfg.rmsprop_eps) + diff);
                const float hs = (hn - pl.center) * pl.inv_bw;
                for (int rk = 0; rk < team.size; ++rk) team.at(sm.h[cur ^ 1], rk)[i] = hs;
            }
            team.sync();
            cur ^= 1;
        }
        if (pl.temp > 1e-6f) ++kn;
    }

    // own rows' RMSProp state back to global memory
    for (int li = tid; li < sm.row1 - sm.row0; li += kThreads) io.v[sm.row0 + li] = sm.v[li];
    if (team.rank != 0) return;

    if (tid == 0) {
        if (budget > 0) {
            float acc = 0.0f;
            for (int r = 0; r < team.size; ++r) acc += pl.ksd_slot[r];
            const float k2 = acc / ((float)n * (float)n);
            ctl.ksd_last = sqrtf(fmaxf(k2, 0.0f));
        }
        ctl.stein_steps_used = budget;
    }

    // ---- back to log-volatility coordinates
    float* hf = sm.h[cur];
    if (budget > 0) {
        for (int i = tid; i < n; i += kThreads) hf[i] = fmaf(hf[i], pl.bw, pl.center);
        __syncthreads();
    }
    // ---- partial rejuvenation (svpf_opt_kernels.cu:1248-1275)
    if (pl.rejuv) {
        const int ku = pl.uses_uniform_predict;
        const float b = cfg.rejuv_blend;
        for (int i = tid; i < n; i += kThreads) {
            const float u = nz.uniform(i, ku);
            if (u < cfg.rejuv_prob) {
                const float zz = nz.normal(i, kn);
                hf[i] = clamp_h((1.0f - b) * hf[i] + b * (pl.guide_mean + pl.gstd * zz));
            }
        }
    }
    __syncthreads();

    // ---- outputs (svpf_fused_outputs_kernel, svpf_opt_kernels.cu:1109-1153)
    float mx[1] = {-1e10f};
    for (int i = tid; i < n; i += kThreads) mx[0] = fmaxf(mx[0], io.lw[i]);
    {
        const int op[1] = {1};
        block_reduce<1>(mx, op, pl);
    }
    float acc[3] = {0.0f, 0.0f, 0.0f};
    for (int i = tid; i < n; i += kThreads) {
        acc[0] += ex2_approx((io.lw[i] - mx[0]) * kLog2e);
        acc[1] += expf(fminf(hf[i] * 0.5f, 20.0f));
        acc[2] += hf[i];
    }
    {
        const int op[3] = {0, 0, 0};
        block_reduce<3>(acc, op, pl);
    }
    // write back positions: h_prev <- positions at tick start, h <- final
    for (int i = tid; i < n; i += kThreads) {
        io.h_prev[i] = io.h[i];
        io.h[i] = hf[i];
    }
    if (tid == 0) {
        const float inv_n = 1.0f / (float)n;
        const float ll = mx[0] + logf(fmaxf(acc[0] * inv_n, 1e-10f));
        const float vol = acc[1] * inv_n;
        const float hm = acc[2] * inv_n;
        ctl.h_mean_prev = hm;
        // host tail (svpf_optimized_graph.cu:1361-1388): smoother, outputs, adaptive mu
        float hm_out = hm;
        const float bwl = ctl.bw;
        if (cfg.use_smoothing) {
            // svpf_smooth_backward (:658-717)
            const int k = min(max(cfg.smooth_lag, 1), SVPF_SMOOTH_MAX_LAG);
            const int head = ctl.smooth_head;
            ctl.smooth_h_mean[head] = hm;
            ctl.smooth_h_var[head] = bwl * bwl;
            ctl.smooth_y[head] = y_t;
            ctl.smooth_head = (head + 1) % k;
            if (ctl.timestep >= k) {
                const float rho = prm.rho;
                const float mu = cfg.use_adaptive_mu ? ctl.mu_state : prm.mu;
                const float q = prm.sigma_z * prm.sigma_z;
                for (int lag = 1; lag < k; ++lag) {
                    const int ic = (ctl.smooth_head - lag - 1 + k) % k;
                    const int inx = (ctl.smooth_head - lag + k) % k;
                    const float hc = ctl.smooth_h_mean[ic], hn = ctl.smooth_h_mean[inx];
                    const float vc = ctl.smooth_h_var[ic];
                    const float pv = rho * rho * vc + q;
                    const float J = rho * vc / (pv + 1e-8f);
                    ctl.smooth_h_mean[ic] = hc + J * (hn - (mu + rho * (hc - mu)));
                    ctl.smooth_h_var[ic] = vc * (1.0f - J * rho);
                }
            }
            // svpf_get_smoothed_output (:720-737)
            const int k2 = min(cfg.smooth_lag, SVPF_SMOOTH_MAX_LAG);
            if (k2 >= 1 && ctl.timestep >= k2 && cfg.smooth_output_lag > 0) {
                const int ol = min(cfg.smooth_output_lag, k2 - 1);
                hm_out = ctl.smooth_h_mean[(ctl.smooth_head - ol - 1 + k2) % k2];
            }
        }
        ctl.vol_prev = vol;
        ctl.ksd_prev = ctl.ksd_last;
        if (cfg.use_adaptive_mu && ctl.timestep > 10) {
            // svpf_adaptive_mu_update (:619-642)
            const float mp = ctl.mu_state, Pp = ctl.mu_var + cfg.mu_process_var;
            const float Rm = cfg.mu_obs_var_scale * bwl * bwl;
            const float K = Pp / (Pp + Rm + 1e-8f);
            ctl.mu_state = clampf(mp + K * (hm - mp), cfg.mu_min, cfg.mu_max);
            ctl.mu_var = (1.0f - K) * Pp;
        }
        ctl.loglik_sum += (double)ll;
        ctl.timestep += 1;
        // The reference's clamps (fmaxf/fminf) turn a NaN observation into finite
        // particles; the tick runs the same way here and the status reports it.
        int status = pl.flag;
        if (status == SVPF_OK && !(isfinite(y_t) && isfinite(y_prev) && isfinite(ll) && isfinite(vol) && isfinite(hm)))
            status = SVPF_ERR_NONFINITE;
        ctl.status = status;
        out.loglik = ll;
        out.vol = vol;
        out.h_mean = hm_out;
        out.h_mean_raw = hm;
        out.bw = bwl;
        out.ksd = ctl.ksd_last;
        out.steps_used = budget;
        out.rejuv_fired = pl.rejuv;
    }
}

}  // namespace svpf
