// svpf_multiscale.cu -- the reference's two-scale composition
// (include/svpf_multiscale.cuh) for many instruments on the batch engine.
//
// Instrument i owns filter i (REACTIVE, the fast scout) and filter F + i
// (INERTIAL, the production filter) of one batch; a tick steps all 2F filters
// in one launch, then combines each instrument's pair on the host exactly as
// ms_svpf_step does (:408-536): with the reference's current weights (0 / 1)
// the combined estimate is the INERTIAL one, and the pair yields the
// transient / regime-shift classification.  The reference's cross-scale boost
// is disabled in its source (:446-455) and stays off here.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "svpf.h"
#include "svpf_trace.h"

struct svpf_ms_batch {
    int F = 0;
    svpf_ms_config_t cfg;
    svpf_batch_t* batch = nullptr;
    std::vector<float> y2, yp2, ll, vol, hm;
    std::vector<svpf_out_t> outs;
    std::vector<float> y_prev, vol_prev, surprise_ema;
    float mim_base = 0.25f;
};

namespace {

// REACTIVE scale (ms_svpf_create, :212-259)
void reactive_config(svpf_config_t* f, int n_stein) {
    svpf_config_init(f, n_stein, 5.0f);
    f->use_asymmetric_rho = 1; f->rho_up = 0.94f; f->rho_down = 0.88f;
    f->use_mim = 1; f->mim_jump_prob = 0.30f; f->mim_jump_scale = 10.0f;
    f->use_guide = 0; f->use_guided = 0; f->use_adaptive_guide = 0;
    f->use_svld = 1; f->temperature = 0.55f; f->rmsprop_rho = 0.9f; f->rmsprop_eps = 1e-6f;
    f->use_annealing = 0; f->n_anneal_steps = 1;
    f->use_newton = 0; f->use_full_newton = 0;
    f->use_adaptive_mu = 0; f->use_adaptive_sigma = 0;
    f->use_local_params = 0; f->delta_rho = 0.0f; f->delta_sigma = 0.0f;
    f->use_exact_gradient = 1; f->lik_offset = 0.35f;
    f->stein_min_steps = 2; f->stein_max_steps = 5; f->ksd_improvement_threshold = 0.10f;
}

// INERTIAL scale (ms_svpf_create, :268-350)
void inertial_config(svpf_config_t* f, int n_stein) {
    svpf_config_init(f, n_stein, 5.0f);
    f->use_asymmetric_rho = 1; f->rho_up = 0.98f; f->rho_down = 0.93f;
    f->use_mim = 1; f->mim_jump_prob = 0.25f; f->mim_jump_scale = 9.0f;
    f->use_guide = 1; f->use_guide_preserving = 1; f->guide_strength = 0.05f;
    f->use_adaptive_guide = 1; f->guide_strength_base = 0.05f; f->guide_strength_max = 0.30f;
    f->guide_innovation_threshold = 1.0f;
    f->use_guided = 1; f->guided_alpha_base = 0.0f; f->guided_alpha_shock = 0.40f;
    f->guided_innovation_threshold = 1.5f;
    f->use_svld = 1; f->temperature = 0.45f; f->rmsprop_rho = 0.9f; f->rmsprop_eps = 1e-6f;
    f->use_annealing = 1; f->n_anneal_steps = 3;
    f->use_newton = 1; f->use_full_newton = 1;
    f->use_adaptive_mu = 1; f->mu_process_var = 0.001f; f->mu_obs_var_scale = 11.0f;
    f->mu_min = -4.0f; f->mu_max = -1.0f;
    f->use_adaptive_sigma = 1; f->sigma_boost_threshold = 0.95f; f->sigma_boost_max = 3.2f;
    f->use_local_params = 0; f->delta_rho = 0.0f; f->delta_sigma = 0.0f;
    f->use_exact_gradient = 1; f->lik_offset = 0.35f;
    f->stein_min_steps = 8; f->stein_max_steps = 16; f->ksd_improvement_threshold = 0.05f;
}

}  // namespace

extern "C" {

// ms_svpf_default_config (:145-169)
svpf_ms_config_t svpf_ms_default_config(void) {
    svpf_ms_config_t c;
    c.n_particles_reactive = 256;
    c.n_particles_inertial = 1024;
    c.n_stein_reactive = 3;
    c.n_stein_inertial = 8;
    c.surprise_mild_threshold = 2.0f;
    c.surprise_high_threshold = 3.5f;
    c.boost_mild_factor = 1.5f;
    c.boost_high_factor = 2.5f;
    c.weight_reactive = 0.10f;
    c.weight_inertial = 0.90f;
    return c;
}

svpf_ms_batch_t* svpf_ms_batch_create(int F, const svpf_ms_config_t* cfg_in, const SVPFParams* base,
                                      cudaStream_t stream) {
    SVPF_TRACE();
    if (F < 1 || !base) return nullptr;
    svpf_ms_batch* m = new svpf_ms_batch();
    m->F = F;
    m->cfg = cfg_in ? *cfg_in : svpf_ms_default_config();
    std::vector<int> ns(2 * (size_t)F);
    std::vector<svpf_config_t> cfgs(2 * (size_t)F);
    std::vector<SVPFParams> prms(2 * (size_t)F);
    svpf_config_t cr, ci;
    reactive_config(&cr, m->cfg.n_stein_reactive);
    inertial_config(&ci, m->cfg.n_stein_inertial);
    for (int i = 0; i < F; ++i) {
        ns[i] = m->cfg.n_particles_reactive;
        ns[F + i] = m->cfg.n_particles_inertial;
        cfgs[i] = cr;
        cfgs[F + i] = ci;
        prms[i] = base[i];
        prms[i].rho = 0.92f;     // rho_reactive, sigma_z_reactive (:222-223)
        prms[i].sigma_z = 0.18f;
        prms[F + i] = base[i];
    }
    m->batch = svpf_batch_create(2 * F, ns.data(), cfgs.data(), prms.data(), stream);
    if (!m->batch) {
        delete m;
        return nullptr;
    }
    m->y2.assign(2 * (size_t)F, 0.0f);
    m->yp2.assign(2 * (size_t)F, 0.0f);
    m->ll.assign(2 * (size_t)F, 0.0f);
    m->vol.assign(2 * (size_t)F, 0.0f);
    m->hm.assign(2 * (size_t)F, 0.0f);
    m->outs.resize(2 * (size_t)F);
    m->y_prev.assign(F, 0.0f);
    m->vol_prev.assign(F, 0.01f);
    m->surprise_ema.assign(F, 0.0f);
    return m;
}

svpf_batch_t* svpf_ms_batch_inner(svpf_ms_batch_t* m) { return m ? m->batch : nullptr; }

void svpf_ms_batch_destroy(svpf_ms_batch_t* m) {
    if (!m) return;
    svpf_batch_destroy(m->batch);
    delete m;
}

// ms_svpf_init (:383-405): both scales from the same seed.  The INERTIAL scale
// is initialised with the scale's own dynamics (rho_inertial 0.98, sigma_z_inertial
// 0.10, :269-270, :388-390) -- its stationary draw, EKF variance and effective
// sigma_z -- while its ticks use the instrument's base parameters (:468).
int svpf_ms_batch_init(svpf_ms_batch_t* m, float initial_vol, unsigned long long seed) {
    SVPF_TRACE();
    if (!m) return SVPF_ERR_INVALID_ARG;
    const int F = m->F;
    std::vector<SVPFParams> base(F);
    for (int i = 0; i < F; ++i) {
        svpf_batch_get_params(m->batch, F + i, &base[i]);
        SVPFParams pi = base[i];
        pi.rho = 0.98f;
        pi.sigma_z = 0.10f;
        svpf_batch_set_params(m->batch, F + i, &pi);
    }
    int rc = svpf_batch_initialize(m->batch, seed);
    for (int i = 0; i < F; ++i) {
        const int r = svpf_batch_set_params(m->batch, F + i, &base[i]);
        if (rc == SVPF_OK) rc = r;
    }
    std::fill(m->vol_prev.begin(), m->vol_prev.end(), initial_vol);
    std::fill(m->y_prev.begin(), m->y_prev.end(), 0.0f);
    std::fill(m->surprise_ema.begin(), m->surprise_ema.end(), 0.0f);
    return rc;
}

// ms_svpf_step (:408-536) for every instrument
int svpf_ms_batch_step(svpf_ms_batch_t* m, const float* y, svpf_ms_output_t* out) {
    SVPF_TRACE();
    if (!m || !y || !out) return SVPF_ERR_INVALID_ARG;
    const int F = m->F;
    for (int i = 0; i < F; ++i) {
        m->y2[i] = m->y2[F + i] = y[i];
        m->yp2[i] = m->yp2[F + i] = m->y_prev[i];
    }
    int rc = svpf_batch_step(m->batch, m->y2.data(), m->yp2.data(), m->ll.data(), m->vol.data(), m->hm.data());
    if (rc != SVPF_OK) return rc;
    svpf_batch_last_outputs(m->batch, m->outs.data());
    for (int i = 0; i < F; ++i) {
        const svpf_out_t& r = m->outs[i];
        const svpf_out_t& n = m->outs[F + i];
        svpf_ms_output_t& o = out[i];
        std::memset(&o, 0, sizeof(o));
        o.vol_reactive = r.vol;
        o.h_reactive = r.h_mean;
        o.loglik_reactive = r.loglik;
        o.ksd_reactive = r.ksd;
        o.stein_steps_reactive = r.steps_used;
        // a non-finite observation is refused by both scales (their states are
        // left as they were); the composition's own state is left too
        const bool ok = std::isfinite(y[i]);
        const float surprise = std::fabs(y[i]) / std::max(m->vol_prev[i], 1e-6f);
        if (ok) m->surprise_ema[i] = 0.3f * surprise + 0.7f * m->surprise_ema[i];
        o.surprise_reactive = surprise;
        o.cross_scale_boost = 0;
        o.mim_prob_inertial_used = m->mim_base;
        o.vol_inertial = n.vol;
        o.h_inertial = n.h_mean;
        o.loglik_inertial = n.loglik;
        o.ksd_inertial = n.ksd;
        o.stein_steps_inertial = n.steps_used;
        const float w_r = 0.0f, w_i = 1.0f;   // :497-498
        o.h_combined = w_r * r.h_mean + w_i * n.h_mean;
        o.vol_combined = std::pow(r.vol, w_r) * std::pow(n.vol, w_i);
        o.loglik_combined = w_r * r.loglik + w_i * n.loglik;
        o.transient_magnitude = r.vol - n.vol;
        o.transient_ratio = r.vol / std::max(n.vol, 1e-8f);
        const float vol_elevated = 0.02f, ratio_transient = 1.3f;
        o.is_transient = (r.vol > vol_elevated) && (o.transient_ratio > ratio_transient) && (n.vol < vol_elevated);
        o.is_regime_shift = (r.vol > vol_elevated) && (n.vol > vol_elevated);
        o.is_calm = (r.vol < vol_elevated) && (n.vol < vol_elevated);
        if (ok) {
            m->vol_prev[i] = o.vol_combined;
            m->y_prev[i] = y[i];
        }
    }
    return SVPF_OK;
}

}  // extern "C"
