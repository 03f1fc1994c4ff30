"""The reference's two-scale composition (include/svpf_multiscale.cuh) on the
batch engine: per-scale knobs as ms_svpf_create sets them, one batch launch
per tick for all 2F filters, and each instrument's output combined from its
two filters' outputs the way ms_svpf_step combines them."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_scales_carry_the_reference_knobs(pkg):
    base = [pkg.Params(0.98, 0.10, -3.5, 0.0)] * 3
    m = pkg.MultiScale(base)
    r, i = m.inner_config(0), m.inner_config(3)
    # REACTIVE: fast scout (svpf_multiscale.cuh:212-259)
    assert (r.use_newton, r.use_annealing, r.use_guide, r.stein_min_steps, r.stein_max_steps) == (0, 0, 0, 2, 5)
    assert abs(r.mim_jump_prob - 0.30) < 1e-7 and abs(r.temperature - 0.55) < 1e-7 and r.n_stein_steps == 3
    # INERTIAL: production filter (:268-350)
    assert (i.use_newton, i.use_full_newton, i.use_guided, i.use_adaptive_mu, i.use_adaptive_sigma) == (1, 1, 1, 1, 1)
    assert (i.stein_min_steps, i.stein_max_steps, i.n_anneal_steps, i.n_stein_steps) == (8, 16, 3, 8)
    assert abs(i.nu - 5.0) < 1e-7 and abs(r.nu - 5.0) < 1e-7
    m.close()


def test_combination_follows_ms_svpf_step(pkg):
    F = 5
    base = [pkg.Params(0.98, 0.10 + 0.02 * k, -3.5 + 0.2 * k, 0.0) for k in range(F)]
    m = pkg.MultiScale(base)
    m.init(0.01, seed=4)
    rng = np.random.default_rng(0)
    vol_prev = np.full(F, 0.01)
    ema = np.zeros(F)
    for t in range(6):
        y = (0.02 * rng.standard_t(5, size=F)).astype(np.float32)
        out = m.step(y)
        inner = m.inner_outputs()
        for k in range(F):
            o, r, n = out[k], inner[k], inner[F + k]
            assert (o.vol_reactive, o.h_reactive, o.loglik_reactive) == (r.vol, r.h_mean, r.loglik)
            assert (o.vol_inertial, o.h_inertial, o.loglik_inertial) == (n.vol, n.h_mean, n.loglik)
            assert o.stein_steps_reactive == r.steps_used and o.stein_steps_inertial == n.steps_used
            # weights 0 / 1: the combined estimate is the INERTIAL one
            assert o.h_combined == n.h_mean and o.loglik_combined == n.loglik
            assert abs(o.vol_combined - n.vol) <= 1e-7 * max(1.0, n.vol)
            s = abs(float(y[k])) / max(vol_prev[k], 1e-6)
            assert abs(o.surprise_reactive - s) <= 1e-5 * max(1.0, s)
            ema[k] = 0.3 * s + 0.7 * ema[k]
            assert o.is_regime_shift == int(r.vol > 0.02 and n.vol > 0.02)
            assert o.is_calm == int(r.vol < 0.02 and n.vol < 0.02)
            assert o.cross_scale_boost == 0
            vol_prev[k] = o.vol_combined
    m.close()
