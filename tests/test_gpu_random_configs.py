"""Randomised configurations against the FP64 oracle.

The fixture families pin the reference's knob sets one family at a time.
Here every filter of one batch draws its own combination of the knobs a
caller may set (predict: MIM, asymmetric rho, guided predict, local
parameters, Student-t state noise; guide: preserving or blending, adaptive
strength; Stein loop: vanilla / Newton / full Newton, repulsion sign, fixed
or adaptive beta, annealing stages, SVLD, Heun, exact or approximate
likelihood score, budget bounds; rejuvenation; adaptive mu and sigma; the
smoother; Fan mode) and its own particle count, including ragged ones.  The
batch is ticked through svpf_batch_graph_launch with a noise tape for 12
ticks (across t = 10, where the KSD-driven budget and rejuvenation switch
on), each tick compared with the oracle from the engine's re-synced state
(tolerances as in test_gpu_batch_parity: 1e-4 relative, KSD 1e-3, Stein
steps and rejuvenation decisions exact; where a tick is ill-conditioned in
FP32 -- the first tick after initialisation starts from zero RMSProp moments,
and without SVLD noise some knob sets amplify rounding there -- four times
the oracle's own FP32 mirror's deviation from its FP64 result on the same
state and tape).  Seeded, so a failure reproduces.
"""
import numpy as np
import pytest

from test_gpu_batch_parity import _run

pytestmark = pytest.mark.gpu


def _random_config(pkg, rng, p_fan=0.1):
    n_stein = int(rng.integers(3, 9))
    nu = float(rng.uniform(4.0, 30.0))
    c = pkg.default_config(n_stein, nu)
    b = lambda p=0.5: int(rng.random() < p)   # noqa: E731
    newton = b(0.7)
    hi = int(rng.integers(3, 9))
    kw = dict(
        use_svld=b(0.7), temperature=float(rng.uniform(0.2, 0.6)),
        use_annealing=b(0.8), n_anneal_steps=int(rng.integers(1, 5)), use_adaptive_beta=b(),
        use_mim=b(0.6), mim_jump_prob=float(rng.uniform(0.05, 0.3)), mim_jump_scale=float(rng.uniform(2.0, 9.0)),
        use_asymmetric_rho=b(), use_local_params=b(0.3), delta_rho=float(rng.uniform(0.0, 0.02)),
        delta_sigma=float(rng.uniform(0.0, 0.1)),
        use_guided=b(0.4), use_guide=b(0.7), use_guide_preserving=b(), use_adaptive_guide=b(0.3),
        use_newton=newton, use_full_newton=int(newton and rng.random() < 0.6),
        stein_repulsive_sign=b(), use_exact_gradient=b(),
        use_rejuvenation=b(0.6), rejuv_ksd_threshold=float(rng.uniform(0.02, 0.2)),
        use_adaptive_mu=b(0.3), use_adaptive_sigma=b(0.3),
        use_student_t_state=b(0.2), nu_state=float(rng.uniform(4.0, 9.0)),
        use_heun=b(0.2), use_smoothing=b(0.3), smooth_lag=int(rng.integers(2, 7)),
        smooth_output_lag=int(rng.integers(0, 2)), use_fan_mode=b(p_fan),
        stein_min_steps=int(rng.integers(1, hi + 1)), stein_max_steps=hi,
    )
    c.update(**kw)
    return c


SMALL = [1, 2, 33, 64, 100, 257, 512]
LARGE = [256, 700, 1024, 2048]


@pytest.mark.parametrize("seed,sizes,p_fan", [(20261204, SMALL, 0.1), (7, SMALL, 0.1), (99, SMALL, 0.1),
                                              (5, SMALL, 0.4), (13, LARGE, 0.1), (21, LARGE, 0.4)])
def test_random_configurations_match_oracle(pkg, oracle_mod, seed, sizes, p_fan):
    rng = np.random.default_rng(seed)
    F = 24
    ns = [int(x) for x in rng.choice(sizes, size=F)]
    cfgs = [_random_config(pkg, rng, p_fan) for _ in range(F)]
    params = [(float(rng.uniform(0.9, 0.99)), float(rng.uniform(0.08, 0.3)), float(rng.uniform(-2.0, -0.5)),
               float(rng.choice([0.0, -0.3]))) for _ in range(F)]
    T = 12
    h = np.array([p[2] for p in params], np.float32)
    ys = (np.exp(0.5 * h)[None, :] * rng.standard_normal((T, F))).astype(np.float32)
    # noise slots: predict (1 + Student-t state draws), one per Stein iteration
    # (and one per Heun corrector), rejuvenation, with margin
    nu_state = max((c.nu_state for c in cfgs if c.use_student_t_state), default=0.0)
    slots = 4 + int(nu_state + 1.5) + 2 * max(c.stein_max_steps for c in cfgs)
    _run(pkg, oracle_mod, ns, cfgs, params, ys, ticks=T, slots=slots, sensitivity=True)


@pytest.mark.parametrize("seed", [3, 11, 42])
def test_random_configurations_single_filter_match_oracle(pkg, oracle_mod, seed):
    """The same random knob sets through svpf_step_graph: the single-filter
    cluster kernels (the latency kernels, with their own tiles, the min-pass
    row maximum at N <= 1024 and the kernel compiled for the production
    configuration alone), cluster sizes from the engine's choice or forced,
    12 ticks each against the oracle from the engine's re-synced state.
    Where a tick is ill-conditioned in FP32 (the first tick after
    initialisation starts from zero RMSProp moments; without SVLD noise a
    few knob sets amplify rounding there), the tolerance is widened to four
    times the oracle's own FP32 mirror's deviation from its FP64 result on
    the same state and tape, as the size sweeps do."""
    import tape
    from test_gpu_parity import oracle_twin
    from test_oracle import TOL, rel_err

    rng = np.random.default_rng(seed)
    for k in range(6):
        cfg = _random_config(pkg, rng)
        n = int(rng.choice([1, 2, 33, 100, 257, 512, 1000]))
        clusters = [0] + [c for c in (1, 2, 4, 8, 16) if 32 * c <= n]
        cluster = int(rng.choice(clusters))
        params = (float(rng.uniform(0.9, 0.99)), float(rng.uniform(0.08, 0.3)), float(rng.uniform(-2.0, -0.5)),
                  float(rng.choice([0.0, -0.3])))
        slots = 4 + int(cfg.nu_state + 1.5) * cfg.use_student_t_state + 2 * cfg.stein_max_steps
        f = pkg.SVPF(n, cfg.n_stein_steps, cfg.nu)
        f.configure(**cfg.to_dict())
        if cluster:
            f.set_cluster_size(cluster)
        f.initialize(*params, seed=seed + k)
        yp = 0.0
        for t in range(12):
            y = float(np.exp(0.5 * params[2]) * rng.standard_normal())
            o = oracle_twin(oracle_mod, pkg, f, params)
            o32 = oracle_mod.OracleFilter(n, o.cfg, oracle_mod.OracleParams(*params), 1)   # FP32 mirror
            o32.ctl = oracle_mod.OracleCtl.from_buffer_copy(o.ctl)
            o32.h, o32.h_prev, o32.v, o32.log_w = o.h.copy(), o.h_prev.copy(), o.v.copy(), o.log_w.copy()
            nrm, uni = tape.tape(1000 * seed + k, t, n, slots, 2)
            f.set_noise_tape(nrm, uni)
            rc, out = f.step_raw(y, yp)
            oo = o.step(y, yp, nrm, uni)
            o32o = o32.step(y, yp, nrm, uni)
            tag = (k, t, n, cluster)
            assert rc == 0, tag
            assert out.steps_used == oo.steps_used and out.rejuv_fired == oo.rejuv_fired, tag
            tol = max(TOL, 4 * rel_err(o32.h, o.h))
            assert rel_err(f.get_particles(), o.h) < tol, (tag, rel_err(f.get_particles(), o.h), tol)
            for name in ("loglik", "vol", "h_mean"):
                a, b, c = getattr(out, name), getattr(oo, name), getattr(o32o, name)
                tol = max(TOL, 4 * abs(c - b) / max(1.0, abs(b)))
                assert abs(a - b) < tol * max(1.0, abs(b)), (tag, name, a, b, tol)
            assert abs(out.ksd - oo.ksd) < 1e-3 * max(1.0, abs(oo.ksd)), (tag, out.ksd, oo.ksd)
            yp = y
        f.close()


def _random_config_2f(pkg, rng):
    n_stein = int(rng.integers(2, 9))
    c = pkg.default_config(n_stein, float(rng.uniform(4.0, 30.0)))
    b = lambda p=0.5: int(rng.random() < p)   # noqa: E731
    c.update(use_two_factor=1, rho_fast=float(rng.uniform(0.7, 0.95)), sigma_fast=float(rng.uniform(0.1, 0.35)),
             rho_slow=float(rng.uniform(0.98, 0.998)), sigma_slow=float(rng.uniform(0.03, 0.08)),
             bw_floor_fast=0.01, bw_floor_slow=0.05, use_svld=b(0.7), temperature=float(rng.uniform(0.2, 0.6)),
             use_annealing=b(0.8), n_anneal_steps=int(rng.integers(1, 5)), use_mim=b(0.6),
             mim_jump_prob=float(rng.uniform(0.05, 0.3)), mim_jump_scale=float(rng.uniform(2.0, 9.0)),
             use_guide=b(0.7), use_guide_preserving=b(), guide_strength=float(rng.uniform(0.05, 0.3)),
             use_exact_gradient=b(), lik_offset=float(rng.uniform(0.2, 0.4)), stein_repulsive_sign=b())
    return c


@pytest.mark.parametrize("seed", [31, 57])
def test_random_two_factor_configurations_match_oracle(pkg, oracle_mod, seed):
    """Two-factor filters (h = mu + h_fast + h_slow) with random factor
    dynamics, annealing, SVLD, MIM, guide and score knobs, mixed with
    single-factor filters in one batch (two persistent launches per tick),
    12 graph-replayed ticks against the oracle, as above."""
    rng = np.random.default_rng(seed)
    F = 24
    ns = [int(x) for x in rng.choice(SMALL, size=F)]
    cfgs = [_random_config_2f(pkg, rng) if f % 3 else _random_config(pkg, rng) for f in range(F)]
    params = [(float(rng.uniform(0.9, 0.99)), float(rng.uniform(0.08, 0.3)), float(rng.uniform(-4.0, -2.0)),
               0.0) for _ in range(F)]
    T = 12
    h = np.array([p[2] for p in params], np.float32)
    ys = (np.exp(0.5 * h)[None, :] * rng.standard_normal((T, F))).astype(np.float32)
    nu_state = max((c.nu_state for c in cfgs if c.use_student_t_state and not c.use_two_factor), default=0.0)
    steps_2f = max((c.n_stein_steps * (c.n_anneal_steps if c.use_annealing else 1) for c in cfgs
                    if c.use_two_factor), default=0)
    steps_1f = max((c.stein_max_steps for c in cfgs if not c.use_two_factor), default=0)
    slots = 4 + max(int(nu_state + 1.5) + 2 * steps_1f, 2 * steps_2f)
    _run(pkg, oracle_mod, ns, cfgs, params, ys, ticks=T, slots=slots, sensitivity=True)


def _random_v2(rng):
    import cases
    b = lambda p=0.5: int(rng.random() < p)   # noqa: E731
    mu, rho, sz = float(rng.uniform(-4.5, -0.5)), float(rng.uniform(0.9, 0.99)), float(rng.uniform(0.08, 0.3))
    newton = b(0.7)
    p = dict(cases.V2_REFERENCE_TEST, mu=mu, rho=rho, sigma_z=sz, nu=float(rng.uniform(4.0, 30.0)),
             gamma=float(rng.choice([0.0, -0.3])), delta_rho=float(rng.uniform(0.0, 0.02)) * b(0.3),
             delta_sigma=float(rng.uniform(0.0, 0.1)) * b(0.3), mim_jump_prob=float(rng.uniform(0.0, 0.3)),
             mim_jump_scale=float(rng.uniform(2.0, 9.0)), use_guide=b(0.7), use_guided_predict=b(0.5),
             use_guide_preserving=b(), use_newton=newton, use_full_newton=int(rng.random() < 0.5),
             use_rejuvenation=b(0.6), rejuv_ksd_threshold=float(rng.uniform(0.0, 0.1)),
             use_adaptive_mu=b(0.3), mu_ema_alpha=float(rng.uniform(0.01, 0.1)), use_adaptive_sigma=b(0.5),
             step_size=float(rng.uniform(0.05, 0.3)), temperature=float(rng.uniform(0.2, 1.0)) * b(0.7),
             n_stein_steps=int(rng.integers(1, 9)), n_anneal_steps=int(rng.integers(1, 5)),
             stein_sign_mode=b())
    return p, (mu, rho, sz)


@pytest.mark.parametrize("seed", [2, 17])
def test_random_v2_configurations_match_oracle(pkg, oracle_mod, seed):
    """svpf_fully_fused_step_v2 (the reference's second entry point) with
    random knobs and sizes, 4 ticks each from the engine's re-synced state
    against the oracle's restatement of its kernel; the tolerance is widened
    to four times the oracle's own sensitivity where that is larger (its FP32
    mirror, and its response to a 1e-7 relative change of the positions), as
    the v2 size sweep does."""
    import tape
    from test_gpu_v2 import check_against, load_state
    from test_oracle import TOL, rel_err
    from test_oracle_v2 import v2_params

    rng = np.random.default_rng(seed)
    for k in range(6):
        praw, (mu, rho, sz) = _random_v2(rng)
        n = int(rng.choice([1, 31, 100, 257, 512, 1000]))
        p = v2_params(oracle_mod, praw)
        params = p.to_dict()
        slots = 4 + max(praw["n_stein_steps"], 1) + 1
        st = oracle_mod.V2State(n)
        st.h[:] = np.clip(mu + sz / np.sqrt(1 - rho * rho) * tape.init_normals(5 + k, n), -15, 5).astype(np.float32)
        st.mu_state[0] = mu
        _, ys = tape.sv_path(5, mu, rho, sz, seed=100 * seed + k)
        f = pkg.FusedV2(n)
        yp, hmp, volp, ksdp = 0.0, mu, float(np.exp(mu / 2)), 0.1
        for t in range(4):
            load_state(f, oracle_mod, st)
            nrm, uni = tape.tape(1000 * seed + k, t, n, slots, 2)
            f.set_tape(nrm, uni)
            assert f.step(params, ys[t], yp, hmp, volp, ksdp, 12 + t) == 0, (k, t)
            s32, spert = st.copy(), st.copy()
            spert.h = spert.h * (1 + 1e-7 * np.random.default_rng(t).standard_normal(n))
            out = oracle_mod.v2_tick(p, st, ys[t], yp, hmp, volp, ksdp, 12 + t, nrm, uni)
            oracle_mod.v2_tick(p, s32, ys[t], yp, hmp, volp, ksdp, 12 + t, nrm, uni, precision=1)
            oracle_mod.v2_tick(p, spert, ys[t], yp, hmp, volp, ksdp, 12 + t, nrm, uni)
            sens = max(rel_err(s32.h, st.h), rel_err(spert.h, st.h), rel_err(s32.lw, st.lw), rel_err(spert.lw, st.lw))
            check_against(f, oracle_mod, st, out, tol=max(TOL, 4 * sens))
            st = oracle_mod.V2State(n)
            for a in oracle_mod.V2State.ARRAYS:
                setattr(st, a, f.get(a).astype(np.float64))
            st.guide_mean[0], st.guide_var[0] = f.get("guide_mean"), f.get("guide_var")
            st.mu_state[0] = f.get("mu_state")
            yp, hmp, volp, ksdp = float(ys[t]), out.h_mean, out.vol, out.ksd
        f.close()


def _random_grad_config(pkg, rng):
    """A random member of the differentiable configuration set."""
    b = lambda p=0.5: int(rng.random() < p)   # noqa: E731
    n_stein = int(rng.integers(1, 9))
    c = pkg.grad_config(n_stein, 12.0, full_newton=bool(b(0.6)))
    c.update(use_mim=b(0.6), mim_jump_prob=float(rng.uniform(0.05, 0.3)), mim_jump_scale=float(rng.uniform(2.0, 9.0)),
             use_guide=b(0.7), use_guide_preserving=b(), guide_strength=float(rng.uniform(0.02, 0.3)),
             use_exact_gradient=b(), lik_offset=float(rng.uniform(0.2, 0.4)), use_svld=b(0.7),
             temperature=float(rng.uniform(0.2, 0.6)), use_annealing=b(0.8), n_anneal_steps=int(rng.integers(1, 5)),
             stein_repulsive_sign=b())
    return c


@pytest.mark.parametrize("seed", [4, 9])
def test_random_differentiable_configurations_match_oracle(pkg, oracle_mod, seed):
    """The adjoint engine on random members of its differentiable set (predict
    with or without MIM, guide preserving or blending, exact or approximate
    score, vanilla or full-Newton transport, SVLD, annealing stages, budget,
    repulsion sign), both objectives, with or without truncation, random
    checkpoint intervals: per-tick log-likelihoods and gradients against the
    FP64 forward-mode oracle, tolerances as in test_gpu_grad."""
    from test_gpu_grad import check_against_oracle

    rng = np.random.default_rng(seed)
    for _ in range(3):
        cfg = _random_grad_config(pkg, rng)
        assert pkg.lib().svpf_grad_supported(cfg)
        # a single particle sits at the bandwidth floor (1/bw = 100), where the
        # adjoint's 1/bw^2 terms cancel in FP32 to ~3e-4 of the gradient: N = 1
        # is checked by test_gpu_grad's size sweep on its own configuration
        ns = [int(x) for x in rng.choice([2, 33, 100, 257], size=3)]
        T = int(rng.integers(6, 13))
        check_against_oracle(pkg, oracle_mod, cfg, ns, T=T, k=int(rng.integers(1, 9)), seed=int(rng.integers(1, 99)),
                             objective=int(rng.integers(0, 2)), trunc=int(rng.choice([0, 0, 4])))


@pytest.mark.parametrize("seed", [6, 23])
def test_random_estimator_configurations_match_oracle(pkg, seed):
    """The reference's torch estimator model as its CUDA engine, with random
    particle counts, Stein steps and step sizes, truncation and checkpoint
    intervals, tick weights and theta, against the FP64 oracle restatement
    (tolerances as in test_gpu_estimator)."""
    import oracle
    from test_gpu_estimator import G_TOL, LL_TOL, _random_case, sensitivity

    rng = np.random.default_rng(seed)
    for _ in range(3):
        n = int(rng.choice([2, 8, 64, 130, 512]))
        S = int(rng.integers(0, 5))
        lr = float(rng.uniform(0.05, 0.3))
        T = int(rng.integers(8, 25))
        trunc = int(rng.choice([0, 0, 3, 7]))
        k = int(rng.integers(1, 9))
        F = 3
        thetas = np.stack([rng.uniform(-4, -2, F), rng.uniform(0.85, 0.98, F), rng.uniform(0.1, 0.3, F),
                           rng.uniform(5, 20, F)], 1)
        cases = [_random_case(n, T, int(rng.integers(1, 1 << 30))) for _ in range(F)]
        w = rng.uniform(-1, 1, (F, T))
        e = pkg.Estimator(F, n, S, lr, T_max=T, checkpoint_every=k, truncate_every=trunc)
        tape = np.stack([pkg.Estimator.make_tape(c[1], c[2]) for c in cases])
        ll, vol, _ = e.forward(thetas, np.stack([c[0] for c in cases]), tape=tape)
        g = e.backward(w.astype(np.float32))
        e.close()
        for f in range(F):
            ys, ti, tt = cases[f]
            oll, ovol, og = oracle.estimator_run(n, S, lr, thetas[f], ys, ti, tt, trunc, w[f])
            sl, sv, sg = sensitivity(n, S, lr, thetas[f], ys, ti, tt, trunc, w[f])
            tag = (n, S, lr, T, trunc, k, f)
            assert np.max(np.abs(ll[f] - oll) / np.maximum(1.0, np.abs(oll))) < max(LL_TOL, 4 * sl), tag
            assert np.max(np.abs(vol[f] - ovol) / ovol) < max(LL_TOL, 4 * sv), tag
            err = np.abs(g[f] - og) / np.maximum(np.abs(og), 1e-3)
            assert np.all(err < max(G_TOL, 4 * sg)), (tag, g[f], og, err, sg)
