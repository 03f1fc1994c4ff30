"""The reference's two-scale composition (include/svpf_multiscale.cuh) on the
batch engine: per-scale knobs as ms_svpf_create sets them, one batch launch
per tick for all 2F filters, each instrument's output combined from its two
filters' outputs the way ms_svpf_step combines them, and -- pinned to the
reference itself -- the outputs of the reference's own ms_svpf_step
recorded tick by tick (tests/golden/ms_composition.npz, made by
tests/golden/make_ms_golden.py from the unmodified header and sources)."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import tape
from test_oracle import TOL

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


FIXTURE = os.path.join(os.path.dirname(__file__), "golden", "ms_composition.npz")


@pytest.mark.skipif(not os.path.exists(FIXTURE), reason="fixture not recorded")
def test_composition_matches_reference_ms_svpf_step(pkg):
    """Both scales of every instrument start each tick from the reference's
    recorded state (after the first tick, which starts from the engine's own
    initialisation on the recorded initial-draw tape) and draw the recorded
    tape; every output field of the composition must match the reference's
    ms_svpf_step within 1e-4 relative (integers and flags exactly)."""
    z = np.load(FIXTURE)
    fields = json.loads(str(z["fields"]))
    ctls = json.loads(str(z["ctl"]))
    F = z["params"].shape[0]
    n_max = int(z["n_max"])
    ns_slots = int(z["normal_slots"])
    seed = int(z["tape_seed"])
    L = pkg.lib()
    m = pkg.MultiScale([pkg.Params(*[float(x) for x in p]) for p in z["params"]])
    inner = L.svpf_ms_batch_inner(m._m)
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    init = np.ascontiguousarray(tape.init_normals(seed, n_max)[None, :])
    ones = np.ones((1, n_max), np.float32)
    assert L.svpf_batch_set_noise_tape(inner, fp(init), 1, fp(ones), 1) == 0
    m.init(float(z["initial_vol"]), seed=0)
    sizes = (m.config.n_particles_reactive, m.config.n_particles_inertial)
    T = z["ys"].shape[1]
    for t in range(T):
        if t > 0:
            for i in range(F):
                for s, n in enumerate(sizes):
                    c = pkg.Ctl()
                    for k, v in ctls[i][t - 1][s].items():
                        if hasattr(c, k) and not isinstance(v, list):
                            setattr(c, k, type(getattr(c, k))(v))
                    arrs = [np.ascontiguousarray(z[k][i, t - 1, s, :n]) for k in ("h", "hp", "v", "lw")]
                    assert L.svpf_batch_set_state(inner, i + s * F, C.byref(c), *[fp(a) for a in arrs]) == 0
        nrm, uni = tape.tape(seed, t, n_max, ns_slots, 2)
        assert L.svpf_batch_set_noise_tape(inner, fp(nrm), ns_slots, fp(uni), 2) == 0
        out = m.step(z["ys"][:, t])
        for i in range(F):
            for q, k in enumerate(fields):
                got, want = getattr(out[i], k), z["outs"][i, t, q]
                if isinstance(got, int):
                    assert got == int(want), (t, i, k, got, want)
                else:
                    assert abs(got - want) <= TOL * max(1.0, abs(want)), (t, i, k, got, want)
    m.close()
