"""The oracle on randomised configurations (CPU): the same knob draws the
GPU tests use (test_gpu_random_configs), run through the FP64 oracle and its
FP32 mirror from the same state and tape each tick.  Every output stays
finite; most ticks agree to FP32 rounding; the few ill-conditioned ones (the
first tick after initialisation without SVLD noise, two-factor filters
without SVLD noise) stay within 5e-3 -- the bound the GPU tests' widened
tolerances rest on."""
import numpy as np
import pytest

import oracle
import tape
from test_oracle import rel_err


@pytest.mark.parametrize("seed", [20261204, 31])
def test_oracle_fp32_mirror_on_random_configurations(pkg, seed):
    from test_gpu_random_configs import _random_config, _random_config_2f

    rng = np.random.default_rng(seed)
    F, T = 12, 12
    ns = [int(x) for x in rng.choice([1, 2, 33, 64, 100, 257], size=F)]
    cfgs = [_random_config_2f(pkg, rng) if f % 3 == 2 else _random_config(pkg, rng) for f in range(F)]
    params = [(float(rng.uniform(0.9, 0.99)), float(rng.uniform(0.08, 0.3)), float(rng.uniform(-3.0, -0.5)),
               float(rng.choice([0.0, -0.3]))) for _ in range(F)]
    n_max = max(ns)
    devs = []
    for f in range(F):
        c, n = cfgs[f], ns[f]
        tf = bool(c.use_two_factor)
        steps = c.n_stein_steps * (c.n_anneal_steps if c.use_annealing else 1) if tf else c.stein_max_steps
        slots = 6 + int(c.nu_state + 1.5) * c.use_student_t_state + 2 * steps
        init = tape.init_normals(7 + f, n_max, 3)
        o64 = oracle.OracleFilter(n, oracle.config_from_dict(c.to_dict()), oracle.OracleParams(*params[f]), 0)
        o64.initialize(init[:, :n] if tf else init[0, :n], seed=1, filter_id=f)
        yp = 0.0
        for t in range(T):
            y = float(np.exp(0.5 * params[f][2]) * rng.standard_normal())
            nrm, uni = tape.tape(100 + f, t, n, slots, 2)
            o32 = oracle.OracleFilter(n, o64.cfg, o64.params, 1)
            o32.ctl = oracle.OracleCtl.from_buffer_copy(o64.ctl)
            o32.h, o32.h_prev, o32.v, o32.log_w = o64.h.copy(), o64.h_prev.copy(), o64.v.copy(), o64.log_w.copy()
            r32 = o32.step(y, yp, nrm, uni)
            r64 = o64.step(y, yp, nrm, uni)
            for r in (r32, r64):
                assert np.isfinite([r.loglik, r.vol, r.h_mean]).all(), (f, t)
            assert np.isfinite(o64.h).all() and np.isfinite(o32.h).all(), (f, t)
            assert r32.steps_used == r64.steps_used, (f, t)
            devs.append(rel_err(o32.h, o64.h))
            yp = y
    devs = np.array(devs)
    assert np.median(devs) < 1e-5, np.median(devs)
    assert devs.max() < 5e-3, devs.max()
