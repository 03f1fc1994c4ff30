"""The oracle's restatement of svpf_fully_fused_step_v2: FP32 mirror vs FP64,
and replay of the reference's own recorded v2 calls (golden fixtures made by
make_golden.py from the reference kernel with a noise tape)."""
import json

import numpy as np
import pytest

import cases
import tape
from test_oracle import TOL, _v2_fixtures, rel_err


def v2_params(oracle_mod, d):
    import make_golden
    return make_golden.v2_params(oracle_mod, d)


def load_v2(path):
    z = np.load(path, allow_pickle=False)
    d = {k: z[k] for k in z.files}
    d["params"] = json.loads(str(z["params"]))
    return d


def state_at(oracle_mod, fx, t):
    st = oracle_mod.V2State(int(fx["n"]))
    for a in oracle_mod.V2State.ARRAYS:
        setattr(st, a, fx[a][t].astype(np.float64))
    gm, gv, ms, hmp, volp, ksdp = fx["scalars"][t]
    st.guide_mean[0], st.guide_var[0], st.mu_state[0] = gm, gv, ms
    return st, hmp, volp, ksdp


def test_v2_fixtures_present():
    import os
    names = {os.path.basename(p)[:-4] for p in _v2_fixtures()}
    assert set(cases.V2_CASES) <= names, set(cases.V2_CASES) - names


@pytest.mark.parametrize("name", sorted(cases.V2_CASES))
def test_v2_fp32_mirror_tracks_fp64(oracle_mod, name):
    case = cases.V2_CASES[name]
    p = v2_params(oracle_mod, case["p"])
    n = case["n"]
    mu, rho, sz = case["path"]
    sts = []
    for _ in range(2):
        st = oracle_mod.V2State(n)
        st.h[:] = np.clip(mu + sz / np.sqrt(1 - rho * rho) * tape.init_normals(3, n), -15, 5)
        st.mu_state[0] = mu
        sts.append(st)
    _, ys = tape.sv_path(6, mu, rho, sz, seed=4)
    yp, hmp, volp, ksdp = 0.0, mu, float(np.exp(mu / 2)), 0.1
    for t in range(4):
        nrm, uni = tape.tape(7, t, n, cases.v2_normal_slots(case), 2)
        outs = [oracle_mod.v2_tick(p, st, ys[t], yp, hmp, volp, ksdp, t, nrm, uni, precision=prec)
                for st, prec in zip(sts, (0, 1))]
        assert abs(outs[0].loglik - outs[1].loglik) < 1e-3 * max(1, abs(outs[0].loglik))
        yp, hmp, volp, ksdp = float(ys[t]), outs[0].h_mean, outs[0].vol, outs[0].ksd
        sts[1] = sts[0].copy()
    assert np.max(np.abs(sts[0].h - sts[1].h)) < 1e-3


@pytest.mark.parametrize("path", _v2_fixtures(), ids=lambda p: p.split("/")[-1][:-4])
def test_oracle_replays_reference_v2_calls(oracle_mod, path):
    """From every recorded pre-call state of the reference's v2 kernel, one
    oracle call with the same tape lands on the recorded post-call state."""
    fx = load_v2(path)
    p = oracle_mod.OracleV2Params.from_dict(fx["params"])
    n = int(fx["n"])
    T = fx["outs"].shape[0]
    y_prev = 0.0
    for t in range(T):
        st, hmp, volp, ksdp = state_at(oracle_mod, fx, t)
        nrm, uni = tape.tape(int(fx["tape_seed"]), t, n, int(fx["normal_slots"]), 2)
        out = oracle_mod.v2_tick(p, st, fx["ys"][t], y_prev, hmp, volp, ksdp, t, nrm, uni)
        y_prev = float(fx["ys"][t])
        post, _, _, _ = state_at(oracle_mod, fx, t + 1)
        for a in ("h", "h_prev", "lw"):
            assert rel_err(getattr(st, a), getattr(post, a)) < TOL, (t, a, rel_err(getattr(st, a), getattr(post, a)))
        assert rel_err(st.v, post.v, floor=1e-3) < 10 * TOL, t
        ref = fx["outs"][t]
        for k, name in enumerate(("h_mean", "vol", "loglik", "bandwidth", "ksd")):
            a, b = getattr(out, name), ref[k]
            assert abs(a - b) <= TOL * max(1.0, abs(b)), (t, name, a, b)
        for q, name in enumerate(("guide_mean", "guide_var", "mu_state")):
            assert abs(getattr(st, name)[0] - post.__dict__[name][0]) <= TOL * max(1.0, abs(post.__dict__[name][0]))
