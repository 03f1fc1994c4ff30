"""svpf_fully_fused_step_v2 of the engine (through the C ABI) against the
reference's own recorded calls (golden fixtures) and against the FP64 oracle,
with state re-sync and a shared noise tape; sizes beyond the reference's
1024-particle limit; Philox mode.  Tolerance: 1e-4 relative; for the size
sweep, which starts from zero RMSProp moments, four times the oracle's own
sensitivity where that is larger (the FP32 oracle's distance from the FP64
oracle, and the FP64 result's response to a 1e-7 relative change of the
positions: 8e-3 at N = 2048 without SVLD noise)."""
import json

import numpy as np
import pytest

import cases
import tape
from test_oracle import TOL, _v2_fixtures, rel_err
from test_oracle_v2 import load_v2, state_at, v2_params

pytestmark = pytest.mark.gpu


def load_state(f, oracle_mod, st):
    for a in oracle_mod.V2State.ARRAYS:
        f.set(a, getattr(st, a))
    f.set("guide_mean", st.guide_mean[0])
    f.set("guide_var", st.guide_var[0])
    f.set("mu_state", st.mu_state[0])


def check_against(f, oracle_mod, post, out, tol=TOL):
    for a in ("h", "h_prev", "lw"):
        got = f.get(a)
        assert rel_err(got, getattr(post, a)) < tol, (a, rel_err(got, getattr(post, a)), tol)
    assert rel_err(f.get("v"), post.v, floor=1e-3) < 10 * tol
    for name in ("h_mean", "vol", "loglik", "bandwidth", "ksd"):
        a, b = f.get(name), getattr(out, name) if not isinstance(out, np.ndarray) else None
        if b is None:
            continue
        assert abs(a - b) <= tol * max(1.0, abs(b)), (name, a, b)
    for name in ("guide_mean", "guide_var", "mu_state"):
        b = getattr(post, name)[0]
        assert abs(f.get(name) - b) <= tol * max(1.0, abs(b)), (name, f.get(name), b)


@pytest.mark.parametrize("path", _v2_fixtures(), ids=lambda p: p.split("/")[-1][:-4])
def test_v2_matches_reference_calls(pkg, oracle_mod, path):
    fx = load_v2(path)
    n = int(fx["n"])
    params = fx["params"]
    f = pkg.FusedV2(n)
    y_prev = 0.0
    for t in range(fx["outs"].shape[0]):
        st, hmp, volp, ksdp = state_at(oracle_mod, fx, t)
        load_state(f, oracle_mod, st)
        nrm, uni = tape.tape(int(fx["tape_seed"]), t, n, int(fx["normal_slots"]), 2)
        f.set_tape(nrm, uni)
        rc = f.step(params, fx["ys"][t], y_prev, hmp, volp, ksdp, t)
        assert rc == 0
        assert f.rng_state().status == 0
        y_prev = float(fx["ys"][t])
        post, _, _, _ = state_at(oracle_mod, fx, t + 1)
        ref = fx["outs"][t]
        out = type("O", (), dict(zip(("h_mean", "vol", "loglik", "bandwidth", "ksd"), ref)))
        check_against(f, oracle_mod, post, out)
    f.close()


@pytest.mark.parametrize("n", [1, 2, 31, 257, 1000, 1025, 2048, 4096])
@pytest.mark.parametrize("name", ["v2_reference_test_n512", "v2_vanilla_local_n256"])
def test_v2_matches_oracle_sizes(pkg, oracle_mod, name, n):
    case = cases.V2_CASES[name]
    p = v2_params(oracle_mod, case["p"])
    params = p.to_dict()
    mu, rho, sz = case["path"]
    st = oracle_mod.V2State(n)
    st.h[:] = np.clip(mu + sz / np.sqrt(1 - rho * rho) * tape.init_normals(5, n), -15, 5).astype(np.float32)
    st.mu_state[0] = mu
    _, ys = tape.sv_path(4, mu, rho, sz, seed=n)
    f = pkg.FusedV2(n)
    yp, hmp, volp, ksdp = 0.0, mu, float(np.exp(mu / 2)), 0.1
    for t in range(3):
        load_state(f, oracle_mod, st)
        nrm, uni = tape.tape(31, t, n, cases.v2_normal_slots(case), 2)
        f.set_tape(nrm, uni)
        assert f.step(params, ys[t], yp, hmp, volp, ksdp, 12 + t) == 0
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
        st.guide_mean[0], st.guide_var[0], st.mu_state[0] = f.get("guide_mean"), f.get("guide_var"), f.get("mu_state")
        yp, hmp, volp, ksdp = float(ys[t]), out.h_mean, out.vol, out.ksd
    f.close()


def test_v2_philox_mode_and_tape_errors(pkg, oracle_mod):
    case = cases.V2_CASES["v2_reference_test_n512"]
    params = v2_params(oracle_mod, case["p"]).to_dict()
    n = 512
    h0 = np.clip(-4.5 + 0.5 * tape.init_normals(2, n), -15, 5)
    runs = []
    for _ in range(2):
        f = pkg.FusedV2(n, seed=77, filter_id=3)
        f.set("h", h0)
        f.set("mu_state", -4.5)
        for t in range(3):
            assert f.step(params, 0.01 * (t + 1), 0.0, -4.5, 0.1, 0.1, t) == 0
        assert f.rng_state().tick == 3
        runs.append(f.get("h"))
        f.close()
    assert np.array_equal(runs[0], runs[1])            # same seed, same draws
    f = pkg.FusedV2(n, seed=78, filter_id=3)
    f.set("h", h0)
    f.set("mu_state", -4.5)
    for t in range(3):
        f.step(params, 0.01 * (t + 1), 0.0, -4.5, 0.1, 0.1, t)
    assert not np.array_equal(runs[0], f.get("h"))     # another seed, other draws
    f.set_tape(np.zeros((3, n), np.float32), np.full((2, n), 0.5, np.float32))
    assert f.step(params, 0.01, 0.0, -4.5, 0.1, 0.1, 3) == 0
    assert f.rng_state().status == 4                   # SVPF_ERR_TAPE_SHORT
    assert not pkg.lib().svpf_fully_fused_v2_supported(100000)
    # the largest N whose arrays fit a 16-member cluster (227 KB per CTA)
    assert pkg.lib().svpf_fully_fused_v2_supported(8064)
    assert not pkg.lib().svpf_fully_fused_v2_supported(8065)
    f.close()
