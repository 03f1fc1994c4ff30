"""Oracle checks that need no GPU: known-answer vectors for the RNG, FP32 vs
FP64 agreement, and replay of the reference's own recorded ticks."""
import glob
import json
import os

import numpy as np
import pytest

import cases
import tape

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

# Random123 known-answer vectors for Philox4x32-10: counter, key -> output.
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


def test_philox_known_answers(oracle_mod):
    for ctr, key, out in PHILOX_KAT:
        assert oracle_mod.philox(key[0], key[1], *ctr) == list(out)


def _oracle_filter(oracle_mod, case, precision):
    cfg = oracle_mod.default_config(case["n_stein"], case["nu"])
    for k, v in case["cfg"].items():
        setattr(cfg, k, v)
    f = oracle_mod.OracleFilter(case["n"], cfg, oracle_mod.OracleParams(*case["params"]), precision)
    f.initialize(tape.init_normals(cases.TAPE_SEED, case["n"], cases.init_slots(case)))
    return f


@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_fp32_mirror_tracks_fp64(oracle_mod, name):
    case = cases.CASES[name]
    fs = [_oracle_filter(oracle_mod, case, p) for p in (0, 1)]
    _, ys = cases.observations(case, 8, seed=3)
    yp = 0.0
    for t in range(6):
        nrm, uni = tape.tape(cases.TAPE_SEED, t, case["n"], cases.normal_slots(case), 2)
        outs = [f.step(ys[t], yp, nrm, uni) for f in fs]
        yp = float(ys[t])
        assert outs[0].steps_used == outs[1].steps_used
        assert abs(outs[0].loglik - outs[1].loglik) < 1e-3 * max(1, abs(outs[0].loglik))
    d = np.max(np.abs(fs[0].h - fs[1].h))
    assert d < 1e-3, d


def _fixtures():
    """Fixtures of the svpf_step_graph path (the v2 entry point's start with
    v2_, the torch estimator model's with estimator_, the gradient check's with
    grad_, the two-scale composition's with ms_)."""
    return sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith(("v2_", "estimator_", "grad_", "ms_")))


def _v2_fixtures():
    return sorted(glob.glob(os.path.join(GOLDEN, "v2_*.npz")))


def test_fixtures_present():
    names = {os.path.basename(p)[:-4] for p in _fixtures()}
    assert set(cases.CASES) <= names, f"missing golden fixtures: {set(cases.CASES) - names}"


def load_fixture(path):
    z = np.load(path, allow_pickle=False)
    return dict(config=json.loads(str(z["config"])), params=z["params"], n=int(z["n"]), ys=z["ys"],
                normal_slots=int(z["normal_slots"]), tape_seed=int(z["tape_seed"]), h=z["h"], hp=z["hp"],
                v=z["v"], lw=z["lw"], ctl=json.loads(str(z["ctl"])), outs=z["outs"])


def rel_err(a, b, floor=1.0):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))


# Tolerance of per-tick parity with state re-sync: 1e-4 relative.
TOL = 1e-4


@pytest.mark.parametrize("path", _fixtures(), ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_replays_reference_ticks(oracle_mod, path):
    """Pin the oracle: from every recorded pre-tick state of the reference's own
    CUDA step, one oracle tick with the same tape lands on the recorded
    post-tick state (h, h_prev, RMSProp v, log-weights) and outputs."""
    fx = load_fixture(path)
    n = fx["n"]
    cfg = oracle_mod.config_from_dict(fx["config"])
    params = oracle_mod.OracleParams(*[float(x) for x in fx["params"]])
    T = fx["outs"].shape[0]
    y_prev = 0.0
    for t in range(T):
        f = oracle_mod.OracleFilter(n, cfg, params, precision=0)
        f.ctl = oracle_mod.ctl_from_dict(fx["ctl"][t])
        f.h, f.h_prev, f.v, f.log_w = (fx[k][t].astype(np.float64) for k in ("h", "hp", "v", "lw"))
        nrm, uni = tape.tape(fx["tape_seed"], t, n, fx["normal_slots"], 2)
        out = f.step(fx["ys"][t], y_prev, nrm, uni)
        y_prev = float(fx["ys"][t])
        post = fx["ctl"][t + 1]
        if not cfg.use_two_factor:   # the two-factor step leaves the step counter alone
            assert out.steps_used == post["stein_steps_used"], (t, out.steps_used, post["stein_steps_used"])
        assert rel_err(f.h, fx["h"][t + 1]) < TOL, (t, rel_err(f.h, fx["h"][t + 1]))
        assert rel_err(f.h_prev, fx["hp"][t + 1]) < TOL
        assert rel_err(f.v, fx["v"][t + 1], floor=1e-3) < TOL * 10, (t, rel_err(f.v, fx["v"][t + 1], 1e-3))
        assert rel_err(f.log_w, fx["lw"][t + 1]) < TOL, (t, rel_err(f.log_w, fx["lw"][t + 1]))
        ll, vol, hm = fx["outs"][t]
        assert abs(out.loglik - ll) < TOL * max(1, abs(ll)), (t, out.loglik, ll)
        assert abs(out.vol - vol) < TOL * max(1, abs(vol))
        assert abs(out.h_mean - hm) < TOL * max(1, abs(hm)), (t, out.h_mean, hm)
        for k in ("ksd_prev", "bw", "bw_sq", "return_ema", "return_var", "h_mean_prev", "vol_prev", "mu_state"):
            a, b = getattr(f.ctl, k), post[k]
            assert abs(a - b) <= TOL * max(1.0, abs(b)), (t, k, a, b)
        assert abs(f.ctl.guide_mean - post["guide_mean"]) < TOL * max(1, abs(post["guide_mean"]))
        assert abs(f.ctl.guide_var - post["guide_var"]) < TOL * max(1, abs(post["guide_var"]))
        if cfg.use_two_factor:
            for k in TWO_FACTOR_SCALARS:
                a, b = getattr(f.ctl, k), post[k]
                assert abs(a - b) <= TOL * max(1.0, abs(b)), (t, k, a, b)


# Two-factor control fields compared after every replayed tick.
TWO_FACTOR_SCALARS = ("h_fast_mean", "h_slow_mean", "guide_mean_fast", "guide_mean_slow", "guide_var_fast",
                      "guide_var_slow", "guide_2f_initialized", "timestep")


def ctl_mismatches(ctl, want: dict, tol: float = TOL):
    """Fields of a control record (oracle or engine) that differ from a
    recorded one: every scalar and every smoother slot the record holds."""
    bad = {}
    for k, b in want.items():
        if not hasattr(ctl, k):
            continue
        a = getattr(ctl, k)
        if isinstance(b, list):
            a = list(a)
            if any(abs(x - y) > tol * max(1.0, abs(y)) for x, y in zip(a, b)):
                bad[k] = (a, b)
        elif abs(a - b) > tol * max(1.0, abs(b)):
            bad[k] = (a, b)
    return bad


@pytest.mark.parametrize("path", _fixtures(), ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_initialize_matches_reference(oracle_mod, path):
    """svpf_initialize (svpf_optimized_graph.cu:349-451, backend quirks
    :483-494): from the fixture's initial-draw tape, the oracle lands on the
    reference's recorded post-initialise state (tick 0 of the fixture)."""
    fx = load_fixture(path)
    n = fx["n"]
    cfg = oracle_mod.config_from_dict(fx["config"])
    f = oracle_mod.OracleFilter(n, cfg, oracle_mod.OracleParams(*[float(x) for x in fx["params"]]))
    f.initialize(tape.init_normals(fx["tape_seed"], n, 3 if cfg.use_two_factor else 1))
    assert rel_err(f.h, fx["h"][0]) < TOL and rel_err(f.h_prev, fx["hp"][0]) < TOL
    assert np.array_equal(f.v, fx["v"][0]) and np.array_equal(f.log_w, fx["lw"][0])
    assert not ctl_mismatches(f.ctl, fx["ctl"][0])
