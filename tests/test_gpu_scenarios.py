"""The scenario and particle-count sweep on the 1-factor SV model: regime
shift, spikes, jumps, fat tails and crisis paths of 4000 ticks, each filtered
at N = 512, 1024, 2048 and 4096 by the reference's own CUDA step (unmodified
build, its own cuRAND noise) and by this engine (its own Philox noise), both
with the production configuration.  The filtered log-volatility RMSE (after
a 100-tick burn-in) must agree within 2% for every scenario and particle
count.  Per-cell results go to the results folder (reference_scenarios.json).
"""
import json
import os

import numpy as np
import pytest

import tape
from test_gpu_reference import results_dir

pytestmark = pytest.mark.gpu

T = 4000
BURN = 100
NS = (512, 1024, 2048, 4096)
N_STEIN = 8


def _reference_hmean(oracle, reflib, cfg_dict, params, ys, n, nu):
    import ctypes as C
    f = oracle.RefFilter(reflib, n, N_STEIN, nu)
    f.apply_config(oracle.config_from_dict(cfg_dict))
    p = oracle.OracleParams(*params)
    f.L.svpf_ref_initialize(f.s, C.byref(p), tape.init_normals(7, n).ctypes.data_as(C.POINTER(C.c_float)))
    hm = np.zeros(len(ys), np.float64)
    zn, un = np.zeros((1, n), np.float32), np.ones((1, n), np.float32)
    yp = 0.0
    for t in range(len(ys)):
        hm[t] = f.step(ys[t], yp, p, zn, un)[3]
        yp = float(ys[t])
    f.close()
    return hm


def _engine_hmean(pkg, cfg_dict, params, ys, n, nu, seed):
    f = pkg.SVPF(n, N_STEIN, nu)
    f.configure(**cfg_dict)
    f.initialize(*params, seed=seed)
    hm = np.zeros(len(ys), np.float64)
    yp = 0.0
    for t in range(len(ys)):
        rc, out = f.step_raw(ys[t], yp)
        assert rc == 0
        hm[t] = out.h_mean
        yp = float(ys[t])
    f.close()
    return hm


def _rmse(a, b):
    return float(np.sqrt(np.mean((a[BURN:] - b[BURN:]) ** 2)))


@pytest.mark.parametrize("scenario", tape.SCENARIOS)
def test_scenario_rmse_matches_reference(pkg, scenario):
    import oracle
    reflib = oracle.RefLib("stock")
    h, ys, (rho, sz, mu), nu = tape.scenario_path(scenario, T, seed=1)
    params = (rho, sz, mu, 0.0)
    cfg = pkg.production_config(nu, N_STEIN).to_dict()
    rows = []
    for n in NS:
        r_ref = _rmse(_reference_hmean(oracle, reflib, cfg, params, ys, n, nu), h)
        r_eng = _rmse(_engine_hmean(pkg, cfg, params, ys, n, nu, seed=n), h)
        rows.append({"n": n, "rmse_reference": r_ref, "rmse_engine": r_eng, "rel_diff": r_eng / r_ref - 1.0})
    path = os.path.join(results_dir(), "reference_scenarios.json")
    allres = {}
    if os.path.exists(path):
        with open(path) as fh:
            allres = json.load(fh)
    allres[scenario] = rows
    with open(path, "w") as fh:
        json.dump(allres, fh, indent=1)
    for r in rows:
        assert abs(r["rel_diff"]) <= 0.02, (scenario, r)
