"""Generate the golden fixtures from the reference's own CUDA step (needs a GPU).

For every case in cases.py this drives the reference's svpf_step_graph (built
in place with its curand draws routed to a noise tape, oracle/_ref/
libsvpf_ref_tape.so) free-running for ``ticks`` ticks and records, per tick,
the full filter state before and after the tick plus the step outputs.

    python tests/golden/make_golden.py [out_dir [case ...]]

The fixtures are committed under tests/golden/*.npz.
"""
from __future__ import annotations

import json
import os
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import cases  # noqa: E402
import oracle  # noqa: E402
import tape  # noqa: E402


def run_case(name, case, reflib):
    n = case["n"]
    f = oracle.RefFilter(reflib, n, case["n_stein"], case["nu"])
    cfg = f.read_config()
    for k, v in case["cfg"].items():
        setattr(cfg, k, v)
    f.apply_config(cfg)
    params = oracle.OracleParams(*case["params"])
    rc = f.initialize(params, tape.init_normals(cases.TAPE_SEED, n, cases.init_slots(case)))
    assert rc == 0, f"init tape flags {rc}"
    # nu_state is clamped by svpf_initialize; read the effective config back
    cfg = f.read_config()
    _, ys = cases.observations(case, case["ticks"] + 1, seed=zlib.crc32(name.encode()) % 1000)
    ns = cases.normal_slots(case)
    rec = {k: [] for k in ("h", "hp", "v", "lw")}
    ctls, outs = [], []
    ctl, h, hp, v, lw = f.get_state()
    for arr, key in ((h, "h"), (hp, "hp"), (v, "v"), (lw, "lw")):
        rec[key].append(arr.astype(np.float32))
    ctls.append(oracle.ctl_to_dict(ctl))
    y_prev = 0.0
    for t in range(case["ticks"]):
        nrm, uni = tape.tape(cases.TAPE_SEED, t, n, ns, 2)
        flags, ll, vol, hm = f.step(ys[t], y_prev, params, nrm, uni)
        assert flags == 0, f"{name} tick {t}: tape flags {flags}"
        ctl, h, hp, v, lw = f.get_state()
        for arr, key in ((h, "h"), (hp, "hp"), (v, "v"), (lw, "lw")):
            rec[key].append(arr.astype(np.float32))
        ctls.append(oracle.ctl_to_dict(ctl))
        outs.append([ll, vol, hm])
        y_prev = float(ys[t])
    f.close()
    return dict(
        config=json.dumps(oracle.config_to_dict(cfg)),
        params=np.array(case["params"], np.float32),
        n=np.int32(n),
        ys=ys,
        normal_slots=np.int32(ns),
        tape_seed=np.int64(cases.TAPE_SEED),
        h=np.stack(rec["h"]), hp=np.stack(rec["hp"]), v=np.stack(rec["v"]), lw=np.stack(rec["lw"]),
        ctl=json.dumps(ctls),
        outs=np.array(outs, np.float32),
    )


def v2_params(oracle, d):
    """Scalar arguments of one v2 case, with nu's Student-t constants computed
    the way the reference test computes them (in FP32)."""
    import math
    p = oracle.OracleV2Params.from_dict(d)
    nu = np.float32(d["nu"])
    p.student_t_const = float(np.float32(math.lgamma((nu + 1) / 2)) - np.float32(math.lgamma(nu / 2)) -
                              np.float32(0.5) * np.float32(math.log(np.float32(3.14159) * nu)))
    cfg = oracle.default_config(8, float(nu))
    p.student_t_implied_offset = cfg.student_t_implied_offset
    return p


def run_v2_case(name, case, reflib):
    n = case["n"]
    p = v2_params(oracle, case["p"])
    st = oracle.V2State(n)
    mu, rho, sz = case["path"]
    z = tape.init_normals(cases.TAPE_SEED, n)
    st.h[:] = np.clip(mu + sz / np.sqrt(1 - rho * rho) * z.astype(np.float64), -15, 5).astype(np.float32)
    st.h_prev[:] = st.h
    st.mu_state[0] = mu
    _, ys = tape.sv_path(case["ticks"] + 1, mu, rho, sz, seed=zlib.crc32(name.encode()) % 1000)
    ns = cases.v2_normal_slots(case)
    keys = oracle.V2State.ARRAYS
    rec = {k: [] for k in keys}
    scal = []
    outs = []
    h_mean_prev, vol_prev, ksd_prev, y_prev = mu, float(np.exp(mu / 2)), 0.1, 0.0

    def snap():
        for k in keys:
            rec[k].append(getattr(st, k).astype(np.float32))
        scal.append([st.guide_mean[0], st.guide_var[0], st.mu_state[0], h_mean_prev, vol_prev, ksd_prev])

    snap()
    for t in range(case["ticks"]):
        nrm, uni = tape.tape(cases.TAPE_SEED, t, n, ns, 2)
        flags, out = oracle.ref_v2_step(reflib, p, st, ys[t], y_prev, h_mean_prev, vol_prev, ksd_prev, t, nrm, uni)
        assert flags == 0, f"{name} tick {t}: tape flags {flags}"
        h_mean_prev, vol_prev, ksd_prev, y_prev = out.h_mean, out.vol, out.ksd, float(ys[t])
        snap()
        outs.append([out.h_mean, out.vol, out.loglik, out.bandwidth, out.ksd])
    return dict(
        kind=np.array("v2"), params=json.dumps(p.to_dict()), n=np.int32(n), ys=ys, normal_slots=np.int32(ns),
        tape_seed=np.int64(cases.TAPE_SEED), scalars=np.array(scal, np.float64), outs=np.array(outs, np.float32),
        **{k: np.stack(rec[k]) for k in keys})


def main():
    out_dir = sys.argv[1] if len(sys.argv) > 1 else HERE
    only = set(sys.argv[2:])
    os.makedirs(out_dir, exist_ok=True)
    reflib = oracle.RefLib("tape")
    for name, case in cases.CASES.items():
        if only and name not in only:
            continue
        d = run_case(name, case, reflib)
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **d)
        print(f"{name}: ticks={case['ticks']} n={case['n']} loglik[0]={d['outs'][0, 0]:.5f} "
              f"hmean[-1]={d['outs'][-1, 2]:.5f}")
    for name, case in cases.V2_CASES.items():
        if only and name not in only:
            continue
        d = run_v2_case(name, case, reflib)
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **d)
        print(f"{name}: ticks={case['ticks']} n={case['n']} loglik[0]={d['outs'][0, 2]:.5f} "
              f"ksd[-1]={d['outs'][-1, 4]:.5f}")


if __name__ == "__main__":
    main()
