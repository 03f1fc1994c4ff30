"""Record the reference's two-scale composition as fixtures (needs a GPU).

Drives the reference's own ms_svpf_create / ms_svpf_init / ms_svpf_step
(include/svpf_multiscale.cuh, unmodified, compiled with the reference's
sources and its curand draws routed to a noise tape: oracle/_ref/
libsvpf_ref_tape.so) for a few instruments, and stores per tick the
composition's outputs and the post-tick state of both scales' filters.  All
instruments and both scales draw from one tape of stride n_max (1024), the
layout of the batch engine's shared tape.

    python tests/golden/make_ms_golden.py [out_dir]

Output: tests/golden/ms_composition.npz
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
import tape  # noqa: E402

# The reference's MS_SVPF_Output, field by field.
MS_FIELDS = [("vol_reactive", "f"), ("vol_inertial", "f"), ("h_reactive", "f"), ("h_inertial", "f"),
             ("loglik_reactive", "f"), ("loglik_inertial", "f"), ("vol_combined", "f"), ("h_combined", "f"),
             ("loglik_combined", "f"), ("transient_magnitude", "f"), ("transient_ratio", "f"),
             ("ksd_reactive", "f"), ("ksd_inertial", "f"), ("stein_steps_reactive", "i"),
             ("stein_steps_inertial", "i"), ("surprise_reactive", "f"), ("cross_scale_boost", "i"),
             ("mim_prob_inertial_used", "f"), ("is_transient", "i"), ("is_regime_shift", "i"), ("is_calm", "i")]


class MSOut(C.Structure):
    _fields_ = [(k, C.c_float if t == "f" else C.c_int) for k, t in MS_FIELDS]


# Instruments: base parameters (the INERTIAL scale's model) and synthetic paths.
INSTRUMENTS = [dict(params=(0.98, 0.10, -3.5, 0.0), path=(-3.5, 0.98, 0.10), seed=31),
               dict(params=(0.97, 0.15, -3.0, -0.2), path=(-3.0, 0.97, 0.15), seed=32)]
TICKS = 12
N_MAX = 1024            # INERTIAL particles (REACTIVE: 256)
TAPE_SEED = 777
NORMAL_SLOTS = 2 + 16 + 7
INITIAL_VOL = 0.03


def main():
    out_dir = sys.argv[1] if len(sys.argv) > 1 else HERE
    reflib = oracle.RefLib("tape")
    L = reflib.L
    L.svpf_ref_ms_create.restype = C.c_void_p
    L.svpf_ref_ms_destroy.argtypes = [C.c_void_p]
    L.svpf_ref_ms_filter.restype = C.c_void_p
    L.svpf_ref_ms_filter.argtypes = [C.c_void_p, C.c_int]
    L.svpf_ref_ms_init.restype = C.c_int
    L.svpf_ref_ms_init.argtypes = [C.c_void_p, C.c_float, C.POINTER(oracle.OracleParams), C.POINTER(C.c_float),
                                   C.c_int]
    L.svpf_ref_ms_step.restype = C.c_int
    L.svpf_ref_ms_step.argtypes = [C.c_void_p, C.c_float, C.POINTER(oracle.OracleParams), C.POINTER(C.c_float),
                                   C.c_int, C.POINTER(C.c_float), C.c_int, C.c_int, C.POINTER(MSOut)]
    init = tape.init_normals(TAPE_SEED, N_MAX)
    rec = {"ys": [], "outs": [], "ctl": []}
    states = {k: [] for k in ("h", "hp", "v", "lw")}
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    for inst in INSTRUMENTS:
        ms = L.svpf_ref_ms_create()
        assert ms, "ms_svpf_create failed"
        p = oracle.OracleParams(*inst["params"])
        assert L.svpf_ref_ms_init(ms, INITIAL_VOL, C.byref(p), fp(init), N_MAX) == 0
        _, ys = tape.sv_path(TICKS, *inst["path"], seed=inst["seed"])
        outs, ctls = [], []
        st = {k: [] for k in states}
        for t in range(TICKS):
            nrm, uni = tape.tape(TAPE_SEED, t, N_MAX, NORMAL_SLOTS, 2)
            o = MSOut()
            flags = L.svpf_ref_ms_step(ms, float(ys[t]), C.byref(p), fp(nrm), NORMAL_SLOTS, fp(uni), 2, N_MAX,
                                       C.byref(o))
            assert flags == 0, f"tick {t}: tape flags {flags}"
            outs.append([getattr(o, k) for k, _ in MS_FIELDS])
            tick_ctl = []
            tick = {k: [] for k in states}
            for which in (0, 1):
                s = L.svpf_ref_ms_filter(ms, which)
                n = 256 if which == 0 else N_MAX
                ctl = oracle.OracleCtl()
                h, hp, v, lw = (np.zeros(n) for _ in range(4))
                assert L.svpf_ref_get_state(s, C.byref(ctl), *[a.ctypes.data_as(C.POINTER(C.c_double))
                                                               for a in (h, hp, v, lw)]) == 0
                tick_ctl.append(oracle.ctl_to_dict(ctl))
                for k, a in zip(("h", "hp", "v", "lw"), (h, hp, v, lw)):
                    pad = np.zeros(N_MAX, np.float32)
                    pad[:n] = a
                    tick[k].append(pad)
            ctls.append(tick_ctl)
            for k in states:
                st[k].append(np.stack(tick[k]))
        L.svpf_ref_ms_destroy(ms)
        rec["ys"].append(ys)
        rec["outs"].append(outs)
        rec["ctl"].append(ctls)
        for k in states:
            states[k].append(np.stack(st[k]))
    np.savez_compressed(
        os.path.join(out_dir, "ms_composition.npz"),
        fields=json.dumps([k for k, _ in MS_FIELDS]), params=np.array([i["params"] for i in INSTRUMENTS], np.float32),
        ys=np.array(rec["ys"], np.float32), outs=np.array(rec["outs"], np.float64), ctl=json.dumps(rec["ctl"]),
        tape_seed=np.int64(TAPE_SEED), normal_slots=np.int32(NORMAL_SLOTS), n_max=np.int32(N_MAX),
        initial_vol=np.float32(INITIAL_VOL),
        **{k: np.array(v, np.float32) for k, v in states.items()})   # [instrument][tick][scale][N_MAX]
    print("ms fixture: instruments", len(INSTRUMENTS), "ticks", TICKS)


if __name__ == "__main__":
    main()
