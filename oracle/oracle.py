"""Oracle bindings -- TEST INFRASTRUCTURE ONLY.

ctypes access to
  * ``liboracle_svpf.so``: the CPU restatement of one SVPF tick (FP64 oracle,
    FP32 CPU baseline), built from ``svpf_oracle.cpp``;
  * ``_ref/libsvpf_ref_tape.so`` / ``_ref/libsvpf_ref_stock.so``: the
    reference's own CUDA step compiled in place (see ``Makefile``), driven
    through ``ref_harness.cu``.

Only ``tests/``, the smoke check and the CPU-baseline leg of ``bench.py`` use
this module.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SMOOTH_MAX_LAG = 8

CONFIG_FIELDS = [
    ("n_stein_steps", C.c_int), ("nu", C.c_float), ("student_t_implied_offset", C.c_float),
    ("lik_offset", C.c_float), ("use_exact_gradient", C.c_int), ("use_svld", C.c_int),
    ("use_annealing", C.c_int), ("use_adaptive_beta", C.c_int), ("n_anneal_steps", C.c_int),
    ("temperature", C.c_float), ("rmsprop_rho", C.c_float), ("rmsprop_eps", C.c_float),
    ("use_mim", C.c_int), ("mim_jump_prob", C.c_float), ("mim_jump_scale", C.c_float),
    ("use_local_params", C.c_int), ("delta_rho", C.c_float), ("delta_sigma", C.c_float),
    ("use_asymmetric_rho", C.c_int), ("rho_up", C.c_float), ("rho_down", C.c_float),
    ("use_newton", C.c_int), ("use_full_newton", C.c_int), ("use_guided", C.c_int),
    ("guided_alpha_base", C.c_float), ("guided_alpha_shock", C.c_float),
    ("guided_innovation_threshold", C.c_float), ("use_rejuvenation", C.c_int),
    ("rejuv_ksd_threshold", C.c_float), ("rejuv_prob", C.c_float), ("rejuv_blend", C.c_float),
    ("use_guide", C.c_int), ("use_guide_preserving", C.c_int), ("guide_strength", C.c_float),
    ("use_adaptive_guide", C.c_int), ("guide_strength_base", C.c_float),
    ("guide_strength_max", C.c_float), ("guide_innovation_threshold", C.c_float),
    ("use_adaptive_mu", C.c_int), ("mu_process_var", C.c_float), ("mu_obs_var_scale", C.c_float),
    ("mu_min", C.c_float), ("mu_max", C.c_float), ("use_adaptive_sigma", C.c_int),
    ("sigma_boost_threshold", C.c_float), ("sigma_boost_max", C.c_float),
    ("stein_repulsive_sign", C.c_int), ("use_fan_mode", C.c_int), ("stein_min_steps", C.c_int),
    ("stein_max_steps", C.c_int), ("ksd_improvement_threshold", C.c_float),
    ("use_student_t_state", C.c_int), ("nu_state", C.c_float), ("use_smoothing", C.c_int),
    ("smooth_lag", C.c_int), ("smooth_output_lag", C.c_int), ("use_heun", C.c_int),
    ("use_two_factor", C.c_int), ("rho_fast", C.c_float), ("sigma_fast", C.c_float), ("rho_slow", C.c_float),
    ("sigma_slow", C.c_float), ("bw_floor_fast", C.c_float), ("bw_floor_slow", C.c_float),
]


class OracleConfig(C.Structure):
    _fields_ = CONFIG_FIELDS


class OracleParams(C.Structure):
    _fields_ = [("rho", C.c_float), ("sigma_z", C.c_float), ("mu", C.c_float), ("gamma", C.c_float)]


class OracleCtl(C.Structure):
    _fields_ = [
        ("guide_mean", C.c_double), ("guide_var", C.c_double), ("guide_K", C.c_double),
        ("loglik_sum", C.c_double), ("guide_mean_fast", C.c_double), ("guide_mean_slow", C.c_double),
        ("guide_var_fast", C.c_double), ("guide_var_slow", C.c_double), ("timestep", C.c_int),
        ("guide_initialized", C.c_int), ("stein_steps_used", C.c_int), ("smooth_head", C.c_int),
        ("guide_2f_initialized", C.c_int), ("ksd_prev", C.c_float),
        ("ksd_last", C.c_float), ("vol_prev", C.c_float), ("h_mean_prev", C.c_float),
        ("bw", C.c_float), ("bw_sq", C.c_float), ("return_ema", C.c_float),
        ("return_var", C.c_float), ("sigma_z_effective", C.c_float), ("mu_state", C.c_float),
        ("mu_var", C.c_float), ("y_prev", C.c_float), ("h_fast_mean", C.c_float), ("h_slow_mean", C.c_float),
        ("smooth_h_mean", C.c_float * SMOOTH_MAX_LAG), ("smooth_h_var", C.c_float * SMOOTH_MAX_LAG),
        ("smooth_y", C.c_float * SMOOTH_MAX_LAG), ("status", C.c_int), ("reserved", C.c_int),
    ]


class OracleOut(C.Structure):
    _fields_ = [("loglik", C.c_float), ("vol", C.c_float), ("h_mean", C.c_float),
                ("h_mean_raw", C.c_float), ("bw", C.c_float), ("ksd", C.c_float),
                ("steps_used", C.c_int), ("rejuv_fired", C.c_int)]


class OracleNoise(C.Structure):
    _fields_ = [("mode", C.c_int), ("n_normal_slots", C.c_int), ("n_uniform_slots", C.c_int),
                ("filter_id", C.c_int), ("normals", C.POINTER(C.c_float)),
                ("uniforms", C.POINTER(C.c_float)), ("seed", C.c_uint64), ("tick", C.c_uint64)]


CTL_SCALARS = [f for f, _ in OracleCtl._fields_ if f not in ("smooth_h_mean", "smooth_h_var", "smooth_y")]


def ctl_to_dict(c) -> dict:
    d = {f: getattr(c, f) for f in CTL_SCALARS}
    for f in ("smooth_h_mean", "smooth_h_var", "smooth_y"):
        d[f] = list(getattr(c, f))
    return d


def ctl_from_dict(d: dict, cls=None):
    c = (cls or OracleCtl)()
    for f in CTL_SCALARS:
        if f in d:
            setattr(c, f, type(getattr(c, f))(d[f]))
    for f in ("smooth_h_mean", "smooth_h_var", "smooth_y"):
        if f in d:
            arr = getattr(c, f)
            for i, v in enumerate(d[f]):
                arr[i] = v
    return c


def config_to_dict(c) -> dict:
    return {f: getattr(c, f) for f, _ in CONFIG_FIELDS}


def config_from_dict(d: dict, cls=None):
    """Fields missing from d (records written before they existed) stay 0."""
    c = (cls or OracleConfig)()
    for f, _ in CONFIG_FIELDS:
        if f in d:
            setattr(c, f, d[f])
    return c


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def reference_dir() -> str:
    """Where the reference's source tree is read from when the checker builds
    it: $SVPF_REFERENCE_DIR, else the build container's copy."""
    return os.environ.get("SVPF_REFERENCE_DIR") or "/root/reference"


def build(quiet: bool = True) -> None:
    """Compile the oracle and, where the reference tree exists, the reference
    build and the reference callers linked to this engine (test checkers)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE, "all"], check=True, stdout=out)
    ref = reference_dir()
    if os.path.isdir(os.path.join(ref, "src")):
        env = dict(os.environ, SVPF_REFERENCE_DIR=ref)
        subprocess.run(["make", "-C", HERE, "ref", "callers"], check=True, stdout=out, env=env)


_lib = None



V2_FIELDS = [("rho", "f"), ("sigma_z", "f"), ("mu", "f"), ("nu", "f"), ("lik_offset", "f"),
             ("student_t_const", "f"), ("student_t_implied_offset", "f"), ("gamma", "f"),
             ("delta_rho", "f"), ("delta_sigma", "f"), ("mim_jump_prob", "f"), ("mim_jump_scale", "f"),
             ("guide_strength_base", "f"), ("guide_strength_max", "f"), ("guide_innovation_threshold", "f"),
             ("guided_alpha_base", "f"), ("guided_alpha_shock", "f"), ("guided_innovation_thresh_predict", "f"),
             ("use_guide", "i"), ("use_guided_predict", "i"), ("use_guide_preserving", "i"),
             ("use_newton", "i"), ("use_full_newton", "i"), ("use_rejuvenation", "i"),
             ("rejuv_ksd_threshold", "f"), ("rejuv_prob", "f"), ("rejuv_blend", "f"),
             ("use_adaptive_mu", "i"), ("mu_ema_alpha", "f"), ("use_adaptive_sigma", "i"),
             ("sigma_boost_threshold", "f"), ("sigma_boost_max", "f"), ("step_size", "f"), ("temperature", "f"),
             ("rmsprop_rho", "f"), ("rmsprop_eps", "f"), ("n_stein_steps", "i"), ("n_anneal_steps", "i"),
             ("stein_sign_mode", "i")]


class OracleV2Params(C.Structure):
    """oracle_v2_params: the scalar arguments of svpf_fully_fused_step_v2."""
    _fields_ = [(k, C.c_float if t == "f" else C.c_int) for k, t in V2_FIELDS]

    def to_dict(self):
        return {k: getattr(self, k) for k, _ in V2_FIELDS}

    @classmethod
    def from_dict(cls, d):
        p = cls()
        for k, _ in V2_FIELDS:
            if k in d:
                setattr(p, k, d[k])
        return p


class OracleV2Out(C.Structure):
    _fields_ = [("h_mean", C.c_float), ("vol", C.c_float), ("loglik", C.c_float), ("bandwidth", C.c_float),
                ("ksd", C.c_float)]

def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle_svpf.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.svpf_oracle_tick.restype = C.c_int
        L.svpf_oracle_tick.argtypes = [C.POINTER(OracleConfig), C.POINTER(OracleParams),
                                       C.POINTER(OracleCtl), C.c_int] + [C.POINTER(C.c_double)] * 4 + [
            C.c_float, C.c_float, C.POINTER(OracleNoise), C.POINTER(OracleOut), C.c_int]
        L.svpf_oracle_initialize.restype = C.c_int
        L.svpf_oracle_initialize.argtypes = [C.POINTER(OracleConfig), C.POINTER(OracleParams),
                                             C.POINTER(OracleCtl), C.c_int] + [C.POINTER(C.c_double)] * 3 + [
            C.POINTER(C.c_float), C.c_uint64, C.c_int]
        L.svpf_oracle_ctl_defaults.argtypes = [C.POINTER(OracleCtl)]
        L.svpf_oracle_config_defaults.argtypes = [C.POINTER(OracleConfig), C.c_int, C.c_float]
        L.svpf_oracle_philox.argtypes = [C.c_uint32] * 6 + [C.POINTER(C.c_uint32)]
        L.svpf_oracle_batch_tick_f32.restype = C.c_int
        L.svpf_oracle_batch_tick_f32.argtypes = [
            C.c_int, C.POINTER(OracleConfig), C.POINTER(OracleParams), C.POINTER(OracleCtl),
            C.POINTER(C.c_int), C.c_int] + [C.POINTER(C.c_float)] * 6 + [
            C.c_uint64, C.c_uint64, C.c_int, C.POINTER(OracleOut)]
        L.svpf_oracle_grad_supported.restype = C.c_int
        L.svpf_oracle_grad_supported.argtypes = [C.POINTER(OracleConfig)]
        L.svpf_oracle_v2_tick.restype = C.c_int
        L.svpf_oracle_v2_tick.argtypes = [C.POINTER(OracleV2Params), C.c_int] + [C.POINTER(C.c_double)] * 6 + [
            C.c_float] * 5 + [C.c_int] + [C.POINTER(C.c_double)] * 3 + [C.POINTER(OracleNoise), C.POINTER(OracleV2Out),
                                                                        C.c_int]
        L.svpf_oracle_grad_run2.restype = C.c_int
        L.svpf_oracle_grad_run2.argtypes = [C.POINTER(OracleConfig), C.c_int, C.c_int, C.POINTER(C.c_double),
                                            C.c_double, C.POINTER(C.c_float), C.POINTER(C.c_double),
                                            C.c_uint64, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                            C.POINTER(C.c_double), C.c_int]
        L.svpf_oracle_grad_run3.restype = C.c_int
        L.svpf_oracle_grad_run3.argtypes = L.svpf_oracle_grad_run2.argtypes + [C.c_int]
        L.svpf_oracle_grad_run.restype = C.c_int
        L.svpf_oracle_grad_run.argtypes = [C.POINTER(OracleConfig), C.c_int, C.c_int, C.POINTER(C.c_double),
                                           C.c_double, C.POINTER(C.c_float), C.POINTER(C.c_double),
                                           C.c_uint64, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                           C.POINTER(C.c_double)]
        L.svpf_oracle_estimator_run2.restype = C.c_int
        L.svpf_oracle_estimator_run2.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int] + [
            C.POINTER(C.c_float)] * 3 + [C.POINTER(C.c_double), C.c_int] + [C.POINTER(C.c_double)] * 6
        _lib = L
    return _lib


def default_config(n_stein_steps: int = 8, nu: float = 30.0) -> OracleConfig:
    c = OracleConfig()
    lib().svpf_oracle_config_defaults(C.byref(c), n_stein_steps, nu)
    return c


def default_ctl() -> OracleCtl:
    c = OracleCtl()
    lib().svpf_oracle_ctl_defaults(C.byref(c))
    return c


def grad_supported(cfg: OracleConfig) -> bool:
    return bool(lib().svpf_oracle_grad_supported(C.byref(cfg)))


def grad_run(cfg: OracleConfig, n: int, theta, ys, gamma: float = 0.0, w=None, seed: int = 0,
             filter_id: int = 0, objective: int = 0, truncate_every: int = 0):
    """FP64 forward-mode gradient oracle of one filter's run: initialisation
    from theta = (mu, rho, sigma_z, nu), then len(ys) ticks (Philox noise keyed
    by seed and filter_id).  Returns (loglik[T], grad[4] of sum_t w_t loglik_t,
    final particles[n])."""
    ys = np.ascontiguousarray(ys, np.float32)
    T = int(ys.shape[0])
    th = np.ascontiguousarray(theta, np.float64)
    ll = np.zeros(T)
    g = np.zeros(4)
    hf = np.zeros(n)
    wv = None if w is None else np.ascontiguousarray(w, np.float64)
    rc = lib().svpf_oracle_grad_run3(C.byref(cfg), n, T, _dptr(th), float(gamma), _fptr(ys),
                                     _dptr(wv) if wv is not None else None, seed, filter_id,
                                     _dptr(ll), _dptr(g), _dptr(hf), int(objective), int(truncate_every))
    if rc != 0:
        raise RuntimeError(f"grad oracle rc={rc}")
    return ll, g, hf


def run_loglik(cfg: OracleConfig, n: int, theta, ys, gamma: float = 0.0, seed: int = 0, filter_id: int = 0,
               precision: int = 0):
    """The main oracle (OracleFilter) run the same way as grad_run: Philox
    initialisation and noise, nu taken from theta.  Returns loglik[T]."""
    c = OracleConfig.from_buffer_copy(cfg)
    c.nu = float(theta[3])
    p = OracleParams(float(theta[1]), float(theta[2]), float(theta[0]), float(gamma))
    f = OracleFilter(n, c, p, precision)
    f.initialize(None, seed=seed, filter_id=filter_id)
    out = []
    yp = 0.0
    for t, y in enumerate(np.asarray(ys, np.float32)):
        o = f.step(float(y), yp, seed=seed, tick=t, filter_id=filter_id)
        out.append(o.loglik)
        yp = float(y)
    return np.array(out)


def estimator_run(n: int, n_stein: int, stein_lr: float, theta, ys, tape_init, tape_ticks,
                  truncate_every: int = 0, w=None, bw_fixed=None, return_bw: bool = False):
    """FP64 forward-mode restatement of the reference's differentiable torch
    model (SVPFParamEstimator.forward, py-torch/diff_svpf_torch.py:147-217)
    on one path with its noise as a tape.  Returns (loglik[T] predictive,
    vol[T], grad[4] of sum_t w_t loglik_t w.r.t. (mu, rho, sigma_z, nu)), and
    the per-tick bandwidths when return_bw; bw_fixed[T] replays bandwidths."""
    ys = np.ascontiguousarray(ys, np.float32)
    T = int(ys.shape[0])
    ti = np.ascontiguousarray(tape_init, np.float32)
    tt = np.ascontiguousarray(tape_ticks, np.float32)
    assert ti.shape == (n,) and tt.shape == (T, n // 2)
    th = np.ascontiguousarray(theta, np.float64)
    ll, vol, g = np.zeros(T), np.zeros(T), np.zeros(4)
    wv = None if w is None else np.ascontiguousarray(w, np.float64)
    bf = None if bw_fixed is None else np.ascontiguousarray(bw_fixed, np.float64)
    bo = np.zeros(T)
    rc = lib().svpf_oracle_estimator_run2(n, n_stein, float(stein_lr), T, _fptr(ys), _fptr(ti), _fptr(tt), _dptr(th),
                                          int(truncate_every), _dptr(wv) if wv is not None else None, _dptr(ll),
                                          _dptr(vol), _dptr(g), _dptr(bf) if bf is not None else None, _dptr(bo))
    if rc != 0:
        raise RuntimeError(f"estimator oracle rc={rc}")
    return (ll, vol, g, bo) if return_bw else (ll, vol, g)


class V2State:
    """Arrays and device scalars of one svpf_fully_fused_step_v2 filter, FP64."""

    ARRAYS = ("h", "h_prev", "grad", "lw", "v", "inv_hess")

    def __init__(self, n):
        self.n = n
        for a in self.ARRAYS:
            setattr(self, a, np.zeros(n))
        self.guide_mean = np.zeros(1)
        self.guide_var = np.zeros(1)
        self.mu_state = np.zeros(1)

    def copy(self):
        c = V2State(self.n)
        for a in self.ARRAYS + ("guide_mean", "guide_var", "mu_state"):
            setattr(c, a, getattr(self, a).copy())
        return c


def v2_tick(p: OracleV2Params, st: V2State, y_t, y_prev, h_mean_prev, vol_prev, ksd_prev, timestep,
            normals=None, uniforms=None, seed=0, filter_id=0, precision=0) -> OracleV2Out:
    nz = OracleNoise()
    keep = []
    if normals is not None:
        nrm = np.ascontiguousarray(normals, np.float32)
        uni = np.ascontiguousarray(uniforms, np.float32)
        keep += [nrm, uni]
        nz.mode, nz.n_normal_slots, nz.n_uniform_slots = 0, nrm.shape[0], uni.shape[0]
        nz.normals, nz.uniforms = _fptr(nrm), _fptr(uni)
    else:
        nz.mode = 1
    nz.seed, nz.tick, nz.filter_id = seed, timestep, filter_id
    out = OracleV2Out()
    rc = lib().svpf_oracle_v2_tick(C.byref(p), st.n, *[_dptr(getattr(st, a)) for a in V2State.ARRAYS],
                                   float(y_t), float(y_prev), float(h_mean_prev), float(vol_prev), float(ksd_prev),
                                   int(timestep), _dptr(st.guide_mean), _dptr(st.guide_var), _dptr(st.mu_state),
                                   C.byref(nz), C.byref(out), precision)
    if rc != 0:
        raise RuntimeError(f"oracle v2 tick rc={rc}")
    return out


def philox(k0, k1, c0, c1, c2, c3):
    out = (C.c_uint32 * 4)()
    lib().svpf_oracle_philox(k0, k1, c0, c1, c2, c3, out)
    return list(out)


class OracleFilter:
    """One filter driven by the oracle, state in float64 numpy arrays."""

    def __init__(self, n: int, cfg: OracleConfig, params: OracleParams, precision: int = 0):
        self.n = n
        self.cfg = cfg
        self.params = params
        self.ctl = default_ctl()
        m = 2 * n if cfg.use_two_factor else n   # two factors: [fast; slow]
        self.h = np.zeros(m)
        self.h_prev = np.zeros(m)
        self.v = np.zeros(m)
        self.log_w = np.zeros(n)
        self.precision = precision

    def initialize(self, init_normals=None, seed: int = 0, filter_id: int = 0):
        ptr = _fptr(np.ascontiguousarray(init_normals, np.float32)) if init_normals is not None else None
        keep = np.ascontiguousarray(init_normals, np.float32) if init_normals is not None else None
        rc = lib().svpf_oracle_initialize(C.byref(self.cfg), C.byref(self.params), C.byref(self.ctl),
                                          self.n, _dptr(self.h), _dptr(self.h_prev), _dptr(self.v),
                                          _fptr(keep) if keep is not None else ptr, seed, filter_id)
        assert rc == 0, rc

    def step(self, y_t, y_prev, normals=None, uniforms=None, seed=0, tick=0, filter_id=0):
        nz = OracleNoise()
        keep = []
        if normals is not None:
            nrm = np.ascontiguousarray(normals, np.float32)
            uni = np.ascontiguousarray(uniforms, np.float32)
            keep += [nrm, uni]
            nz.mode = 0
            nz.n_normal_slots = nrm.shape[0]
            nz.n_uniform_slots = uni.shape[0]
            nz.normals = _fptr(nrm)
            nz.uniforms = _fptr(uni)
        else:
            nz.mode = 1
        nz.seed = seed
        nz.tick = tick
        nz.filter_id = filter_id
        out = OracleOut()
        rc = lib().svpf_oracle_tick(C.byref(self.cfg), C.byref(self.params), C.byref(self.ctl), self.n,
                                    _dptr(self.h), _dptr(self.h_prev), _dptr(self.v), _dptr(self.log_w),
                                    float(y_t), float(y_prev), C.byref(nz), C.byref(out), self.precision)
        if rc != 0:
            raise RuntimeError(f"oracle tick failed rc={rc}")
        return out


# ---------------------------------------------------------------------------
# Reference CUDA step (GPU only)
# ---------------------------------------------------------------------------
class RefLib:
    def __init__(self, kind: str = "tape"):
        path = os.path.join(HERE, "_ref", f"libsvpf_ref_{kind}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = C.CDLL(path)
        L.svpf_ref_create.restype = C.c_void_p
        L.svpf_ref_create.argtypes = [C.c_int, C.c_int, C.c_float]
        L.svpf_ref_destroy.argtypes = [C.c_void_p]
        L.svpf_ref_apply_config.argtypes = [C.c_void_p, C.POINTER(OracleConfig)]
        L.svpf_ref_read_config.argtypes = [C.c_void_p, C.POINTER(OracleConfig)]
        L.svpf_ref_initialize.restype = C.c_int
        L.svpf_ref_initialize.argtypes = [C.c_void_p, C.POINTER(OracleParams), C.POINTER(C.c_float)]
        L.svpf_ref_set_state.restype = C.c_int
        L.svpf_ref_set_state.argtypes = [C.c_void_p, C.POINTER(OracleCtl)] + [C.POINTER(C.c_double)] * 4
        L.svpf_ref_get_state.restype = C.c_int
        L.svpf_ref_get_state.argtypes = [C.c_void_p, C.POINTER(OracleCtl)] + [C.POINTER(C.c_double)] * 4
        L.svpf_ref_step.restype = C.c_int
        L.svpf_ref_step.argtypes = [C.c_void_p, C.c_float, C.c_float, C.POINTER(OracleParams),
                                    C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_float), C.c_int,
                                    C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.svpf_ref_v2_step.restype = C.c_int
        L.svpf_ref_v2_step.argtypes = [C.POINTER(OracleV2Params), C.c_int] + [C.POINTER(C.c_double)] * 6 + [
            C.c_float] * 5 + [C.c_int] + [C.POINTER(C.c_double)] * 3 + [C.POINTER(C.c_float), C.c_int,
                                                                        C.POINTER(C.c_float), C.c_int,
                                                                        C.POINTER(OracleV2Out)]
        L.svpf_ref_v2_time.restype = C.c_int
        L.svpf_ref_v2_time.argtypes = [C.POINTER(OracleV2Params), C.c_int, C.POINTER(C.c_float), C.c_int,
                                       C.POINTER(C.c_float)]
        L.svpf_ref_steps_used.restype = C.c_int
        L.svpf_ref_steps_used.argtypes = [C.c_void_p]
        L.svpf_ref_time_steps.restype = C.c_int
        L.svpf_ref_time_steps.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.c_int,
                                          C.POINTER(OracleParams), C.POINTER(C.c_float)]
        self.L = L


def ref_v2_step(reflib, p: OracleV2Params, st: V2State, y_t, y_prev, h_mean_prev, vol_prev, ksd_prev, timestep,
                normals, uniforms):
    """The reference's svpf_fully_fused_step_v2 (tape build) on st, in place."""
    nrm = np.ascontiguousarray(normals, np.float32)
    uni = np.ascontiguousarray(uniforms, np.float32)
    out = OracleV2Out()
    flags = reflib.L.svpf_ref_v2_step(C.byref(p), st.n, *[_dptr(getattr(st, a)) for a in V2State.ARRAYS],
                                      float(y_t), float(y_prev), float(h_mean_prev), float(vol_prev),
                                      float(ksd_prev), int(timestep), _dptr(st.guide_mean), _dptr(st.guide_var),
                                      _dptr(st.mu_state), _fptr(nrm), nrm.shape[0], _fptr(uni), uni.shape[0],
                                      C.byref(out))
    return flags, out


class RefFilter:
    """The reference's svpf_step_graph on one filter, via the harness."""

    def __init__(self, reflib: RefLib, n: int, n_stein: int, nu: float):
        self.L = reflib.L
        self.n = n
        self.s = self.L.svpf_ref_create(n, n_stein, nu)
        if not self.s:
            raise RuntimeError("svpf_create failed")

    def close(self):
        if self.s:
            self.L.svpf_ref_destroy(self.s)
            self.s = None

    def read_config(self) -> OracleConfig:
        c = OracleConfig()
        self.L.svpf_ref_read_config(self.s, C.byref(c))
        return c

    def apply_config(self, cfg: OracleConfig):
        self.L.svpf_ref_apply_config(self.s, C.byref(cfg))

    def initialize(self, params: OracleParams, init_normals):
        z = np.ascontiguousarray(init_normals, np.float32)
        return self.L.svpf_ref_initialize(self.s, C.byref(params), _fptr(z))

    def get_state(self):
        ctl = OracleCtl()
        m = 2 * self.n if self.read_config().use_two_factor else self.n
        h, hp, v = (np.zeros(m) for _ in range(3))
        lw = np.zeros(self.n)
        rc = self.L.svpf_ref_get_state(self.s, C.byref(ctl), _dptr(h), _dptr(hp), _dptr(v), _dptr(lw))
        assert rc == 0, rc
        return ctl, h, hp, v, lw

    def set_state(self, ctl, h, hp, v, lw):
        arrs = [np.ascontiguousarray(a, np.float64) for a in (h, hp, v, lw)]
        rc = self.L.svpf_ref_set_state(self.s, C.byref(ctl), *[_dptr(a) for a in arrs])
        assert rc == 0, rc

    def steps_used(self) -> int:
        """Stein steps the last svpf_step_graph call ran."""
        return self.L.svpf_ref_steps_used(self.s)

    def step(self, y_t, y_prev, params, normals, uniforms):
        nrm = np.ascontiguousarray(normals, np.float32)
        uni = np.ascontiguousarray(uniforms, np.float32)
        ll, vol, hm = C.c_float(), C.c_float(), C.c_float()
        flags = self.L.svpf_ref_step(self.s, float(y_t), float(y_prev), C.byref(params),
                                     _fptr(nrm), nrm.shape[0], _fptr(uni), uni.shape[0],
                                     C.byref(ll), C.byref(vol), C.byref(hm))
        return flags, ll.value, vol.value, hm.value
