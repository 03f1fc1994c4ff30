"""Host-side mirror of the reference's Python binding over libsvpf_b200.so.

``SVPF`` keeps the method names, defaults and argument meaning of the
reference's ``pysvpf.SVPF`` (py-torch/svpf_python.cpp:483-653): ``initialize``,
``step``, ``run``, ``reset``, the ``set_*`` configuration calls, ``nu`` /
``lik_offset`` properties, ``get_particles``, ``get_ess``.  ``Batch`` drives
many independent filters with one persistent kernel launch per tick.

Everything runs through the C ABI declared in include/svpf.h; there is no
CPU path.  If the library has not been built this module raises on import of
the library instead of falling back.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsvpf_b200.so")
SMOOTH_MAX_LAG = 8

SVPF_OK = 0
ERRORS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "not initialized",
          4: "noise tape too short", 5: "non-finite observation or output", 6: "unsupported",
          7: "does not fit the HBM budget"}

_I, _F = C.c_int, C.c_float
CONFIG_FIELDS = [
    ("n_stein_steps", _I), ("nu", _F), ("student_t_implied_offset", _F), ("lik_offset", _F),
    ("use_exact_gradient", _I), ("use_svld", _I), ("use_annealing", _I), ("use_adaptive_beta", _I),
    ("n_anneal_steps", _I), ("temperature", _F), ("rmsprop_rho", _F), ("rmsprop_eps", _F),
    ("use_mim", _I), ("mim_jump_prob", _F), ("mim_jump_scale", _F), ("use_local_params", _I),
    ("delta_rho", _F), ("delta_sigma", _F), ("use_asymmetric_rho", _I), ("rho_up", _F),
    ("rho_down", _F), ("use_newton", _I), ("use_full_newton", _I), ("use_guided", _I),
    ("guided_alpha_base", _F), ("guided_alpha_shock", _F), ("guided_innovation_threshold", _F),
    ("use_rejuvenation", _I), ("rejuv_ksd_threshold", _F), ("rejuv_prob", _F), ("rejuv_blend", _F),
    ("use_guide", _I), ("use_guide_preserving", _I), ("guide_strength", _F), ("use_adaptive_guide", _I),
    ("guide_strength_base", _F), ("guide_strength_max", _F), ("guide_innovation_threshold", _F),
    ("use_adaptive_mu", _I), ("mu_process_var", _F), ("mu_obs_var_scale", _F), ("mu_min", _F),
    ("mu_max", _F), ("use_adaptive_sigma", _I), ("sigma_boost_threshold", _F),
    ("sigma_boost_max", _F), ("stein_repulsive_sign", _I), ("use_fan_mode", _I),
    ("stein_min_steps", _I), ("stein_max_steps", _I), ("ksd_improvement_threshold", _F),
    ("use_student_t_state", _I), ("nu_state", _F), ("use_smoothing", _I), ("smooth_lag", _I),
    ("smooth_output_lag", _I), ("use_heun", _I), ("use_two_factor", _I), ("rho_fast", _F),
    ("sigma_fast", _F), ("rho_slow", _F), ("sigma_slow", _F), ("bw_floor_fast", _F), ("bw_floor_slow", _F),
]


class Config(C.Structure):
    """svpf_config_t (include/svpf.h)."""
    _fields_ = CONFIG_FIELDS

    def to_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in CONFIG_FIELDS}

    def update(self, **kw):
        for k, v in kw.items():
            if k not in dict(CONFIG_FIELDS):
                raise KeyError(f"unknown configuration field {k!r}")
            setattr(self, k, v)
        return self


class Params(C.Structure):
    """SVPFParams (include/svpf.cuh:257-262 of the reference)."""
    _fields_ = [("rho", _F), ("sigma_z", _F), ("mu", _F), ("gamma", _F)]


class Ctl(C.Structure):
    """svpf_ctl_t: per-filter control record."""
    _fields_ = [
        ("guide_mean", C.c_double), ("guide_var", C.c_double), ("guide_K", C.c_double),
        ("loglik_sum", C.c_double), ("guide_mean_fast", C.c_double), ("guide_mean_slow", C.c_double),
        ("guide_var_fast", C.c_double), ("guide_var_slow", C.c_double), ("timestep", _I),
        ("guide_initialized", _I), ("stein_steps_used", _I), ("smooth_head", _I),
        ("guide_2f_initialized", _I), ("ksd_prev", _F), ("ksd_last", _F),
        ("vol_prev", _F), ("h_mean_prev", _F), ("bw", _F), ("bw_sq", _F), ("return_ema", _F),
        ("return_var", _F), ("sigma_z_effective", _F), ("mu_state", _F), ("mu_var", _F),
        ("y_prev", _F), ("h_fast_mean", _F), ("h_slow_mean", _F),
        ("smooth_h_mean", _F * SMOOTH_MAX_LAG), ("smooth_h_var", _F * SMOOTH_MAX_LAG),
        ("smooth_y", _F * SMOOTH_MAX_LAG), ("status", _I), ("reserved", _I),
    ]


class Out(C.Structure):
    """svpf_out_t: per-tick outputs of one filter."""
    _fields_ = [("loglik", _F), ("vol", _F), ("h_mean", _F), ("h_mean_raw", _F), ("bw", _F),
                ("ksd", _F), ("steps_used", _I), ("rejuv_fired", _I)]


_FP = C.POINTER(C.c_float)
_lib = None


class MSConfig(C.Structure):
    _fields_ = [("n_particles_reactive", _I), ("n_particles_inertial", _I), ("n_stein_reactive", _I),
                ("n_stein_inertial", _I), ("surprise_mild_threshold", _F), ("surprise_high_threshold", _F),
                ("boost_mild_factor", _F), ("boost_high_factor", _F), ("weight_reactive", _F),
                ("weight_inertial", _F)]


class MSOutput(C.Structure):
    _fields_ = [(k, _F) for k in ("vol_reactive", "vol_inertial", "h_reactive", "h_inertial", "loglik_reactive",
                                  "loglik_inertial", "vol_combined", "h_combined", "loglik_combined",
                                  "transient_magnitude", "transient_ratio", "ksd_reactive", "ksd_inertial")] + \
                [("stein_steps_reactive", _I), ("stein_steps_inertial", _I), ("surprise_reactive", _F),
                 ("cross_scale_boost", _I), ("mim_prob_inertial_used", _F), ("is_transient", _I),
                 ("is_regime_shift", _I), ("is_calm", _I)]


def lib() -> C.CDLL:
    """The engine library.  Raises if it is missing: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built (run build.py); the SVPF engine has no CPU fallback")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    sig = {
        "svpf_create": (vp, [_I, _I, _F, vp]),
        "svpf_destroy": (None, [vp]),
        "svpf_initialize": (None, [vp, C.POINTER(Params), C.c_ulonglong]),
        "svpf_step_graph": (None, [vp, _F, _F, C.POINTER(Params), _FP, _FP, _FP]),
        "svpf_step_optimized": (None, [vp, _F, _F, C.POINTER(Params), _FP, _FP]),
        "svpf_step_adaptive": (None, [vp, _F, _F, C.POINTER(Params), _FP, _FP, _FP]),
        "svpf_step_seeded": (None, [vp, _F, C.POINTER(Params), C.c_ulonglong, vp]),
        "svpf_run_sequence": (None, [vp, _FP, _I, C.POINTER(Params), _FP, _FP]),
        "svpf_get_particles": (None, [vp, _FP]),
        "svpf_get_stats": (None, [vp, _FP, _FP]),
        "svpf_get_ess": (_F, [vp]),
        "svpf_get_ksd_stats": (None, [vp, _FP, C.POINTER(_I)]),
        "svpf_graph_is_captured": (C.c_bool, [vp]),
        "svpf_graph_invalidate": (None, [vp]),
        "svpf_last_error": (_I, [vp]),
        "svpf_get_config": (None, [vp, C.POINTER(Config)]),
        "svpf_config_init": (None, [C.POINTER(Config), _I, _F]),
        "svpf_set_config": (None, [vp, C.POINTER(Config)]),
        "svpf_get_state": (_I, [vp, C.POINTER(Ctl), _FP, _FP, _FP, _FP]),
        "svpf_set_state": (_I, [vp, C.POINTER(Ctl), _FP, _FP, _FP, _FP]),
        "svpf_get_state_2f": (_I, [vp, _FP, _FP, _FP, _FP, _FP, _FP]),
        "svpf_set_state_2f": (_I, [vp, _FP, _FP, _FP, _FP, _FP, _FP]),
        "svpf_set_noise_tape": (_I, [vp, _FP, _I, _FP, _I]),
        "svpf_get_last_output": (_I, [vp, C.POINTER(Out)]),
        "svpf_set_cluster_size": (_I, [vp, _I]),
        "svpf_batch_create": (vp, [_I, C.POINTER(_I), C.POINTER(Config), C.POINTER(Params), vp]),
        "svpf_batch_destroy": (None, [vp]),
        "svpf_batch_initialize": (_I, [vp, C.c_ulonglong]),
        "svpf_batch_step": (_I, [vp, _FP, _FP, _FP, _FP, _FP]),
        "svpf_batch_step_device": (_I, [vp, vp, vp, vp]),
        "svpf_batch_graph_launch": (_I, [vp, vp, vp, vp]),
        "svpf_batch_sync": (_I, [vp]),
        "svpf_batch_n_filters": (_I, [vp]),
        "svpf_batch_kernel_launches": (_I, [vp]),
        "svpf_batch_get_ctl": (_I, [vp, C.POINTER(Ctl)]),
        "svpf_batch_get_particles": (_I, [vp, _I, _FP]),
        "svpf_batch_set_noise_tape": (_I, [vp, _FP, _I, _FP, _I]),
        "svpf_batch_tile_of": (_I, [vp, _I, C.POINTER(_I), C.POINTER(_I)]),
        "svpf_batch_tile_of_filter": (_I, [vp, _I, C.POINTER(_I), C.POINTER(_I)]),
        "svpf_batch_set_tile": (_I, [vp, _I, _I, _I]),
        "svpf_batch_get_state": (_I, [vp, _I, C.POINTER(Ctl), _FP, _FP, _FP, _FP]),
        "svpf_batch_get_params": (_I, [vp, _I, C.POINTER(Params)]),
        "svpf_batch_set_params": (_I, [vp, _I, C.POINTER(Params)]),
        "svpf_batch_set_state": (_I, [vp, _I, C.POINTER(Ctl), _FP, _FP, _FP, _FP]),
        "svpf_autotune": (_I, [C.POINTER(_I), _I, _I]),
        "svpf_tile_choice": (_I, [_I, C.POINTER(_I), C.POINTER(_I)]),
        "svpf_build_info": (C.c_char_p, []),
        "svpf_grad_supported": (_I, [C.POINTER(Config)]),
        "svpf_grad_create": (vp, [_I, C.POINTER(_I), C.POINTER(Config), _I, _I, vp]),
        "svpf_grad_destroy": (None, [vp]),
        "svpf_grad_forward": (_I, [vp, _FP, _FP, _FP, _I, C.c_ulonglong, _FP, C.POINTER(C.c_double)]),
        "svpf_grad_backward": (_I, [vp, _FP, C.POINTER(C.c_double)]),
        "svpf_grad_forward_device": (_I, [vp, vp, vp, vp, _I, C.c_ulonglong, vp]),
        "svpf_grad_backward_device": (_I, [vp, vp, vp]),
        "svpf_grad_checkpoint_every": (_I, [vp]),
        "svpf_grad_segment_records": (_I, [vp]),
        "svpf_grad_set_segment_records": (_I, [vp, _I]),
        "svpf_grad_set_objective": (_I, [vp, _I]),
        "svpf_grad_get_status": (_I, [vp, C.POINTER(_I)]),
        "svpf_grad_run_records": (_I, [vp]),
        "svpf_grad_set_truncation": (_I, [vp, _I]),
        "svpf_grad_truncation": (_I, [vp]),
        "svpf_grad_set_run_records": (_I, [vp, _I]),
        "svpf_stream_create": (vp, [_I, C.c_size_t, _I, vp]),
        "svpf_stream_destroy": (None, [vp]),
        "svpf_stream_set_seed": (None, [vp, C.c_ulonglong]),
        "svpf_stream_admit": (_I, [vp, _I, C.POINTER(Config), C.POINTER(Params), C.c_ulonglong]),
        "svpf_stream_evict": (_I, [vp, _I]),
        "svpf_stream_bytes_in_use": (C.c_size_t, [vp]),
        "svpf_stream_bytes_budget": (C.c_size_t, [vp]),
        "svpf_stream_process": (_I, [vp, _I, C.POINTER(_I), _FP, vp]),
        "svpf_stream_process_device": (_I, [vp, _I, _I, vp, vp, vp]),
        "svpf_stream_get_ctl": (_I, [vp, _I, C.POINTER(Ctl)]),
        "svpf_stream_get_particles": (_I, [vp, _I, _FP]),
        "svpf_stream_kernel_launches": (C.c_longlong, [vp]),
        "svpf_fully_fused_v2_supported": (C.c_bool, [_I]),
        "svpf_ms_default_config": (MSConfig, []),
        "svpf_ms_batch_create": (vp, [_I, C.POINTER(MSConfig), C.POINTER(Params), vp]),
        "svpf_ms_batch_destroy": (None, [vp]),
        "svpf_ms_batch_init": (_I, [vp, _F, C.c_ulonglong]),
        "svpf_ms_batch_step": (_I, [vp, _FP, C.POINTER(MSOutput)]),
        "svpf_ms_batch_inner": (vp, [vp]),
        "svpf_batch_last_outputs": (_I, [vp, C.POINTER(Out)]),
        "svpf_batch_get_config": (_I, [vp, _I, C.POINTER(Config)]),
        "svpf_fully_fused_step_v2": (_I, [vp] * 7 + [_F] * 5 + [vp] * 7 + [_F] * 18 + [_I] * 6 + [_F] * 3 +
                                     [_I, vp, _F, _I] + [_F] * 6 + [_I] * 5 + [vp]),
        "svpf_fully_fused_v2_rng_create": (vp, [C.c_ulonglong, C.c_uint]),
        "svpf_fully_fused_v2_rng_destroy": (None, [vp]),
        "svpf_fully_fused_v2_rng_get": (_I, [vp, vp]),
        "svpf_fully_fused_v2_rng_set": (_I, [vp, vp]),
        "svpf_debug_philox": (_I, [C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), _I]),
        "svpf_measure_pipe_rates": (_I, [C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "svpf_estimator_create": (vp, [_I, _I, _I, _F, _I, _I, _I, vp]),
        "svpf_estimator_destroy": (None, [vp]),
        "svpf_estimator_tape_floats": (C.c_longlong, [_I, _I]),
        "svpf_estimator_forward": (_I, [vp, _FP, _FP, _I, C.c_ulonglong, _FP, _FP, _FP, C.POINTER(C.c_double)]),
        "svpf_estimator_backward": (_I, [vp, _FP, C.POINTER(C.c_double)]),
        "svpf_estimator_forward_device": (_I, [vp, vp, vp, _I, C.c_ulonglong, vp, vp, vp]),
        "svpf_estimator_backward_device": (_I, [vp, vp, vp]),
        "svpf_estimator_get_status": (_I, [vp, C.POINTER(_I)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _fp(a: np.ndarray):
    return a.ctypes.data_as(_FP)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _tape(normals, uniforms, width: int):
    """A noise tape as the C entry points read it: [slots][width] float32
    rows.  A 1-D array of ``width`` values is one slot; any other shape is
    refused here, since the C side reads slots x width values from the
    pointer and cannot check the buffer's size."""
    out = []
    for name, a in (("normals", normals), ("uniforms", uniforms)):
        if a is None and name == "uniforms":   # no uniform slots: the C call takes (NULL, 0)
            out.append(None)
            continue
        a = _f32(a)
        if a.ndim == 1 and a.shape[0] == width:
            a = a[None, :]
        if a.ndim != 2 or a.shape[1] != width or a.shape[0] < 1:
            raise ValueError(f"{name} tape must be [slots, {width}], got shape {a.shape}")
        out.append(a)
    return tuple(out)


def default_config(n_stein_steps: int = 8, nu: float = 30.0) -> Config:
    """The reference's svpf_create defaults (svpf_optimized_graph.cu:116-283)."""
    c = Config()
    lib().svpf_config_init(C.byref(c), int(n_stein_steps), float(nu))
    return c


def production_config(nu: float = 30.0, max_steps: int = 8) -> Config:
    """The batched/plain production configuration used by the benchmarks:
    svpf_create defaults plus full Newton, at most ``max_steps`` Stein
    iterations over 3 annealing stages."""
    return default_config(max_steps, nu).update(use_newton=1, use_full_newton=1, stein_min_steps=4,
                                                stein_max_steps=max_steps, n_anneal_steps=3)


@dataclass
class SVPFResult:
    """Mirror of pysvpf.SVPFResult."""
    log_lik: float
    vol_mean: float
    vol_std: float
    h_mean: float
    mu_estimate: float


class SVPF:
    """One filter; mirror of pysvpf.SVPF (py-torch/svpf_python.cpp:57-480)."""

    def __init__(self, n_particles: int = 400, n_stein: int = 8, nu: float = 30.0, stream=None):
        self._s = lib().svpf_create(int(n_particles), int(n_stein), float(nu), stream)
        if not self._s:
            raise RuntimeError("Failed to create SVPF filter")
        self._n = int(n_particles)
        self._n_stein = int(n_stein)
        self.params = Params(0.97, 0.15, -3.5, -0.5)
        self._y_prev = 0.0
        self._initialized = False
        self.set_defaults()

    def close(self):
        if getattr(self, "_s", None):
            lib().svpf_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- configuration -----------------------------------------------------
    @property
    def config(self) -> Config:
        c = Config()
        lib().svpf_get_config(self._s, C.byref(c))
        return c

    def configure(self, **kw) -> "SVPF":
        c = self.config.update(**kw)
        lib().svpf_set_config(self._s, C.byref(c))
        return self

    def _ctl(self) -> Ctl:
        c = Ctl()
        self._check(lib().svpf_get_state(self._s, C.byref(c), None, None, None, None))
        return c

    def _set_ctl(self, **kw):
        c = self._ctl()
        for k, v in kw.items():
            setattr(c, k, v)
        self._check(lib().svpf_set_state(self._s, C.byref(c), None, None, None, None))

    def set_defaults(self):
        """Production defaults of the reference binding (svpf_python.cpp:90-176)."""
        self.configure(
            nu=30.0, lik_offset=0.345, use_asymmetric_rho=1, rho_up=0.98, rho_down=0.93, use_svld=1,
            temperature=0.45, rmsprop_rho=0.9, rmsprop_eps=1e-6, use_annealing=1, n_anneal_steps=5,
            use_mim=1, mim_jump_prob=0.25, mim_jump_scale=9.0, use_adaptive_beta=1, use_rejuvenation=1,
            rejuv_ksd_threshold=0.05, rejuv_prob=0.30, rejuv_blend=0.30, use_newton=1, use_full_newton=1,
            use_exact_gradient=1, stein_min_steps=8, stein_max_steps=16, ksd_improvement_threshold=0.05,
            use_guided=1, guided_alpha_base=0.0, guided_alpha_shock=0.40, guided_innovation_threshold=1.5,
            use_guide=1, use_guide_preserving=1, guide_strength=0.05, use_adaptive_guide=1,
            guide_strength_base=0.05, guide_strength_max=0.30, guide_innovation_threshold=1.0,
            use_adaptive_mu=1, mu_process_var=0.001, mu_obs_var_scale=11.0, mu_min=-4.0, mu_max=-1.0,
            use_adaptive_sigma=1, sigma_boost_threshold=0.95, sigma_boost_max=3.2, use_local_params=0,
            delta_rho=0.0, delta_sigma=0.0)
        self._set_ctl(guide_mean=0.0, guide_var=0.0, guide_K=0.0, guide_initialized=0, mu_state=-3.5,
                      mu_var=1.0, sigma_z_effective=0.10)

    def set_adaptive_mu(self, enabled=True, process_var=0.001, obs_var_scale=11.0, mu_min=-4.0, mu_max=-1.0):
        self.configure(use_adaptive_mu=int(enabled), mu_process_var=process_var,
                       mu_obs_var_scale=obs_var_scale, mu_min=mu_min, mu_max=mu_max)

    def set_adaptive_sigma(self, enabled=True, threshold=0.95, max_boost=3.2):
        self.configure(use_adaptive_sigma=int(enabled), sigma_boost_threshold=threshold, sigma_boost_max=max_boost)

    def set_adaptive_guide(self, enabled=True, base=0.05, max=0.30, threshold=1.0):  # noqa: A002
        self.configure(use_adaptive_guide=int(enabled), guide_strength_base=base, guide_strength_max=max,
                       guide_innovation_threshold=threshold)

    def set_asymmetric_rho(self, enabled=True, rho_up=0.98, rho_down=0.93):
        self.configure(use_asymmetric_rho=int(enabled), rho_up=rho_up, rho_down=rho_down)

    def set_mim(self, enabled=True, jump_prob=0.25, jump_scale=9.0):
        self.configure(use_mim=int(enabled), mim_jump_prob=jump_prob, mim_jump_scale=jump_scale)

    def set_svld(self, enabled=True, temperature=0.45):
        self.configure(use_svld=int(enabled), temperature=temperature)

    def set_annealing(self, enabled=True, n_steps=5):
        self.configure(use_annealing=int(enabled), n_anneal_steps=n_steps)

    def set_newton(self, enabled=True):
        self.configure(use_newton=int(enabled))

    def set_guide(self, enabled=True, strength=0.05):
        self.configure(use_guide=int(enabled), guide_strength=strength)

    def set_adaptive_beta(self, enabled=True):
        self.configure(use_adaptive_beta=int(enabled))

    def set_full_newton(self, enabled=True):
        self.configure(use_full_newton=int(enabled))

    def set_exact_gradient(self, enabled=True):
        self.configure(use_exact_gradient=int(enabled))

    def set_stein_steps(self, min_steps=8, max_steps=16, ksd_threshold=0.05):
        self.configure(stein_min_steps=min_steps, stein_max_steps=max_steps, ksd_improvement_threshold=ksd_threshold)

    def set_guided_innovation(self, alpha_base=0.0, alpha_shock=0.40, threshold=1.5):
        self.configure(guided_alpha_base=alpha_base, guided_alpha_shock=alpha_shock,
                       guided_innovation_threshold=threshold)

    def set_rejuvenation(self, enabled=True, ksd_threshold=0.05, prob=0.30, blend=0.30):
        self.configure(use_rejuvenation=int(enabled), rejuv_ksd_threshold=ksd_threshold, rejuv_prob=prob,
                       rejuv_blend=blend)

    def set_params(self, rho, sigma_z, mu, gamma):
        self.params = Params(rho, sigma_z, mu, gamma)
        self.invalidate_graph()

    @property
    def nu(self) -> float:
        return self.config.nu

    @nu.setter
    def nu(self, value: float):
        # the reference setter recomputes only the normaliser; the implied
        # offset stays at its create-time value (svpf_python.cpp:259-266)
        self.configure(nu=float(value))

    @property
    def lik_offset(self) -> float:
        return self.config.lik_offset

    @lik_offset.setter
    def lik_offset(self, value: float):
        self.configure(lik_offset=float(value))

    @property
    def n_particles(self) -> int:
        return self._n

    @property
    def n_stein_steps(self) -> int:
        return self._n_stein

    # -- core ----------------------------------------------------------------
    def _check(self, rc: int):
        if rc != SVPF_OK:
            raise RuntimeError(f"svpf error {rc}: {ERRORS.get(rc, '?')}")

    def initialize(self, rho=0.97, sigma_z=0.15, mu=-3.5, gamma=-0.5, seed=42):
        self.params = Params(rho, sigma_z, mu, gamma)
        lib().svpf_initialize(self._s, C.byref(self.params), int(seed))
        self._check(lib().svpf_last_error(self._s))
        if self.config.use_adaptive_mu:
            self._set_ctl(mu_state=mu, mu_var=0.01)
        self._y_prev = 0.0
        self._initialized = True

    def step(self, y_t: float) -> SVPFResult:
        if not self._initialized:
            raise RuntimeError("Filter not initialized. Call initialize() first.")
        ll, vol, hm = C.c_float(), C.c_float(), C.c_float()
        lib().svpf_step_graph(self._s, float(y_t), float(self._y_prev), C.byref(self.params),
                              C.byref(ll), C.byref(vol), C.byref(hm))
        rc = lib().svpf_last_error(self._s)
        if rc not in (SVPF_OK, 5):
            self._check(rc)
        self._y_prev = float(y_t)
        mu_est = self._ctl().mu_state if self.config.use_adaptive_mu else self.params.mu
        return SVPFResult(ll.value, vol.value, 0.0, hm.value, mu_est)

    def run(self, observations):
        if not self._initialized:
            raise RuntimeError("Filter not initialized. Call initialize() first.")
        obs = _f32(observations)
        if obs.ndim != 1:
            raise RuntimeError("Observations must be 1-dimensional")
        T = obs.shape[0]
        vol, hm, ll = (np.empty(T, np.float32) for _ in range(3))
        p = C.byref(self.params)
        for t in range(T):
            a, b, c = C.c_float(), C.c_float(), C.c_float()
            lib().svpf_step_graph(self._s, float(obs[t]), float(self._y_prev), p, C.byref(a), C.byref(b), C.byref(c))
            ll[t], vol[t], hm[t] = a.value, b.value, c.value
            self._y_prev = float(obs[t])
        return vol, hm, ll

    def reset(self, seed=42):
        lib().svpf_initialize(self._s, C.byref(self.params), int(seed))
        if self.config.use_adaptive_mu:
            self._set_ctl(mu_state=self.params.mu, mu_var=0.01)
        self._y_prev = 0.0

    def get_particles(self) -> np.ndarray:
        out = np.empty(self._n, np.float32)
        lib().svpf_get_particles(self._s, _fp(out))
        return out

    def get_ess(self) -> float:
        return float(lib().svpf_get_ess(self._s))

    def invalidate_graph(self):
        lib().svpf_graph_invalidate(self._s)

    def is_graph_captured(self) -> bool:
        return bool(lib().svpf_graph_is_captured(self._s))

    # -- engine extras (no reference counterpart) ------------------------------
    def last_error(self) -> int:
        return int(lib().svpf_last_error(self._s))

    def last_output(self) -> Out:
        o = Out()
        self._check(lib().svpf_get_last_output(self._s, C.byref(o)))
        return o

    def get_state(self):
        ctl = Ctl()
        h, hp, v, lw = (np.empty(self._n, np.float32) for _ in range(4))
        self._check(lib().svpf_get_state(self._s, C.byref(ctl), _fp(h), _fp(hp), _fp(v), _fp(lw)))
        return ctl, h, hp, v, lw

    def set_state(self, ctl: Ctl, h, hp, v, lw):
        """Restore the control record and the arrays; an array given as None is left as it is."""
        arrs = [None if a is None else _f32(a) for a in (h, hp, v, lw)]
        self._check(lib().svpf_set_state(self._s, C.byref(ctl), *[None if a is None else _fp(a) for a in arrs]))

    def get_state_2f(self):
        """Two-factor particle arrays, each [2n] as (fast, slow) concatenated:
        positions, previous positions, RMSProp moments."""
        n = self._n
        bufs = [np.empty(n, np.float32) for _ in range(6)]
        self._check(lib().svpf_get_state_2f(self._s, *[_fp(b) for b in bufs]))
        return (np.concatenate(bufs[0:2]), np.concatenate(bufs[2:4]), np.concatenate(bufs[4:6]))

    def set_state_2f(self, h, hp, v):
        n = self._n
        arrs = [_f32(a) for a in (h, hp, v)]
        parts = [np.ascontiguousarray(a[k * n:(k + 1) * n]) for a in arrs for k in range(2)]
        self._check(lib().svpf_set_state_2f(self._s, *[_fp(a) for a in parts]))

    def set_noise_tape(self, normals=None, uniforms=None):
        if normals is None:
            self._check(lib().svpf_set_noise_tape(self._s, None, 0, None, 0))
            return
        self._tape = _tape(normals, uniforms, self._n)
        nrm, uni = self._tape
        self._check(lib().svpf_set_noise_tape(self._s, _fp(nrm), nrm.shape[0], None if uni is None else _fp(uni),
                                                       0 if uni is None else uni.shape[0]))

    def set_cluster_size(self, ctas: int):
        self._check(lib().svpf_set_cluster_size(self._s, int(ctas)))

    def step_raw(self, y_t: float, y_prev: float):
        """One svpf_step_graph call with explicit y_prev; returns the full outputs."""
        lib().svpf_step_graph(self._s, float(y_t), float(y_prev), C.byref(self.params), None, None, None)
        rc = lib().svpf_last_error(self._s)
        return rc, self.last_output()


class Batch:
    """Many independent filters; one persistent kernel launch per tick."""

    def __init__(self, ns, configs, params, stream=None):
        ns = np.ascontiguousarray(ns, dtype=np.int32)
        F = int(ns.shape[0])
        if isinstance(configs, Config):
            configs = [configs] * F
        if isinstance(params, Params):
            params = [params] * F
        self._cfgs = (Config * F)(*configs)
        self._prms = (Params * F)(*params)
        self._ns = ns
        self._b = lib().svpf_batch_create(F, ns.ctypes.data_as(C.POINTER(_I)), self._cfgs, self._prms, stream)
        if not self._b:
            raise RuntimeError("svpf_batch_create failed")
        self.F = F

    def close(self):
        if getattr(self, "_b", None):
            lib().svpf_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != SVPF_OK:
            raise RuntimeError(f"svpf batch error {rc}: {ERRORS.get(rc, '?')}")

    def initialize(self, seed: int = 0):
        self._check(lib().svpf_batch_initialize(self._b, int(seed)))

    def step(self, y_t, y_prev):
        """One tick from host observations; returns host (loglik, vol, h_mean)."""
        yt, yp = _f32(y_t), _f32(y_prev)
        ll, vol, hm = (np.empty(self.F, np.float32) for _ in range(3))
        self._check(lib().svpf_batch_step(self._b, _fp(yt), _fp(yp), _fp(ll), _fp(vol), _fp(hm)))
        return ll, vol, hm

    def step_device(self, d_y_t: int, d_y_prev: int, d_out: int | None = None):
        """One tick from device pointers (asynchronous)."""
        self._check(lib().svpf_batch_step_device(self._b, d_y_t, d_y_prev, d_out))

    def graph_launch(self, d_y_t: int, d_y_prev: int, d_out: int | None = None):
        self._check(lib().svpf_batch_graph_launch(self._b, d_y_t, d_y_prev, d_out))

    def sync(self):
        self._check(lib().svpf_batch_sync(self._b))

    @property
    def kernel_launches(self) -> int:
        return int(lib().svpf_batch_kernel_launches(self._b))

    def ctl(self):
        arr = (Ctl * self.F)()
        self._check(lib().svpf_batch_get_ctl(self._b, arr))
        return arr

    def get_particles(self, f: int) -> np.ndarray:
        """Positions of filter f: [n], or [2n] (fast then slow) for two factors."""
        m = 2 if self._cfgs[f].use_two_factor else 1
        out = np.empty(m * int(self._ns[f]), np.float32)
        self._check(lib().svpf_batch_get_particles(self._b, int(f), _fp(out)))
        return out

    def get_state(self, f: int):
        """(ctl, h, h_prev, v, log_w) of filter f (h/h_prev/v [2n] for two factors)."""
        n = int(self._ns[f])
        m = (2 if self._cfgs[f].use_two_factor else 1) * n
        ctl = Ctl()
        h, hp, v = (np.empty(m, np.float32) for _ in range(3))
        lw = np.empty(n, np.float32)
        self._check(lib().svpf_batch_get_state(self._b, int(f), C.byref(ctl), _fp(h), _fp(hp), _fp(v), _fp(lw)))
        return ctl, h, hp, v, lw

    def set_state(self, f: int, ctl=None, h=None, hp=None, v=None, lw=None):
        arrs = [None if a is None else _f32(a) for a in (h, hp, v, lw)]
        self._check(lib().svpf_batch_set_state(self._b, int(f), None if ctl is None else C.byref(ctl),
                                               *[None if a is None else _fp(a) for a in arrs]))

    def set_noise_tape(self, normals=None, uniforms=None):
        if normals is None:
            self._check(lib().svpf_batch_set_noise_tape(self._b, None, 0, None, 0))
            return
        self._tape = _tape(normals, uniforms, int(self._ns.max()))
        nrm, uni = self._tape
        self._check(lib().svpf_batch_set_noise_tape(self._b, _fp(nrm), nrm.shape[0], None if uni is None else _fp(uni),
                                                             0 if uni is None else uni.shape[0]))

    def tile_of(self, n: int):
        r, s = C.c_int(), C.c_int()
        lib().svpf_batch_tile_of(self._b, int(n), C.byref(r), C.byref(s))
        return r.value, s.value

    def tile_of_filter(self, f: int):
        """(rows per thread, column split) filter f runs with."""
        r, s = C.c_int(), C.c_int()
        self._check(lib().svpf_batch_tile_of_filter(self._b, int(f), C.byref(r), C.byref(s)))
        return r.value, s.value

    def set_tile(self, f: int, rows_per_thread: int, col_split: int):
        """Force filter f's tile shape (a compiled batch tile)."""
        self._check(lib().svpf_batch_set_tile(self._b, int(f), int(rows_per_thread), int(col_split)))


def grad_config(n_stein: int = 8, nu: float = 12.0, full_newton: bool = True, **kw) -> Config:
    """The svpf_create defaults moved into the differentiable set: the model's
    rho in predict (no asymmetric rho), no rejuvenation, fixed beta schedule
    and a fixed Stein budget of n_stein iterations over 3 stages."""
    c = default_config(n_stein, nu)
    c.update(use_asymmetric_rho=0, use_rejuvenation=0, use_adaptive_beta=0, use_newton=int(full_newton),
             use_full_newton=int(full_newton), stein_min_steps=n_stein, stein_max_steps=n_stein,
             n_anneal_steps=3, use_exact_gradient=1)
    c.update(**kw)
    return c


class Grad:
    """Gradient engine: d(sum_t w_t loglik_t)/d(mu, rho, sigma_z, nu) for F
    filters over a run of T ticks (svpf_grad_* in the C ABI).  Reverse mode
    with a checkpoint every `checkpoint_every` ticks."""

    def __init__(self, ns, configs, T_max: int, checkpoint_every: int = 64, stream=None):
        ns = np.ascontiguousarray(ns, dtype=np.int32)
        F = int(ns.shape[0])
        if isinstance(configs, Config):
            configs = [configs] * F
        self._cfgs = (Config * F)(*configs)
        self._ns = ns
        self._g = lib().svpf_grad_create(F, ns.ctypes.data_as(C.POINTER(_I)), self._cfgs, int(T_max),
                                         int(checkpoint_every), stream)
        if not self._g:
            raise RuntimeError("svpf_grad_create failed (configuration outside the differentiable set, "
                               "sizes, or device)")
        self.F = F
        self.T_max = int(T_max)
        self.T = 0
        self.forward_id = 0

    def close(self):
        if getattr(self, "_g", None):
            lib().svpf_grad_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def supported(cfg: Config) -> bool:
        return bool(lib().svpf_grad_supported(C.byref(cfg)))

    TICK_LOGLIK = 0
    PREDICTIVE = 1

    def set_objective(self, objective: int):
        """0: each tick's loglik as the step reports it; 1: the predictive
        log p(y_t | y_1:t-1) at the predicted particles."""
        self._check(lib().svpf_grad_set_objective(self._g, int(objective)))
        return self

    @property
    def checkpoint_every(self) -> int:
        return int(lib().svpf_grad_checkpoint_every(self._g))

    @property
    def segment_records(self) -> bool:
        """True when the backward records whole checkpoint segments."""
        return bool(lib().svpf_grad_segment_records(self._g))

    @segment_records.setter
    def segment_records(self, on: bool):
        self._check(lib().svpf_grad_set_segment_records(self._g, int(bool(on))))

    @property
    def truncate_every(self) -> int:
        """Truncated backpropagation every k ticks (0: the exact gradient)."""
        return int(lib().svpf_grad_truncation(self._g))

    @truncate_every.setter
    def truncate_every(self, every: int):
        self._check(lib().svpf_grad_set_truncation(self._g, int(every)))

    @property
    def run_records(self) -> bool:
        """True when the forward keeps every tick's record (no recomputation)."""
        return bool(lib().svpf_grad_run_records(self._g))

    @run_records.setter
    def run_records(self, on: bool):
        self._check(lib().svpf_grad_set_run_records(self._g, int(bool(on))))

    def _check(self, rc):
        if rc != SVPF_OK:
            raise RuntimeError(f"svpf grad error {rc}: {ERRORS.get(rc, '?')}")

    def forward(self, theta, y, gamma=None, seed: int = 0):
        """theta [F,4] = (mu, rho, sigma_z, nu), y [F,T] (host arrays).
        Returns (loglik [F,T] float32, loglik_sum [F] float64)."""
        th = _f32(theta).reshape(self.F, 4)
        yy = _f32(y).reshape(self.F, -1)
        T = yy.shape[1]
        gm = None if gamma is None else _f32(gamma)
        ll = np.empty((self.F, T), np.float32)
        ls = np.empty(self.F, np.float64)
        self._check(lib().svpf_grad_forward(self._g, _fp(th), None if gm is None else _fp(gm), _fp(yy), T,
                                            int(seed), _fp(ll), ls.ctypes.data_as(C.POINTER(C.c_double))))
        self.T = T
        self.forward_id += 1
        return ll, ls

    def backward(self, w=None) -> np.ndarray:
        """Gradient [F,4] of sum_t w[f,t] loglik[f,t] (w None: all ones)."""
        ww = None if w is None else _f32(w).reshape(self.F, self.T)
        out = np.empty((self.F, 4), np.float64)
        self._check(lib().svpf_grad_backward(self._g, None if ww is None else _fp(ww),
                                             out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def forward_device(self, d_theta: int, d_gamma, d_y: int, T: int, seed: int, d_loglik: int):
        self._check(lib().svpf_grad_forward_device(self._g, d_theta, d_gamma, d_y, int(T), int(seed), d_loglik))
        self.T = int(T)
        self.forward_id += 1

    def backward_device(self, d_w, d_grad: int):
        self._check(lib().svpf_grad_backward_device(self._g, d_w, d_grad))

    def status(self) -> np.ndarray:
        """Per-filter status of the last forward/backward (SVPF_ERR_INVALID_ARG
        for a theta outside the domain)."""
        st = np.zeros(self.F, np.int32)
        self._check(lib().svpf_grad_get_status(self._g, st.ctypes.data_as(C.POINTER(_I))))
        return st


class Stream:
    """Request loop over instruments held in a fixed HBM budget
    (svpf_stream_* in the C ABI)."""

    def __init__(self, max_instruments: int, hbm_budget_bytes: int, n_max: int, stream=None, seed: int = 0):
        self._s = lib().svpf_stream_create(int(max_instruments), int(hbm_budget_bytes), int(n_max), stream)
        if not self._s:
            raise RuntimeError("svpf_stream_create failed (budget below the fixed records, sizes, or device)")
        lib().svpf_stream_set_seed(self._s, int(seed))
        self._cfg = {}
        self._n = {}

    def close(self):
        if getattr(self, "_s", None):
            lib().svpf_stream_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def admit(self, n: int, cfg: Config, params: Params, seed: int = 0) -> int:
        """Slot of the admitted instrument, or -SVPF_ERR_* (-7: does not fit the budget)."""
        slot = int(lib().svpf_stream_admit(self._s, int(n), C.byref(cfg), C.byref(params), int(seed)))
        if slot >= 0:
            self._cfg[slot] = Config.from_buffer_copy(cfg)
            self._n[slot] = int(n)
        return slot

    def evict(self, slot: int):
        rc = lib().svpf_stream_evict(self._s, int(slot))
        if rc != SVPF_OK:
            raise RuntimeError(f"evict failed rc={rc}")
        self._cfg.pop(slot, None)
        self._n.pop(slot, None)

    @property
    def bytes_in_use(self) -> int:
        return int(lib().svpf_stream_bytes_in_use(self._s))

    @property
    def bytes_budget(self) -> int:
        return int(lib().svpf_stream_bytes_budget(self._s))

    @property
    def kernel_launches(self) -> int:
        return int(lib().svpf_stream_kernel_launches(self._s))

    def process(self, slots, y):
        """Serve requests (slot, y) in order per instrument; returns Out[count]."""
        sl = np.ascontiguousarray(slots, dtype=np.int32)
        yy = _f32(y)
        out = (Out * max(len(sl), 1))()
        rc = lib().svpf_stream_process(self._s, len(sl), sl.ctypes.data_as(C.POINTER(_I)), _fp(yy), out)
        if rc != SVPF_OK:
            raise RuntimeError(f"svpf_stream_process rc={rc}: {ERRORS.get(rc, '?')}")
        return out

    def process_device(self, count1: int, count2: int, d_slots: int, d_y: int, d_out: int):
        rc = lib().svpf_stream_process_device(self._s, int(count1), int(count2), d_slots, d_y, d_out)
        if rc != SVPF_OK:
            raise RuntimeError(f"svpf_stream_process_device rc={rc}")

    def ctl(self, slot: int) -> Ctl:
        c = Ctl()
        rc = lib().svpf_stream_get_ctl(self._s, int(slot), C.byref(c))
        if rc != SVPF_OK:
            raise RuntimeError(f"get_ctl rc={rc}")
        return c

    def particles(self, slot: int) -> np.ndarray:
        m = 2 if self._cfg[slot].use_two_factor else 1
        out = np.empty(m * self._n[slot], np.float32)
        rc = lib().svpf_stream_get_particles(self._s, int(slot), _fp(out))
        if rc != SVPF_OK:
            raise RuntimeError(f"get_particles rc={rc}")
        return out


class MultiScale:
    """The reference's two-scale filter (REACTIVE + INERTIAL per instrument,
    include/svpf_multiscale.cuh) for F instruments on one batch
    (svpf_ms_batch_* in the C ABI)."""

    def __init__(self, base_params, config=None, stream=None):
        F = len(base_params)
        self._prms = (Params * F)(*base_params)
        cfg = config if config is not None else lib().svpf_ms_default_config()
        self.config = cfg
        self._m = lib().svpf_ms_batch_create(F, C.byref(cfg), self._prms, stream)
        if not self._m:
            raise RuntimeError("svpf_ms_batch_create failed")
        self.F = F

    def close(self):
        if getattr(self, "_m", None):
            lib().svpf_ms_batch_destroy(self._m)
            self._m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self, initial_vol: float, seed: int = 0):
        rc = lib().svpf_ms_batch_init(self._m, float(initial_vol), int(seed))
        if rc != SVPF_OK:
            raise RuntimeError(f"ms init rc={rc}")

    def step(self, y):
        yy = _f32(y)
        out = (MSOutput * self.F)()
        rc = lib().svpf_ms_batch_step(self._m, _fp(yy), out)
        if rc != SVPF_OK:
            raise RuntimeError(f"ms step rc={rc}")
        return out

    def inner_outputs(self):
        b = lib().svpf_ms_batch_inner(self._m)
        out = (Out * (2 * self.F))()
        lib().svpf_batch_last_outputs(b, out)
        return out

    def inner_config(self, f: int) -> Config:
        c = Config()
        lib().svpf_batch_get_config(lib().svpf_ms_batch_inner(self._m), int(f), C.byref(c))
        return c


class V2Rng(C.Structure):
    """svpf_v2_rng_t."""
    _fields_ = [("seed", C.c_ulonglong), ("tick", C.c_uint), ("filter", C.c_uint), ("status", _I),
                ("slots_n", _I), ("slots_u", _I), ("reserved", _I), ("tape_normals", C.c_void_p),
                ("tape_uniforms", C.c_void_p)]


# scalar arguments of svpf_fully_fused_step_v2 between the device outputs and
# the arrays' length, in order (include/svpf_fully_fused_v2.cuh:43-119)
V2_ARG_ORDER = ["rho", "sigma_z", "mu", "nu", "lik_offset", "student_t_const", "student_t_implied_offset",
                "gamma", "delta_rho", "delta_sigma", "mim_jump_prob", "mim_jump_scale", "guide_strength_base",
                "guide_strength_max", "guide_innovation_threshold", "guided_alpha_base", "guided_alpha_shock",
                "guided_innovation_thresh_predict", "use_guide", "use_guided_predict", "use_guide_preserving",
                "use_newton", "use_full_newton", "use_rejuvenation", "rejuv_ksd_threshold", "rejuv_prob",
                "rejuv_blend", "use_adaptive_mu", "@mu_state", "mu_ema_alpha", "use_adaptive_sigma",
                "sigma_boost_threshold", "sigma_boost_max", "step_size", "temperature", "rmsprop_rho",
                "rmsprop_eps", "n_stein_steps", "n_anneal_steps", "stein_sign_mode"]


class FusedV2:
    """svpf_fully_fused_step_v2 on device buffers owned by this object (torch
    tensors): arrays h, h_prev, grad, lw, v, inv_hess [n] and the device
    scalars.  A test-and-tooling wrapper around the C entry point."""

    ARRAYS = ("h", "h_prev", "grad", "lw", "v", "inv_hess")
    SCALARS = ("h_mean", "vol", "loglik", "bandwidth", "ksd", "guide_mean", "guide_var", "mu_state")

    def __init__(self, n: int, seed: int = 0, filter_id: int = 0):
        import torch
        self.torch = torch
        self.n = n
        self.arr = {a: torch.zeros(n, dtype=torch.float32, device="cuda") for a in self.ARRAYS}
        self.sc = torch.zeros(len(self.SCALARS), dtype=torch.float32, device="cuda")
        self._rng = lib().svpf_fully_fused_v2_rng_create(int(seed), int(filter_id))
        if not self._rng:
            raise RuntimeError("svpf_fully_fused_v2_rng_create failed")
        self._tape = None
        # the buffers never move (set() copies into them): their addresses
        # once, so that a call does no tensor work on the host
        base = self.sc.data_ptr()
        self._sp = [base + 4 * k for k in range(len(self.SCALARS))]
        self._arr_ptrs = [self.arr[a].data_ptr() for a in self.ARRAYS] + [self._rng]

    def close(self):
        if getattr(self, "_rng", None):
            lib().svpf_fully_fused_v2_rng_destroy(self._rng)
            self._rng = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set(self, name, values):
        if name in self.ARRAYS:
            self.arr[name].copy_(self.torch.as_tensor(np.asarray(values, np.float32)))
        else:
            self.sc[self.SCALARS.index(name)] = float(values)

    def get(self, name):
        self.torch.cuda.synchronize()
        if name in self.ARRAYS:
            return self.arr[name].cpu().numpy()
        return float(self.sc[self.SCALARS.index(name)].item())

    def rng_state(self) -> V2Rng:
        r = V2Rng()
        lib().svpf_fully_fused_v2_rng_get(self._rng, C.byref(r))
        return r

    def set_tape(self, normals=None, uniforms=None, tick=None):
        """Device noise tape [slots][n] (None: back to Philox)."""
        r = self.rng_state()
        if normals is None:
            self._tape = None
            r.tape_normals = r.tape_uniforms = None
            r.slots_n = r.slots_u = 0
        else:
            nrm = self.torch.as_tensor(np.ascontiguousarray(normals, np.float32)).cuda()
            uni = self.torch.as_tensor(np.ascontiguousarray(uniforms, np.float32)).cuda()
            self._tape = (nrm, uni)
            r.tape_normals, r.tape_uniforms = nrm.data_ptr(), uni.data_ptr()
            r.slots_n, r.slots_u = nrm.shape[0], uni.shape[0]
        if tick is not None:
            r.tick = tick
        lib().svpf_fully_fused_v2_rng_set(self._rng, C.byref(r))

    def step(self, params: dict, y_t, y_prev, h_mean_prev, vol_prev, ksd_prev, timestep, stream=None,
             sync: bool = True) -> int:
        """One call on `stream` (None: the legacy default stream); waits for
        the device unless sync is False, as the C entry point itself does not."""
        sp = self._sp
        scal = [sp[7] if k == "@mu_state" else params[k] for k in V2_ARG_ORDER]
        rc = lib().svpf_fully_fused_step_v2(
            *self._arr_ptrs, float(y_t), float(y_prev), float(h_mean_prev), float(vol_prev), float(ksd_prev),
            *sp[:7], *scal, self.n, int(timestep), stream)
        if sync:
            self.torch.cuda.synchronize()
        return int(rc)


class Estimator:
    """The reference's differentiable torch model (SVPFParamEstimator,
    py-torch/diff_svpf_torch.py:147-217) for F paths on the GPU
    (svpf_estimator_* in the C ABI): forward gives the predictive
    log-likelihood and volatility estimate of every tick, backward
    d(sum_t w_t loglik_t)/d(mu, rho, sigma_z, nu) by the CUDA adjoint."""

    def __init__(self, n_paths: int, n_particles: int = 64, n_stein_steps: int = 2, stein_lr: float = 0.1,
                 T_max: int = 1000, checkpoint_every: int = 64, truncate_every: int = 0, stream=None):
        self._e = lib().svpf_estimator_create(int(n_paths), int(n_particles), int(n_stein_steps), float(stein_lr),
                                              int(T_max), int(checkpoint_every), int(truncate_every), stream)
        if not self._e:
            raise RuntimeError("svpf_estimator_create failed (odd or too many particles, sizes, or device)")
        self.F = int(n_paths)
        self.n = int(n_particles)
        self.T_max = int(T_max)
        self.T = 0
        self.forward_id = 0

    def close(self):
        if getattr(self, "_e", None):
            lib().svpf_estimator_destroy(self._e)
            self._e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def tape_floats(n_particles: int, T: int) -> int:
        return int(lib().svpf_estimator_tape_floats(int(n_particles), int(T)))

    @staticmethod
    def make_tape(tape_init, tape_ticks) -> np.ndarray:
        """One path's tape from its initial normals [n] and per-tick halves [T, n/2]."""
        return np.concatenate([_f32(tape_init).ravel(), _f32(tape_ticks).ravel()])

    def _check(self, rc):
        if rc != SVPF_OK:
            raise RuntimeError(f"svpf estimator error {rc}: {ERRORS.get(rc, '?')}")

    def forward(self, theta, y, seed: int = 0, tape=None):
        """theta [F,4] = (mu, rho, sigma_z, nu), y [F,T]; tape [F, tape_floats]
        or None.  Returns (loglik [F,T], vol [F,T], loglik_sum [F])."""
        th = _f32(theta).reshape(self.F, 4)
        yy = _f32(y).reshape(self.F, -1)
        T = yy.shape[1]
        tp = None
        if tape is not None:
            tp = _f32(tape).reshape(self.F, self.tape_floats(self.n, T))
        ll = np.zeros((self.F, T), np.float32)
        vol = np.zeros((self.F, T), np.float32)
        ls = np.zeros(self.F, np.float64)
        self._check(lib().svpf_estimator_forward(self._e, _fp(th), _fp(yy), T, int(seed),
                                                 _fp(tp) if tp is not None else None, _fp(ll), _fp(vol),
                                                 ls.ctypes.data_as(C.POINTER(C.c_double))))
        self.T = T
        self.forward_id += 1
        return ll, vol, ls

    def backward(self, w=None):
        """grad [F,4] (float64) of sum_t w_t loglik_t; w [F,T] or None (ones)."""
        ww = None if w is None else _f32(w).reshape(self.F, self.T)
        g = np.zeros((self.F, 4), np.float64)
        self._check(lib().svpf_estimator_backward(self._e, _fp(ww) if ww is not None else None,
                                                  g.ctypes.data_as(C.POINTER(C.c_double))))
        return g

    def forward_device(self, d_theta: int, d_y: int, T: int, seed: int, d_tape, d_loglik: int, d_vol: int):
        self._check(lib().svpf_estimator_forward_device(self._e, d_theta, d_y, int(T), int(seed), d_tape, d_loglik,
                                                        d_vol))
        self.T = int(T)
        self.forward_id += 1

    def backward_device(self, d_w, d_grad: int):
        self._check(lib().svpf_estimator_backward_device(self._e, d_w, d_grad))

    def status(self) -> np.ndarray:
        """Per-path status of the last forward/backward."""
        st = np.zeros(self.F, np.int32)
        self._check(lib().svpf_estimator_get_status(self._e, st.ctypes.data_as(C.POINTER(_I))))
        return st


def autotune(ns, ticks: int = 2):
    arr = np.ascontiguousarray(sorted(set(int(n) for n in ns)), dtype=np.int32)
    rc = lib().svpf_autotune(arr.ctypes.data_as(C.POINTER(_I)), int(arr.shape[0]), int(ticks))
    if rc != SVPF_OK:
        raise RuntimeError(f"autotune failed: {ERRORS.get(rc, rc)}")
    out = {}
    for n in arr:
        r, s = C.c_int(), C.c_int()
        lib().svpf_tile_choice(int(n), C.byref(r), C.byref(s))
        out[int(n)] = (r.value, s.value)
    return out


def philox(k0: int, k1: int, counters: np.ndarray) -> np.ndarray:
    """Philox4x32-10 blocks computed on the GPU (for bit-exact checks)."""
    ctr = np.ascontiguousarray(counters, dtype=np.uint32).reshape(-1, 4)
    out = np.empty_like(ctr)
    rc = lib().svpf_debug_philox(k0, k1, ctr.ctypes.data_as(C.POINTER(C.c_uint32)),
                                 out.ctypes.data_as(C.POINTER(C.c_uint32)), ctr.shape[0])
    if rc != SVPF_OK:
        raise RuntimeError(f"philox failed: {ERRORS.get(rc, rc)}")
    return out


def pipe_rates() -> dict:
    """Measured MUFU and FP32 results per SM clock on the current device
    (svpf_measure_pipe_rates) and the pair-iteration peak they give."""
    mufu, fp32 = C.c_double(0.0), C.c_double(0.0)
    rc = lib().svpf_measure_pipe_rates(C.byref(mufu), C.byref(fp32))
    if rc != SVPF_OK:
        raise RuntimeError(f"svpf_measure_pipe_rates failed: {ERRORS.get(rc, rc)}")
    return {"mufu_per_clk_sm": mufu.value, "fp32_per_clk_sm": fp32.value,
            "pairs_per_clk_sm": min(mufu.value / 2.0, fp32.value / 13.0)}


def build_info() -> str:
    return lib().svpf_build_info().decode()
