"""Parity cases: configuration overrides on top of the reference's svpf_create
defaults (svpf_optimized_graph.cu:116-283), model parameters and sizes.

Each case is run tick by tick on the reference's own CUDA step with a noise
tape (make_golden.py, GPU) and stored as a fixture; the oracle and the product
engine replay every tick from the stored pre-tick state with the same tape.
"""
import tape

# The plain single-filter workload on the reference knobs: N=512, at most 8
# Newton-Stein iterations over 3 annealing stages, full Newton, SVLD, MIM,
# asymmetric rho, preserving EKF guide, rejuvenation, Student-t nu = 30.
PRODUCTION = dict(use_newton=1, use_full_newton=1, stein_min_steps=4, stein_max_steps=8,
                  n_anneal_steps=3)

# The pybind production defaults (py-torch/svpf_python.cpp:90-176).
PYBIND = dict(lik_offset=0.345, use_asymmetric_rho=1, rho_up=0.98, rho_down=0.93, use_svld=1,
              temperature=0.45, rmsprop_rho=0.9, rmsprop_eps=1e-6, use_annealing=1,
              n_anneal_steps=5, use_mim=1, mim_jump_prob=0.25, mim_jump_scale=9.0,
              use_adaptive_beta=1, use_rejuvenation=1, rejuv_ksd_threshold=0.05,
              rejuv_prob=0.30, rejuv_blend=0.30, use_newton=1, use_full_newton=1,
              use_exact_gradient=1, stein_min_steps=8, stein_max_steps=16,
              use_guided=1, guided_alpha_base=0.0, guided_alpha_shock=0.40,
              guided_innovation_threshold=1.5, use_guide=1, use_guide_preserving=1,
              guide_strength=0.05, use_adaptive_guide=1, guide_strength_base=0.05,
              guide_strength_max=0.30, guide_innovation_threshold=1.0, use_adaptive_mu=1,
              mu_process_var=0.001, mu_obs_var_scale=11.0, mu_min=-4.0, mu_max=-1.0,
              use_adaptive_sigma=1, sigma_boost_threshold=0.95, sigma_boost_max=3.2,
              use_local_params=0, delta_rho=0.0, delta_sigma=0.0)

CASES = {
    "production_n512": dict(n=512, n_stein=8, nu=30.0, cfg=PRODUCTION,
                            params=(0.97, 0.15, -1.0, 0.0), path=(-1.0, 0.97, 0.15), ticks=14),
    "pybind_n256": dict(n=256, n_stein=8, nu=30.0, cfg=PYBIND,
                        params=(0.97, 0.15, -3.5, -0.5), path=(-3.5, 0.97, 0.25), ticks=14),
    "vanilla_paper_n300": dict(n=300, n_stein=6, nu=5.0,
                               cfg=dict(use_newton=0, use_adaptive_beta=0, use_guide_preserving=0,
                                        stein_repulsive_sign=1, stein_min_steps=3, stein_max_steps=7,
                                        rejuv_ksd_threshold=0.05),
                               params=(0.95, 0.2, -2.0, -0.2), path=(-2.0, 0.95, 0.2), ticks=14),
    "newton_local_n256": dict(n=256, n_stein=8, nu=8.0,
                              cfg=dict(use_newton=1, use_full_newton=0, use_local_params=1,
                                       use_exact_gradient=1, lik_offset=0.27, stein_min_steps=4,
                                       stein_max_steps=9, use_adaptive_sigma=1),
                              params=(0.98, 0.12, -1.5, 0.0), path=(-1.5, 0.98, 0.12), ticks=14),
    "student_t_state_n200": dict(n=200, n_stein=6, nu=6.0,
                                 cfg=dict(use_student_t_state=1, nu_state=5.0, use_newton=1,
                                          use_full_newton=1, stein_min_steps=4, stein_max_steps=6,
                                          use_guided=1),
                                 params=(0.96, 0.18, -1.0, 0.0), path=(-1.0, 0.96, 0.18), ticks=14),
    "heun_n256": dict(n=256, n_stein=6, nu=30.0,
                      cfg=dict(use_heun=1, use_newton=1, use_full_newton=1, stein_min_steps=3,
                               stein_max_steps=6),
                      params=(0.97, 0.15, -1.0, 0.0), path=(-1.0, 0.97, 0.15), ticks=14),
    "fan_smooth_n128": dict(n=128, n_stein=5, nu=10.0,
                            cfg=dict(use_fan_mode=1, stein_repulsive_sign=1, use_annealing=0,
                                     use_smoothing=1, smooth_lag=4, smooth_output_lag=1,
                                     use_adaptive_mu=1, mu_min=-3.0, mu_max=0.0,
                                     stein_min_steps=2, stein_max_steps=5, use_guide=1),
                            params=(0.97, 0.15, -1.0, 0.0), path=(-1.0, 0.97, 0.15), ticks=14),
}

# Two-factor cases.  TWO_FACTOR_TEST is the reference's two-factor test setup
# (test/test_two_factor.cu:199-280: the production single-factor knobs, then
# guide strength 0.12 and the factor parameters of its "balanced" process).
TWO_FACTOR_TEST = dict(use_two_factor=1, rho_fast=0.90, sigma_fast=0.15, rho_slow=0.99, sigma_slow=0.05,
                       bw_floor_fast=0.01, bw_floor_slow=0.05, use_svld=1, use_annealing=1,
                       n_anneal_steps=5, temperature=0.45, use_mim=1, mim_jump_prob=0.25,
                       mim_jump_scale=9.0, use_guide=1, use_guide_preserving=1, guide_strength=0.12,
                       use_exact_gradient=1, lik_offset=0.345)

CASES.update({
    "two_factor_n512": dict(n=512, n_stein=8, nu=7.0, cfg=TWO_FACTOR_TEST,
                            params=(0.99, 0.05, -3.5, 0.0), path=("2f", -3.5, 0.90, 0.15, 0.99, 0.05, 7.0),
                            ticks=12),
    # factor parameters of the reference test's "slow dominant" process.  (Its
    # "fast dominant" process, sigma_slow = 0.02, makes the first tick after
    # initialisation chaotic in FP32: with the RMSProp moments at zero the
    # slow factor's stiff prior moves particles by several bandwidths per
    # step, and the FP32 and FP64 oracles already differ by 2.7e-4 there.)
    "two_factor_plain_n256": dict(n=256, n_stein=6, nu=30.0,
                                  cfg=dict(use_two_factor=1, use_svld=0, use_mim=0, use_guide=0,
                                           use_annealing=0, use_exact_gradient=0, stein_repulsive_sign=1,
                                           rho_fast=0.95, sigma_fast=0.08, rho_slow=0.98, sigma_slow=0.12),
                                  params=(0.98, 0.12, -3.5, 0.0),
                                  path=("2f", -3.5, 0.95, 0.08, 0.98, 0.12, 0.0), ticks=12),
    "two_factor_blend_n300": dict(n=300, n_stein=4, nu=5.0,
                                  cfg=dict(use_two_factor=1, use_guide=1, use_guide_preserving=0,
                                           guide_strength=0.2, n_anneal_steps=3, use_svld=1, temperature=0.6,
                                           use_mim=1, rho_fast=0.92, sigma_fast=0.20, rho_slow=0.995,
                                           sigma_slow=0.08, bw_floor_slow=0.1),
                                  params=(0.995, 0.08, -3.0, 0.0),
                                  path=("2f", -3.0, 0.92, 0.20, 0.995, 0.08, 5.0), ticks=12),
})

TAPE_SEED = 20240601


def is_two_factor(case) -> bool:
    return bool(case["cfg"].get("use_two_factor", 0))


def init_slots(case) -> int:
    """Initial draws per particle: the single-factor draw, plus fast and slow."""
    return 3 if is_two_factor(case) else 1


def observations(case, T: int, seed: int):
    """(h, y) of the case's synthetic path, T ticks."""
    path = case["path"]
    if path[0] == "2f":
        return tape.sv2_path(T, *path[1:6], seed=seed, nu_obs=path[6])
    return tape.sv_path(T, *path, seed=seed)


def normal_slots(case) -> int:
    """Upper bound on normal draws per particle per tick for the case."""
    cfg = case["cfg"]
    if is_two_factor(case):
        na = cfg.get("n_anneal_steps", 3) if cfg.get("use_annealing", 1) else 1
        return 2 + 2 * na * case["n_stein"]
    max_steps = cfg.get("stein_max_steps", 12)
    pred = 1
    if cfg.get("use_student_t_state", 0) and cfg.get("nu_state", 5.0) <= 30.0:
        pred = 1 + max(int(cfg.get("nu_state", 5.0) + 0.5), 3)
    return pred + max_steps + 1


# ---- svpf_fully_fused_step_v2 cases (include/svpf_fully_fused_v2.cuh:43-119) ----
# V2_REFERENCE_TEST is the parameter set of the reference's own v2 test
# (test/test_fully_fused_v2.cu:60-110), with nu = 5 and its constants.
V2_REFERENCE_TEST = dict(rho=0.98, sigma_z=0.10, mu=-4.5, nu=5.0, lik_offset=0.345, gamma=0.0, delta_rho=0.0,
                         delta_sigma=0.0, mim_jump_prob=0.25, mim_jump_scale=9.0, guide_strength_base=0.05,
                         guide_strength_max=0.30, guide_innovation_threshold=1.0, guided_alpha_base=0.0,
                         guided_alpha_shock=0.40, guided_innovation_thresh_predict=1.5, use_guide=1,
                         use_guided_predict=1, use_guide_preserving=1, use_newton=1, use_full_newton=1,
                         use_rejuvenation=1, rejuv_ksd_threshold=0.05, rejuv_prob=0.30, rejuv_blend=0.30,
                         use_adaptive_mu=0, mu_ema_alpha=0.01, use_adaptive_sigma=1, sigma_boost_threshold=0.95,
                         sigma_boost_max=3.2, step_size=0.25, temperature=0.45, rmsprop_rho=0.9, rmsprop_eps=1e-6,
                         n_stein_steps=10, n_anneal_steps=5, stein_sign_mode=0)

V2_CASES = {
    "v2_reference_test_n512": dict(n=512, p=V2_REFERENCE_TEST, path=(-4.5, 0.98, 0.10), ticks=14),
    "v2_vanilla_local_n256": dict(n=256, p=dict(V2_REFERENCE_TEST, use_newton=0, use_full_newton=0,
                                                use_guided_predict=0, use_rejuvenation=0, temperature=0.0,
                                                use_adaptive_mu=1, mu_ema_alpha=0.05, delta_rho=0.02,
                                                delta_sigma=0.1, gamma=-0.3, stein_sign_mode=1, n_stein_steps=6,
                                                n_anneal_steps=2, mu=-1.0, rho=0.97, sigma_z=0.15, nu=12.0,
                                                step_size=0.1),
                                  path=(-1.0, 0.97, 0.15), ticks=14),
    "v2_newton_blend_n300": dict(n=300, p=dict(V2_REFERENCE_TEST, use_newton=1, use_full_newton=0,
                                               use_guide_preserving=0, rejuv_ksd_threshold=0.0, n_stein_steps=7,
                                               n_anneal_steps=3, mu=-2.0, rho=0.95, sigma_z=0.2, nu=8.0),
                                 path=(-2.0, 0.95, 0.2), ticks=14),
    "v2_full_newton_noguide_n128": dict(n=128, p=dict(V2_REFERENCE_TEST, use_newton=0, use_full_newton=1,
                                                      use_guide=0, temperature=1.0, n_stein_steps=5,
                                                      n_anneal_steps=1, mu=-1.5, rho=0.97, sigma_z=0.15, nu=30.0),
                                        path=(-1.5, 0.97, 0.15), ticks=14),
}


def v2_normal_slots(case) -> int:
    """curand_normal4 (4) + one refresh per Stein step + the rejuvenation normal."""
    return 4 + max(case["p"]["n_stein_steps"], 1) + 1
