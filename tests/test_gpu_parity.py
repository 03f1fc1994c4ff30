"""Per-tick parity of the CUDA engine (through the C ABI) with the reference's
own CUDA step (golden fixtures) and with the FP64 oracle, with state re-sync:
both sides start each tick from the same state and draw the same noise tape.
Tolerance: 1e-4 relative (floor 1 on the denominator)."""
import numpy as np
import pytest

import cases
import tape
from test_oracle import TOL, TWO_FACTOR_SCALARS, _fixtures, ctl_mismatches, load_fixture, rel_err

pytestmark = pytest.mark.gpu

SCALARS = ("ksd_prev", "bw", "bw_sq", "return_ema", "return_var", "h_mean_prev", "vol_prev", "mu_state")


def to_ctl(pkg, d):
    c = pkg.Ctl()
    for k, _ in c._fields_:
        if k not in d:
            continue
        if k in ("smooth_h_mean", "smooth_h_var", "smooth_y"):
            arr = getattr(c, k)
            for i, v in enumerate(d[k]):
                arr[i] = v
        else:
            setattr(c, k, type(getattr(c, k))(d[k]))
    return c


def engine_for(pkg, n, n_stein, nu, cfg_dict, params, cluster=0):
    f = pkg.SVPF(n, n_stein, nu)
    f.configure(**cfg_dict)
    f.params = pkg.Params(*[float(x) for x in params])
    if cluster:
        f.set_cluster_size(cluster)
    f._initialized = True
    return f


@pytest.mark.parametrize("cluster", [0, 1])
@pytest.mark.parametrize("path", _fixtures(), ids=lambda p: p.split("/")[-1][:-4])
def test_engine_matches_reference_ticks(pkg, path, cluster):
    fx = load_fixture(path)
    n = fx["n"]
    tf = bool(fx["config"].get("use_two_factor", 0))
    f = engine_for(pkg, n, fx["config"]["n_stein_steps"], fx["config"]["nu"], fx["config"], fx["params"], cluster)
    y_prev = 0.0
    for t in range(fx["outs"].shape[0]):
        if tf:
            # two factors: h, h_prev, v hold [fast; slow]; the log-weights are [n]
            f.set_state(to_ctl(pkg, fx["ctl"][t]), None, None, None, fx["lw"][t])
            f.set_state_2f(fx["h"][t], fx["hp"][t], fx["v"][t])
        else:
            f.set_state(to_ctl(pkg, fx["ctl"][t]), fx["h"][t], fx["hp"][t], fx["v"][t], fx["lw"][t])
        nrm, uni = tape.tape(fx["tape_seed"], t, n, fx["normal_slots"], 2)
        f.set_noise_tape(nrm, uni)
        rc, out = f.step_raw(fx["ys"][t], y_prev)
        y_prev = float(fx["ys"][t])
        assert rc == 0, (t, rc)
        ctl, h, hp, v, lw = f.get_state()
        if tf:
            h, hp, v = f.get_state_2f()
        post = fx["ctl"][t + 1]
        if not tf:
            assert out.steps_used == post["stein_steps_used"]
        assert rel_err(h, fx["h"][t + 1]) < TOL, (t, rel_err(h, fx["h"][t + 1]))
        assert rel_err(hp, fx["hp"][t + 1]) < TOL
        assert rel_err(v, fx["v"][t + 1], floor=1e-3) < 10 * TOL, (t, rel_err(v, fx["v"][t + 1], 1e-3))
        assert rel_err(lw, fx["lw"][t + 1]) < TOL, (t, rel_err(lw, fx["lw"][t + 1]))
        ll, vol, hm = fx["outs"][t]
        assert abs(out.loglik - ll) < TOL * max(1, abs(ll)), (t, out.loglik, ll)
        assert abs(out.vol - vol) < TOL * max(1, abs(vol)), (t, out.vol, vol)
        assert abs(out.h_mean - hm) < TOL * max(1, abs(hm)), (t, out.h_mean, hm)
        for k in SCALARS + (TWO_FACTOR_SCALARS if tf else ()):
            a, b = getattr(ctl, k), post[k]
            assert abs(a - b) <= TOL * max(1.0, abs(b)), (t, k, a, b)
    f.close()


@pytest.mark.parametrize("path", _fixtures(), ids=lambda p: p.split("/")[-1][:-4])
def test_engine_initialize_matches_reference(pkg, path):
    """svpf_initialize on the engine (svpf_optimized_graph.cu:349-451 and the
    backend quirks at :483-494: stationary draw, reset control record,
    previous mean -3.5): from the fixture's initial-draw tape the engine lands
    on the reference's recorded post-initialise state (fixture tick 0) --
    particles, previous particles, RMSProp moments, log-weights and every
    recorded control field."""
    fx = load_fixture(path)
    n = fx["n"]
    cfg = fx["config"]
    tf = bool(cfg.get("use_two_factor", 0))
    f = pkg.SVPF(n, cfg["n_stein_steps"], cfg["nu"])
    f.configure(**cfg)
    f.set_noise_tape(tape.init_normals(fx["tape_seed"], n, 3 if tf else 1).reshape(-1, n),
                     np.ones((1, n), np.float32))
    # the C entry point itself (the pybind-style initialize() also resets mu_var as pysvpf does)
    import ctypes as C
    f.params = pkg.Params(*[float(x) for x in fx["params"]])
    pkg.lib().svpf_initialize(f._s, C.byref(f.params), 1)
    assert f.last_error() == 0
    ctl, h, hp, v, lw = f.get_state()
    if tf:
        h, hp, v = f.get_state_2f()
    assert rel_err(h, fx["h"][0]) < TOL, rel_err(h, fx["h"][0])
    assert rel_err(hp, fx["hp"][0]) < TOL
    assert np.array_equal(v, fx["v"][0]) and np.array_equal(lw, fx["lw"][0])
    bad = ctl_mismatches(ctl, fx["ctl"][0])
    assert not bad, bad
    f.close()


def oracle_twin(oracle_mod, pkg, f, params):
    o = oracle_mod.OracleFilter(f.n_particles, oracle_mod.config_from_dict(f.config.to_dict()),
                                oracle_mod.OracleParams(*params))
    ctl, h, hp, v, lw = f.get_state()
    o.ctl = oracle_mod.ctl_from_dict({k: getattr(ctl, k) for k, _ in ctl._fields_})   # smoother included
    o.h, o.h_prev, o.v, o.log_w = (a.astype(np.float64) for a in (h, hp, v, lw))
    return o


CONFIGS = {
    "production": cases.PRODUCTION,
    "pybind": cases.PYBIND,
    "vanilla": dict(use_newton=0, stein_min_steps=3, stein_max_steps=5),
    "newton": dict(use_newton=1, use_full_newton=0, stein_min_steps=3, stein_max_steps=5),
    "student_state": dict(use_student_t_state=1, nu_state=5.0, use_newton=1, use_full_newton=1,
                          stein_min_steps=2, stein_max_steps=4),
    "heun": dict(use_heun=1, use_newton=1, use_full_newton=1, stein_min_steps=2, stein_max_steps=4),
}


@pytest.mark.parametrize("n,cluster", [(1, 1), (2, 1), (31, 1), (33, 2), (255, 4), (257, 8), (512, 0),
                                       (1000, 16), (2048, 0), (4096, 16), (4096, 1)])
@pytest.mark.parametrize("cfg_name", ["production", "vanilla", "newton"])
def test_engine_matches_oracle_sizes(pkg, oracle_mod, n, cluster, cfg_name):
    """Edge sizes (1, 2, odd, around warp and tile boundaries, the maximum of
    the configs) and cluster shapes, 3 ticks each from a re-synced state."""
    params = (0.97, 0.15, -1.0, -0.1)
    f = engine_for(pkg, n, 8, 30.0, {}, params, cluster)
    f.configure(**{k: getattr(pkg.default_config(8, 30.0), k) for k, _ in pkg.CONFIG_FIELDS})
    f.configure(**CONFIGS[cfg_name])
    f.set_noise_tape(tape.init_normals(11, n)[None, :], np.ones((1, n), np.float32))
    f.initialize(*params, seed=5)
    _, ys = tape.sv_path(4, -1.0, 0.97, 0.15, seed=n)
    y_prev = 0.0
    slots = 2 + f.config.stein_max_steps + 7
    for t in range(3):
        o = oracle_twin(oracle_mod, pkg, f, params)
        nrm, uni = tape.tape(99, t, n, slots, 2)
        f.set_noise_tape(nrm, uni)
        rc, out = f.step_raw(ys[t], y_prev)
        assert rc == 0
        oo = o.step(ys[t], y_prev, nrm, uni)
        y_prev = float(ys[t])
        h = f.get_particles()
        assert out.steps_used == oo.steps_used
        assert rel_err(h, o.h) < TOL, (t, rel_err(h, o.h))
        assert abs(out.loglik - oo.loglik) < TOL * max(1, abs(oo.loglik)), (t, out.loglik, oo.loglik)
        assert abs(out.ksd - oo.ksd) < 1e-3 * max(1, abs(oo.ksd)), (t, out.ksd, oo.ksd)
    f.close()


@pytest.mark.parametrize("cfg_name", sorted(CONFIGS))
def test_engine_matches_oracle_configs(pkg, oracle_mod, cfg_name):
    """Every configuration family over 12 ticks (crosses t = 10, where the
    KSD-driven budget and rejuvenation switch on), state re-synced each tick."""
    n = 384
    params = (0.96, 0.2, -1.2, -0.2)
    f = engine_for(pkg, n, 8, 12.0, {}, params)
    f.configure(**{k: getattr(pkg.default_config(8, 12.0), k) for k, _ in pkg.CONFIG_FIELDS})
    f.configure(**CONFIGS[cfg_name])
    f.set_noise_tape(tape.init_normals(3, n)[None, :], np.ones((1, n), np.float32))
    f.initialize(*params, seed=1)
    _, ys = tape.sv_path(13, -1.2, 0.96, 0.2, seed=17)
    y_prev = 0.0
    slots = 2 + max(f.config.stein_max_steps, 16) + 7
    for t in range(12):
        o = oracle_twin(oracle_mod, pkg, f, params)
        nrm, uni = tape.tape(5, t, n, slots, 2)
        f.set_noise_tape(nrm, uni)
        rc, out = f.step_raw(ys[t], y_prev)
        assert rc == 0
        oo = o.step(ys[t], y_prev, nrm, uni)
        y_prev = float(ys[t])
        h = f.get_particles()
        assert out.steps_used == oo.steps_used, t
        assert out.rejuv_fired == oo.rejuv_fired, t
        assert rel_err(h, o.h) < TOL, (t, rel_err(h, o.h))
        assert abs(out.loglik - oo.loglik) < TOL * max(1, abs(oo.loglik))
        assert abs(out.h_mean - oo.h_mean) < TOL * max(1, abs(oo.h_mean))
    f.close()


def test_philox_bit_exact(pkg, oracle_mod):
    rng = np.random.default_rng(0)
    ctr = rng.integers(0, 2 ** 32, size=(4096, 4), dtype=np.uint64).astype(np.uint32)
    k0, k1 = 0x12345678, 0x9ABCDEF0
    gpu = pkg.philox(k0, k1, ctr)
    cpu = np.array([oracle_mod.philox(k0, k1, *map(int, c)) for c in ctr[:512]], np.uint32)
    assert np.array_equal(gpu[:512], cpu)
    from test_oracle import PHILOX_KAT
    for c, k, o in PHILOX_KAT:
        assert list(pkg.philox(k[0], k[1], np.array([c], np.uint32))[0]) == list(o)


def test_batch_matches_single_filters(pkg):
    """The persistent batch kernel and the single-filter cluster kernel give the
    same tick for the same filter state and tape (mixed particle counts)."""
    ns = [256, 300, 512, 1024, 64, 2048]
    params = [pkg.Params(0.97, 0.15, -1.0, 0.0), pkg.Params(0.95, 0.3, -0.5, 0.0)]
    cfg = pkg.default_config(8, 30.0)
    cfg.update(**cases.PRODUCTION)
    b = pkg.Batch(ns, cfg, [params[i % 2] for i in range(len(ns))])
    n_max = max(ns)
    init = tape.init_normals(21, n_max)
    b.set_noise_tape(init[None, :], np.ones((1, n_max), np.float32))
    b.initialize(seed=3)
    slots = 12
    nrm, uni = tape.tape(8, 0, n_max, slots, 2)
    singles = []
    for i, n in enumerate(ns):
        f = pkg.SVPF(n, 8, 30.0)
        f.configure(**cfg.to_dict())
        f.params = params[i % 2]
        f._initialized = True
        f.set_noise_tape(init[None, :n], np.ones((1, n), np.float32))
        f.initialize(params[i % 2].rho, params[i % 2].sigma_z, params[i % 2].mu, params[i % 2].gamma, seed=3)
        singles.append(f)
    ys = np.linspace(-0.5, 0.6, len(ns)).astype(np.float32)
    b.set_noise_tape(nrm, uni)
    ll, vol, hm = b.step(ys, np.zeros(len(ns), np.float32))
    for i, (n, f) in enumerate(zip(ns, singles)):
        f.set_noise_tape(np.ascontiguousarray(nrm[:, :n]), np.ascontiguousarray(uni[:, :n]))
        rc, out = f.step_raw(ys[i], 0.0)
        assert rc == 0
        assert rel_err(b.get_particles(i), f.get_particles()) < TOL, (n, rel_err(b.get_particles(i), f.get_particles()))
        assert abs(ll[i] - out.loglik) < TOL * max(1, abs(out.loglik))
        assert abs(hm[i] - out.h_mean) < TOL * max(1, abs(out.h_mean))
        f.close()
    b.close()


def test_status_codes_and_bad_arguments(pkg):
    assert not pkg.lib().svpf_create(0, 8, 30.0, None)
    assert not pkg.lib().svpf_create(100000, 8, 30.0, None)
    f = pkg.SVPF(256, 8, 30.0)
    f.initialize(0.97, 0.15, -1.0, 0.0, seed=1)
    rc, out = f.step_raw(float("nan"), 0.0)
    assert rc == 5   # SVPF_ERR_NONFINITE, reported without faulting
    f.initialize(0.97, 0.15, -1.0, 0.0, seed=1)
    f.set_noise_tape(np.zeros((1, 256), np.float32), np.full((1, 256), 0.5, np.float32))
    rc, _ = f.step_raw(0.1, 0.0)
    assert rc == 4   # SVPF_ERR_TAPE_SHORT: tape has one slot, the tick needs more
    f.set_noise_tape(None)
    rc, _ = f.step_raw(0.1, 0.0)
    assert rc == 0
    f.close()



def test_step_entry_points_agree(pkg):
    """svpf_step_optimized and svpf_step_adaptive (declared by the reference's
    svpf.cuh) tick exactly as svpf_step_graph: three filters from one seed,
    one per entry point, bit-identical outputs over 20 ticks."""
    import ctypes as C

    L = pkg.lib()
    _, ys = tape.sv_path(20, -1.0, 0.97, 0.15, seed=5)
    fs = [pkg.SVPF(512, 8, 30.0) for _ in range(3)]
    for f in fs:
        f.configure(**pkg.production_config(30.0, 8).to_dict())
        f.initialize(0.97, 0.15, -1.0, 0.0, seed=7)
    out = np.zeros((3, 20, 3), np.float32)
    yp = 0.0
    for t in range(20):
        vals = [[C.c_float() for _ in range(3)] for _ in range(3)]
        L.svpf_step_graph(fs[0]._s, float(ys[t]), yp, C.byref(fs[0].params), *[C.byref(v) for v in vals[0]])
        L.svpf_step_adaptive(fs[1]._s, float(ys[t]), yp, C.byref(fs[1].params), *[C.byref(v) for v in vals[1]])
        L.svpf_step_optimized(fs[2]._s, float(ys[t]), yp, C.byref(fs[2].params), C.byref(vals[2][0]),
                              C.byref(vals[2][1]))
        vals[2][2].value = fs[2].last_output().h_mean
        for k in range(3):
            out[k, t] = [v.value for v in vals[k]]
            assert L.svpf_last_error(fs[k]._s) == 0
        yp = float(ys[t])
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])
    for f in fs:
        f.close()
