"""The allocation-free batch tick, checked against the regular batch entry point.

svpf_batch_tick_noalloc exists for callers that cannot call cudaMalloc (an
application that owns all device memory in a fixed arena, a plugin inside
another framework's memory manager, a latency-critical loop that must not take
an allocation's implicit synchronisation): they pass every buffer, and the
kernel's scratch is a fixed array inside the library.  Here the same filters,
from the same state, are stepped twice in a row through both entry points
(svpf_batch_step_device on a regular batch, and svpf_batch_tick_noalloc on
caller-owned torch buffers); outputs and particles must agree within the
parity tolerance of the other GPU tests (1e-4 relative).  Filters whose
layout or configuration the launch was not sized for (n above n_max or below
1, an offset that is not a multiple of 16 floats, Heun without any_heun, two
factors) ride along in the same call: the device leaves them out with a
status in their control record and never touches their particles or outputs.
"""
import ctypes as C

import numpy as np
import pytest

from test_oracle import TOL, rel_err


def _bind(lib):
    vp = C.c_void_p
    lib.svpf_batch_tick_noalloc.restype = C.c_int
    lib.svpf_batch_tick_noalloc.argtypes = [C.c_int] + [vp] * 12 + [C.c_int, C.c_int, C.c_ulonglong, vp]
    lib.svpf_noalloc_max_filters.restype = C.c_int
    return lib


def _dev_bytes(torch, ctypes_array):
    raw = C.string_at(C.addressof(ctypes_array), C.sizeof(ctypes_array))
    return torch.frombuffer(bytearray(raw), dtype=torch.uint8).cuda()


@pytest.mark.gpu
def test_noalloc_tick_matches_batch_entry_point(pkg):
    import torch

    lib = _bind(pkg.lib())
    ns = [256, 512, 300, 1024, 2048, 64, 4096, 700]
    F = len(ns)
    n_max = max(ns)
    nus = np.linspace(5.0, 30.0, F)
    cfgs = (pkg.Config * F)(*[pkg.production_config(float(nus[f]), 8) for f in range(F)])
    prms = (pkg.Params * F)(*[pkg.Params(0.9 + 0.01 * f, 0.1 + 0.03 * f, -1.5 + 0.1 * f, 0.0) for f in range(F)])
    seed = 11

    # regular batch: the existing entry point
    batch = pkg.Batch(ns, list(cfgs), list(prms))
    batch.initialize(seed=seed)

    # caller-owned buffers for the allocation-free entry point, same state;
    # five filters the device must leave out follow the eight real ones
    # (n above n_max, n = 0, a misaligned offset, Heun without any_heun, two factors)
    bad_n = [n_max + 100, 0, 256, 256, 256]
    bad_status = [1, 1, 1, 1, 6]   # SVPF_ERR_INVALID_ARG, ..., SVPF_ERR_UNSUPPORTED
    Fb = F + len(bad_n)
    offs = np.zeros(Fb, np.int64)
    acc = 0
    for f, n in enumerate(ns + bad_n):
        offs[f] = acc
        acc += (max(n, 1) + 15) // 16 * 16 + 16
    offs[F + 2] += 3   # not a multiple of 16 floats
    h0 = np.full(acc, 7.0, np.float32)
    for f, n in enumerate(ns):
        h0[offs[f]:offs[f] + n] = batch.get_particles(f)
    cfg_bad = [pkg.production_config(30.0, 8) for _ in bad_n]
    cfg_bad[3].use_heun = 1
    cfg_bad[4].use_two_factor = 1
    cfgs_all = (pkg.Config * Fb)(*(list(cfgs) + cfg_bad))
    prms_all = (pkg.Params * Fb)(*(list(prms) + [pkg.Params(0.97, 0.15, -1.0, 0.0)] * len(bad_n)))
    ctl_all = (pkg.Ctl * Fb)(*(list(batch.ctl()) + [batch.ctl()[0]] * len(bad_n)))
    d_n = torch.tensor(ns + bad_n, dtype=torch.int32, device="cuda")
    d_off = torch.from_numpy(offs).cuda()
    d_cfg = _dev_bytes(torch, cfgs_all)
    d_prm = _dev_bytes(torch, prms_all)
    d_ctl = _dev_bytes(torch, ctl_all)
    d_h = torch.from_numpy(h0.copy()).cuda()
    d_hp = torch.from_numpy(h0.copy()).cuda()
    d_v = torch.zeros(acc, dtype=torch.float32, device="cuda")
    d_lw = torch.zeros(acc, dtype=torch.float32, device="cuda")
    d_out_a = torch.zeros((F, 8), dtype=torch.float32, device="cuda")
    d_out_b = torch.full((Fb, 8), 7.0, dtype=torch.float32, device="cuda")

    ys = np.array([[0.31, -0.8, 0.05, 1.9, -0.4, 0.2, -0.07, 0.6],
                   [-0.2, 0.5, -1.1, 0.3, 0.9, -0.6, 0.12, -0.3]], np.float32)
    y_prev = np.zeros(F, np.float32)
    for t in range(2):   # two calls in a row
        d_yt = torch.from_numpy(ys[t]).cuda()
        d_yp = torch.from_numpy(y_prev).cuda()
        d_yt_b = torch.from_numpy(np.concatenate([ys[t], np.full(len(bad_n), 0.1, np.float32)])).cuda()
        d_yp_b = torch.from_numpy(np.concatenate([y_prev, np.zeros(len(bad_n), np.float32)])).cuda()
        torch.cuda.synchronize()
        batch.step_device(d_yt.data_ptr(), d_yp.data_ptr(), d_out_a.data_ptr())
        batch.sync()
        rc = lib.svpf_batch_tick_noalloc(Fb, d_n.data_ptr(), d_off.data_ptr(), d_cfg.data_ptr(), d_prm.data_ptr(),
                                         d_ctl.data_ptr(), d_h.data_ptr(), d_hp.data_ptr(), d_v.data_ptr(),
                                         d_lw.data_ptr(), d_yt_b.data_ptr(), d_yp_b.data_ptr(), d_out_b.data_ptr(),
                                         n_max, 0, seed, None)
        assert rc == 0, rc
        torch.cuda.synchronize()
        out_a = d_out_a.cpu().numpy()
        out_all = d_out_b.cpu().numpy()
        out_b = out_all[:F]
        # the left-out filters: status set, nothing of theirs written
        ctl_b = (pkg.Ctl * Fb).from_buffer_copy(d_ctl.cpu().numpy().tobytes())
        assert [ctl_b[F + k].status for k in range(len(bad_n))] == bad_status, [c.status for c in ctl_b]
        assert all(ctl_b[f].status == 0 for f in range(F))
        assert (out_all[F:] == 7.0).all()
        h_all = d_h.cpu().numpy()
        for k in range(len(bad_n)):
            seg = h_all[offs[F + k]:offs[F + k] + max(bad_n[k], 1)]
            assert (seg == 7.0).all(), k
        steps_a = out_a.view(np.int32)[:, 6]
        steps_b = out_b.view(np.int32)[:, 6]
        assert np.array_equal(steps_a, steps_b), (t, steps_a, steps_b)
        for col in (0, 1, 2):   # loglik, vol, h_mean
            assert rel_err(out_b[:, col], out_a[:, col]) < TOL, (t, col, out_a[:, col], out_b[:, col])
        h_b = d_h.cpu().numpy()
        for f, n in enumerate(ns):
            assert rel_err(h_b[offs[f]:offs[f] + n], batch.get_particles(f)) < TOL, (t, f)
        y_prev = ys[t]
    batch.close()


def test_noalloc_rejects_bad_arguments_on_the_host(pkg):
    """Argument errors the host can see are returned before any device work
    (so these run without a GPU)."""
    lib = _bind(pkg.lib())
    fake = [C.c_void_p(16 * (k + 1)) for k in range(12)]   # never dereferenced: the call returns first
    too_many = lib.svpf_noalloc_max_filters() + 1
    assert lib.svpf_batch_tick_noalloc(too_many, *fake, 256, 0, 0, None) == 1   # SVPF_ERR_INVALID_ARG
    assert lib.svpf_batch_tick_noalloc(0, *fake, 256, 0, 0, None) == 1
    assert lib.svpf_batch_tick_noalloc(4, *fake, 0, 0, 0, None) == 1              # n_max = 0
    assert lib.svpf_batch_tick_noalloc(4, *fake, 8192 + 1, 0, 0, None) == 1       # n_max > SVPF_MAX_PARTICLES
    no_h = list(fake)
    no_h[6] = None                                                                 # d_h
    assert lib.svpf_batch_tick_noalloc(4, *no_h, 256, 0, 0, None) == 1


@pytest.mark.gpu
def test_noalloc_tick_on_two_devices_in_one_process(pkg):
    """The scratch array and the kernels' shared-memory opt-in exist per
    device: the same call on two GPUs of one process gives the same results
    (skipped with fewer than two GPUs)."""
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    lib = _bind(pkg.lib())
    ns = [512, 4096, 256]
    F = len(ns)
    cfgs = (pkg.Config * F)(*[pkg.production_config(10.0, 8) for _ in range(F)])
    prms = (pkg.Params * F)(*[pkg.Params(0.97, 0.15, -1.0, 0.0) for _ in range(F)])
    offs = np.cumsum([0] + [(n + 15) // 16 * 16 for n in ns[:-1]]).astype(np.int64)
    total = int(offs[-1] + (ns[-1] + 15) // 16 * 16)
    h0 = (-1.0 + 0.3 * np.random.default_rng(1).standard_normal(total)).astype(np.float32)
    ctl0 = pkg.Batch([64], pkg.production_config(10.0, 8), pkg.Params(0.97, 0.15, -1.0, 0.0)).ctl()[0]
    results = []
    for dev in (0, 1):
        with torch.cuda.device(dev):
            d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda(dev)  # noqa: E731
            d_ctl = _dev_bytes(torch, (pkg.Ctl * F)(*([ctl0] * F))).cuda(dev)
            bufs = [d(np.array(ns, np.int32)), d(offs), _dev_bytes(torch, cfgs).cuda(dev),
                    _dev_bytes(torch, prms).cuda(dev), d_ctl, d(h0), d(h0), d(np.zeros(total, np.float32)),
                    d(np.zeros(total, np.float32)), d(np.full(F, 0.3, np.float32)), d(np.zeros(F, np.float32))]
            d_out = torch.zeros((F, 8), dtype=torch.float32, device=f"cuda:{dev}")
            rc = lib.svpf_batch_tick_noalloc(F, *[b.data_ptr() for b in bufs], d_out.data_ptr(), max(ns), 0, 5,
                                             None)
            assert rc == 0, (dev, rc)
            torch.cuda.synchronize(dev)
            results.append(d_out.cpu().numpy())
    assert np.isfinite(results[0]).all() and np.array_equal(results[0], results[1])
