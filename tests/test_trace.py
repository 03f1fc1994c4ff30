"""Tracing: the library's host entry points open NVTX ranges named after
themselves, so a profiler files each kernel under the C call that issued it.

A minimal NVTX tool (tests/nvtx_probe.c, loaded through
NVTX_INJECTION64_PATH in a child process) records the ranges.  The calls
below return before any device work (invalid arguments), so the test runs
without a GPU; the range is opened before the arguments are checked.
"""
import os
import shutil
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(ROOT, "newton-stein-variational-particle-filter_b200", "libsvpf_b200.so")

CHILD = r"""
import ctypes as C, sys
lib = C.CDLL(sys.argv[1])
probe = C.CDLL(sys.argv[2])
probe.probe_name.restype = C.c_char_p
vp = C.c_void_p
lib.svpf_batch_create.restype = vp
lib.svpf_batch_create.argtypes = [C.c_int, vp, vp, vp, vp]
assert not lib.svpf_batch_create(0, None, None, None, None)
lib.svpf_batch_tick_noalloc.argtypes = [C.c_int] + [vp] * 12 + [C.c_int, C.c_int, C.c_ulonglong, vp]
assert lib.svpf_batch_tick_noalloc(0, *([None] * 12), 256, 0, 0, None) == 1
lib.svpf_step_adaptive.argtypes = [vp, C.c_float, C.c_float, vp, vp, vp, vp]
lib.svpf_step_adaptive(None, 0.0, 0.0, None, None, None, None)   # nests svpf_step_graph
lib.svpf_grad_forward.argtypes = [vp, vp, vp, vp, C.c_int, C.c_ulonglong, vp, vp]
assert lib.svpf_grad_forward(None, None, None, None, 0, 0, None, None) != 0
names = [probe.probe_name(i).decode() for i in range(probe.probe_count())]
print(",".join(names))
print(probe.probe_depth(), probe.probe_max_depth())
"""


def _cc():
    return shutil.which("gcc") or shutil.which("cc")


def _cuda_include():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nvcc))), "include")
    return inc if os.path.isdir(os.path.join(inc, "nvtx3")) else None


@pytest.mark.skipif(not os.path.exists(LIB), reason="libsvpf_b200.so not built")
def test_entry_points_open_named_nvtx_ranges(tmp_path):
    cc, inc = _cc(), _cuda_include()
    if cc is None or inc is None:
        pytest.skip("no host compiler or NVTX headers")
    probe = str(tmp_path / "libnvtx_probe.so")
    subprocess.run([cc, "-shared", "-fPIC", "-O1", "-I" + inc, os.path.join(HERE, "nvtx_probe.c"), "-o", probe],
                   check=True)
    env = dict(os.environ, NVTX_INJECTION64_PATH=probe)
    r = subprocess.run([sys.executable, "-c", CHILD, LIB, probe], env=env, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    names_line, depth_line = r.stdout.strip().splitlines()[-2:]
    assert names_line.split(",") == ["svpf_batch_create", "svpf_batch_tick_noalloc", "svpf_step_adaptive",
                                     "svpf_step_graph", "svpf_grad_forward"]
    depth, max_depth = (int(x) for x in depth_line.split())
    assert depth == 0          # every range is closed, also on the early returns
    assert max_depth == 2      # svpf_step_adaptive -> svpf_step_graph
