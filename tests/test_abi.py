"""The C ABI: the library loads, exports every function include/svpf.h
declares, and the ctypes mirrors have the C layouts.  No compute calls."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "svpf.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"static inline[^{]*\{[^}]*\}", "", text)
    names = set()
    for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(svpf_\w+)\s*\(", text, flags=re.M):
        names.add(m.group(1))
    return sorted(names)


def test_header_declares_reference_entry_points():
    names = set(declared_functions())
    for ref in ("svpf_create", "svpf_destroy", "svpf_initialize", "svpf_step", "svpf_step_seeded",
                "svpf_step_adaptive", "svpf_step_graph", "svpf_run_sequence", "svpf_run_sequence_device",
                "svpf_get_particles", "svpf_get_stats", "svpf_get_ess", "svpf_graph_is_captured",
                "svpf_graph_invalidate"):
        assert ref in names


def test_library_exports_every_declared_function(pkg):
    lib = C.CDLL(pkg.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def _c_sizes():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "svpf.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(svpf_config_t), sizeof(svpf_ctl_t), sizeof(svpf_out_t),
         sizeof(SVPFParams), offsetof(svpf_ctl_t, status));
  return 0;
}'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "s.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "s")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include", c, "-o", exe],
                       check=True)
        return [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]


def test_ctypes_layouts_match_c(pkg, oracle_mod):
    cfg, ctl, out, prm, status_off = _c_sizes()
    assert C.sizeof(pkg.Config) == cfg == C.sizeof(oracle_mod.OracleConfig)
    assert C.sizeof(pkg.Ctl) == ctl == C.sizeof(oracle_mod.OracleCtl)
    assert C.sizeof(pkg.Out) == out == C.sizeof(oracle_mod.OracleOut)
    assert C.sizeof(pkg.Params) == prm
    assert pkg.Ctl.status.offset == status_off


@pytest.mark.parametrize("lang,std", [("c", "-std=c99"), ("c", "-std=c11"), ("c++", "-std=c++11"),
                                      ("c++", "-std=c++17")])
def test_header_compiles_as_c_and_cpp(lang, std):
    """include/svpf.h (and the svpf.cuh shim a reference caller includes) is a
    plain C header: it compiles in C and C++ translation units with warnings
    as errors, the way a caller's own build would include it."""
    cc = "gcc" if lang == "c" else "g++"
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t." + ("c" if lang == "c" else "cpp"))
        open(src, "w").write('#include "svpf.cuh"\nint svpf_header_probe(void) { return SVPF_OK; }\n')
        r = subprocess.run([cc, "-x", lang, std, "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I",
                            os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include", src],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_config_fields_follow_header_order(pkg, oracle_mod):
    text = open(HEADER).read()
    block = text[text.index("#define SVPF_CONFIG_FIELDS"):text.index("#define SVPF_DECL_INT_")]
    names = re.findall(r"X_(?:INT|FLOAT)\((\w+)\)", block)
    assert names == [f for f, _ in pkg.CONFIG_FIELDS]
    assert names == [f for f, _ in oracle_mod.CONFIG_FIELDS]


def test_batch_create_refuses_bad_sizes_before_device_work(pkg):
    """Empty batches, empty or oversized filters and runaway loop counts are
    refused on the host, before any device call (so this runs without a GPU)."""
    import ctypes as C
    lib = pkg.lib()
    cfg = pkg.production_config(30.0, 8)
    prm = pkg.Params(0.97, 0.15, -1.0, 0.0)
    for ns in ([], [0], [8193], [256, -1]):
        arr = (C.c_int * max(1, len(ns)))(*ns)
        cfgs = (pkg.Config * max(1, len(ns)))(*([cfg] * max(1, len(ns))))
        prms = (pkg.Params * max(1, len(ns)))(*([prm] * max(1, len(ns))))
        assert not lib.svpf_batch_create(len(ns), arr, cfgs, prms, None), ns
    bad = pkg.production_config(30.0, 8)
    bad.stein_max_steps = 257   # > SVPF_MAX_STEIN_STEPS
    assert not lib.svpf_batch_create(1, (C.c_int * 1)(256), (pkg.Config * 1)(bad), (pkg.Params * 1)(prm), None)


def test_noise_tape_shape_is_checked_before_the_c_call(pkg):
    """The C entry points read slots x width floats from the tape pointer and
    cannot see the buffer's size, so the Python mirror refuses any tape that
    is not [slots, width] (a 1-D array of width values is one slot)."""
    import numpy as np
    n = 64
    nrm, uni = pkg.svpf._tape(np.zeros(n), np.ones((2, n)), n)
    assert nrm.shape == (1, n) and uni.shape == (2, n) and nrm.dtype == np.float32
    for bad in (np.zeros(n + 1), np.zeros((3, n - 1)), np.zeros((0, n)), np.zeros((2, 2, n))):
        with pytest.raises(ValueError):
            pkg.svpf._tape(bad, np.ones((1, n)), n)
    with pytest.raises(ValueError):
        pkg.svpf._tape(np.zeros((1, n)), np.ones(2 * n), n)
    nrm, uni = pkg.svpf._tape(np.zeros((3, n)), None, n)   # no uniform slots
    assert nrm.shape == (3, n) and uni is None
