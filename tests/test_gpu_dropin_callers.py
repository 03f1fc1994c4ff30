"""Unmodified reference callers on this engine.

The reference's own callers are compiled, unedited, against this project's
include/svpf.cuh (which includes svpf.h) and linked to libsvpf_b200.so by
the checker recipe (oracle/Makefile, target `callers`):

* py-torch/svpf_python.cpp -- the reference's pybind11 module `pysvpf`.  Its
  SVPF class must step exactly like this project's Python mirror of it
  (svpf.py), since both drive the same library with the same configuration
  and seed: bit-identical outputs.
* test/test_svpf_scenarios.cu -- the reference's scenario test program,
  built twice: against this engine and against the reference's own library.
  Each run prints the filtered log-vol RMSE on its 8000-tick synthetic path;
  the two must agree within 2% (each side draws its own noise).
"""
import glob
import importlib.util
import os
import re
import subprocess

import numpy as np
import pytest

import tape

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")


def _need(path):
    if not os.path.exists(path):
        pytest.skip(f"{os.path.basename(path)} not built (oracle/Makefile target `callers` needs the reference tree)")
    return path


def test_reference_pybind_module_on_the_engine(pkg):
    mods = glob.glob(os.path.join(REF_BIN, "pysvpf*.so"))
    _need(mods[0] if mods else os.path.join(REF_BIN, "pysvpf.so"))
    spec = importlib.util.spec_from_file_location("pysvpf", mods[0])
    pysvpf = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(pysvpf)
    _, ys = tape.sv_path(200, -3.5, 0.97, 0.2, seed=9)
    ref = pysvpf.SVPF(256, 8, 30.0)
    ref.initialize(0.97, 0.15, -3.5, -0.5, 42)
    vol_r, h_r, ll_r = ref.run(ys)
    ours = pkg.SVPF(256, 8, 30.0)
    ours.initialize(0.97, 0.15, -3.5, -0.5, seed=42)
    vol_o, h_o, ll_o = ours.run(ys)
    assert np.all(np.isfinite(h_r))
    assert np.array_equal(h_r, h_o) and np.array_equal(vol_r, vol_o) and np.array_equal(ll_r, ll_o)
    r1 = ref.step(0.01)
    r2 = ours.step(0.01)
    assert (r1.h_mean, r1.vol_mean, r1.log_lik, r1.mu_estimate) == (r2.h_mean, r2.vol_mean, r2.log_lik,
                                                                      r2.mu_estimate)
    ours.close()


def _rmse(binary, tmp_path):
    r = subprocess.run([binary, "--seed", "42", "--particles", "512"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    m = re.search(r"Log-Vol RMSE:\s+([0-9.]+)", r.stdout)
    assert m, r.stdout[-2000:]
    return float(m.group(1))


def test_reference_scenario_program_on_the_engine(tmp_path):
    ours = _rmse(_need(os.path.join(REF_BIN, "scenarios_b200")), tmp_path)
    ref = _rmse(_need(os.path.join(REF_BIN, "scenarios_ref")), tmp_path)
    with open(os.path.join(tmp_path, "rmse.txt"), "w") as fh:
        fh.write(f"engine {ours} reference {ref}\n")
    assert abs(ours - ref) <= 0.02 * ref, (ours, ref)
