"""The scalar helpers the device kernels share (csrc/svpf_math.h), compiled
for the CPU with g++ and checked before any kernel runs them: the digamma
used for d/dnu of the Student-t normaliser against scipy and the oracle's own
digamma, its termination on every input (x <= 0, -inf, NaN, huge negative
values, denormals), and the parameter-domain check the gradient and
estimator engines apply to theta."""
import ctypes as C
import math
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "newton-stein-variational-particle-filter_b200", "csrc")

DRIVER = r"""
#include "svpf_math.h"
extern "C" double t_digamma(double x) { return svpf::digamma_bounded(x); }
extern "C" int t_theta_ok(float mu, float rho, float sz, float nu) { return svpf::theta_ok(mu, rho, sz, nu) ? 1 : 0; }
"""


@pytest.fixture(scope="module")
def mathlib(tmp_path_factory):
    d = tmp_path_factory.mktemp("svpf_math")
    src = d / "drv.cpp"
    src.write_text(DRIVER)
    so = d / "libdrv.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I" + CSRC, str(src), "-o", str(so)],
                   check=True)
    L = C.CDLL(str(so))
    L.t_digamma.restype = C.c_double
    L.t_digamma.argtypes = [C.c_double]
    L.t_theta_ok.restype = C.c_int
    L.t_theta_ok.argtypes = [C.c_float] * 4
    return L


def test_digamma_matches_scipy_and_oracle(mathlib, oracle_mod):
    from scipy.special import psi
    L = oracle_mod.lib()
    L.svpf_oracle_digamma.restype = C.c_double
    L.svpf_oracle_digamma.argtypes = [C.c_double]
    xs = np.concatenate([np.geomspace(1e-6, 1e6, 400), np.linspace(0.01, 40.0, 400)])
    for x in xs:
        got = mathlib.t_digamma(float(x))
        want = float(psi(x))
        assert abs(got - want) <= 1e-12 * max(1.0, abs(want)), (x, got, want)
        assert L.svpf_oracle_digamma(float(x)) == got


@pytest.mark.parametrize("x", [0.0, -0.0, -1.0, -1e9, -1e16, -1e30, -math.inf, math.nan, -5e-324])
def test_digamma_terminates_with_nan_outside_domain(mathlib, x):
    # each of these kept the unbounded recurrence running (x += 1 leaves
    # x unchanged below -1e16) or evaluated psi at a pole
    assert math.isnan(mathlib.t_digamma(x))


def test_digamma_edge_values(mathlib):
    assert mathlib.t_digamma(math.inf) == math.inf
    # a denormal: eight shifts take it to 8; the pole term dominates
    v = mathlib.t_digamma(5e-324)
    assert v == -math.inf or v < -1e300


def test_theta_domain(mathlib):
    ok = mathlib.t_theta_ok
    assert ok(-1.0, 0.97, 0.15, 5.0)
    assert ok(0.0, -0.5, 1e-6, 1e6)
    for bad in [(-1.0, 1.0, 0.15, 5.0), (-1.0, -1.0, 0.15, 5.0), (-1.0, 0.97, 0.0, 5.0), (-1.0, 0.97, -0.1, 5.0),
                (-1.0, 0.97, 0.15, 0.0), (-1.0, 0.97, 0.15, -math.inf), (-1.0, 0.97, 0.15, -1e30),
                (-1.0, 0.97, math.nan, 5.0), (math.nan, 0.97, 0.15, 5.0), (math.inf, 0.97, 0.15, 5.0),
                (-1.0, math.nan, 0.15, 5.0), (-1.0, 0.97, 0.15, math.inf), (-1.0, 0.97, math.inf, 5.0)]:
        assert not ok(*bad), bad
