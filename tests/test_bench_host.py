"""Host-side pieces of the benchmark, on the CPU: the workload and its
stratified samples, the plain single-filter path, and the reference arm's
JSON line (its CPU leg runs here; the reference's CUDA step reports itself
unavailable without a GPU)."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
import tape  # noqa: E402


def test_workload_is_seeded_and_stratified_sample_keeps_its_cost_distribution():
    a = bench.make_workload(4096, seed=0)
    b = bench.make_workload(4096, seed=0)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    ns = a[0]
    assert set(np.unique(ns)) == set(bench.N_CHOICES)
    idx = bench.stratified(ns, 13)
    assert len(idx) == 13 * len(bench.N_CHOICES) and len(set(idx.tolist())) == len(idx)
    counts = {n: int((ns[idx] == n).sum()) for n in bench.N_CHOICES}
    assert set(counts.values()) == {13}
    # the sample's mean N^2 is the workload's expected one (uniform over the choices)
    assert np.mean(ns[idx].astype(float) ** 2) == np.mean(np.array(bench.N_CHOICES, float) ** 2)


def test_plain_workload_is_the_projects_counter_based_path():
    h, y = bench.config1_path()
    h2, y2 = tape.sv_path(5000, -1.0, 0.97, 0.15, seed=0)
    assert h.shape == (5000,) and np.array_equal(h, h2) and np.array_equal(y, y2)


def test_cpu_sample_uses_every_thread():
    assert bench.cpu_sample(16) == 4 and bench.cpu_sample(1) == 1 and bench.cpu_sample(8) == 2
    assert isinstance(bench.cpu_model(), str)


def test_reference_arm_prints_one_line():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3", "--filters", "64"], capture_output=True, text=True, timeout=600, env=env,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "filter-ticks/s" and line["higher_is_better"]
    assert line["value"] > 0 and line["e2e"]["h2d_bytes_per_step"] == 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["pair_iterations_per_s"] > 0
    assert "unavailable" in line["reference_cuda_step"]
