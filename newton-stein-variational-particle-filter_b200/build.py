"""Build libsvpf_b200.so in-tree with nvcc for sm_100a.

    python build.py            # incremental: rebuild objects whose inputs changed
    python build.py --force    # rebuild everything

Objects are compiled in parallel and linked into ``libsvpf_b200.so`` next to
this file, so the library travels with the source tree.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsvpf_b200.so")
INCLUDE = os.path.join(ROOT, "include")

SOURCES = ["svpf_kernels.cu", "svpf_single_small.cu", "svpf_single_large.cu", "svpf_single_2f.cu",
           "svpf_batch_kernel.cu", "svpf_capi.cu", "svpf_batch.cu", "svpf_noalloc.cu", "svpf_grad.cu",
           "svpf_stream.cu", "svpf_v2.cu",
           "svpf_multiscale.cu", "svpf_estimator.cu", "svpf_calib.cu"]
HEADERS = ["svpf_device.cuh", "svpf_tick.cuh", "svpf_tick2f.cuh", "svpf_internal.h", "svpf_single.cuh", "svpf_math.h",
           "svpf_trace.h"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _digest(src: str, extra: list[str]) -> str:
    h = hashlib.sha256()
    for p in [os.path.join(CSRC, src)] + [os.path.join(CSRC, x) for x in HEADERS] + [os.path.join(INCLUDE, "svpf.h")]:
        with open(p, "rb") as f:
            h.update(f.read())
    h.update(" ".join(NVCC_FLAGS + extra).encode())
    return h.hexdigest()[:16]


def _compile(src: str, force: bool, verbose: bool, extra: list[str]) -> str:
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    stamp = obj + ".sha"
    dig = _digest(src, extra)
    if not force and os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == dig:
        return obj
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    with open(stamp, "w") as f:
        f.write(dig)
    return obj


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose or ptxas_verbose, extra), SOURCES))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", LIB, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force, verbose=True, ptxas_verbose=args.ptxas_verbose))
