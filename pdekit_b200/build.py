"""Builds librds_b200.so (the CUDA kernels + C ABI) in-tree with nvcc for sm_100a."""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "librds_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["rds_api.cu", "rds_cells_scalar.cu", "rds_cells_scalar_tc.cu", "rds_cells_euler.cu",
           "rds_bc.cu",
           "rds_gather.cu", "rds_peak.cu", "rds_noalloc.cu", "rds_partition.cu", "rds_jacobian.cu", "rds_stab.cu",
           "rds_cells_scalar_dc.cu"]
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
         "-cudart", "static", f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}"]


def _headers():
    inc = os.path.join(ROOT, "include")
    return [os.path.join(d, h) for d in (CSRC, inc) for h in os.listdir(d)
            if h.endswith((".h", ".cuh"))]


def _objs_stale(obj, src):
    return not os.path.exists(obj) or os.path.getmtime(obj) < os.path.getmtime(src) or any(
        os.path.getmtime(h) > os.path.getmtime(obj) for h in _headers())


def build(verbose: bool = False, jobs: int = 8, extra=()) -> str:
    """Compile every kernel source (in parallel) and link the shared library."""
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    procs = []
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(objdir, s.replace(".cu", ".o"))
        objs.append(obj)
        if _objs_stale(obj, src) or not os.path.exists(LIB):
            cmd = [NVCC, *FLAGS, *extra, "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                              stderr=subprocess.STDOUT)))
            while len([p for _, p in procs if p.poll() is None]) >= jobs:
                procs[0][1].wait()
    for s, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out.decode())
            raise RuntimeError(f"nvcc failed on {s}")
        if verbose and out:
            sys.stdout.write(out.decode())
    cmd = [NVCC, *FLAGS, "-shared", *objs, "-o", LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
