"""Build the native libraries in-tree.

* ``libsp_b200.so`` — the sm_100a kernels and the C ABI (include/starplat_b200.h),
  compiled with ``nvcc -gencode arch=compute_100a,code=sm_100a``; CUDA runtime
  linked statically so it does not clash with the runtime PyTorch loads.
* ``libspgen.so`` — seeded graph generators / CSR construction (host C++ + OpenMP).

The libraries land next to this file; a GPU box receives them with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")

CU_SOURCES = ["sp_graph.cu", "sp_pagerank.cu", "sp_tc.cu", "sp_sssp.cu", "sp_bc.cu", "sp_louvain.cu",
              "sp_noalloc.cu", "sp_mlp.cu", "sp_ingest.cu", "sp_centrality.cu",
              "sp_sssp_part.cu"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--cudart", "static",
    "-Xptxas", "-warn-spills",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_gen(force: bool = False, verbose: bool = False) -> str:
    out = os.path.join(HERE, "libspgen.so")
    src = os.path.join(CSRC, "spgen.cpp")
    if force or _stale(out, [src]):
        cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", src, "-o", out]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return out


def build_cuda(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    out = os.path.join(HERE, "libsp_b200.so")
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    if not (force or _stale(out, deps)):
        return out
    objdir = os.path.join(ROOT, "_build")
    os.makedirs(objdir, exist_ok=True)
    nvcc = _nvcc()
    objs = []
    procs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        objs.append(o)
        cmd = [nvcc, *NVCC_FLAGS, "-I", INCLUDE, "-c", s, "-o", o]
        if ptxas_verbose:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd))
        procs.append((s, subprocess.Popen(cmd)))
    for s, p in procs:
        if p.wait() != 0:
            raise RuntimeError(f"nvcc failed on {s}")
    cmd = [nvcc, "-shared", "--cudart", "static", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", out]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return out


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_gen(force, verbose)
    build_cuda(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
