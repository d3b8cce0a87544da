"""Build the engine's native libraries in-tree.

    python -m dynamicgraphs_scc_b200.build          # libscc_b200.so + scc driver

Outputs (git-ignored, shipped with the tree):
    dynamicgraphs_scc_b200/lib/libscc_b200.so   the C-ABI library (sm_100a)
    dynamicgraphs_scc_b200/lib/scc              the drop-in CLI driver
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = [
    "scc_graph.cu",
    "scc_sort.cu",
    "scc_state.cu",
    "scc_trim.cu",
    "scc_fb.cu",
    "scc_reach.cu",
    "scc_tile.cu",
    "scc_batch.cu",
    "scc_wcc.cu",
    "scc_run.cu",
    "scc_gen.cu",
    "scc_noalloc.cu",
    "scc_update.cu",
    "scc_tune.cu",
    "scc_server.cu",
    "scc_mlp.cu",
    "scc_levels.cu",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} (exit {r.returncode})")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    obj_dir = os.path.join(LIB, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "scc_capi.h"))
    objs = []
    flags = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC, *ARCH]
    for src in CU_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(obj_dir, src.replace(".cu", ".o"))
        if force or _stale(obj, [path, *headers]):
            cmd = [nvcc(), *flags, "-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
        objs.append(obj)
    so = os.path.join(LIB, "libscc_b200.so")
    if force or _stale(so, objs):
        _run([nvcc(), *ARCH, "-shared", "-o", so, *objs, "-lcudart"])
    drv_src = os.path.join(CSRC, "scc_main.cpp")
    drv = os.path.join(LIB, "scc")
    if os.path.exists(drv_src) and (force or _stale(drv, [drv_src, so, *headers])):
        _run(["g++", "-O2", "-std=c++17", "-I", INCLUDE, drv_src, "-o", drv, "-L", LIB, "-lscc_b200",
              f"-Wl,-rpath,{LIB}", "-Wl,-rpath,$ORIGIN"])
    return so


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(os.path.join(LIB, "libscc_b200.so"))
