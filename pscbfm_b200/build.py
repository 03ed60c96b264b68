"""Builds pscbfm_b200/libbfm.so (the C-ABI library) from pscbfm_b200/csrc with nvcc for sm_100a.

Objects go to pscbfm_b200/_build/; only changed sources are recompiled. Run as a script or call
build().
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbfm.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", INCLUDE]
CU_FLAGS = ARCH + ["-lineinfo", "--expt-relaxed-constexpr"]

SOURCES = ["bfm_kernels.cu", "bfm_kernels_bc.cu", "bfm_observables.cu", "bfm_engine.cpp", "bfm_batch.cpp",
           "bfm_color.cpp", "bfm_capi.cpp", "bfm_server.cpp", "bfm_noalloc.cu", "bfm_probe.cu"]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return hs


def _stale(obj, src, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + deps)


def _compile(src):
    path = os.path.join(CSRC, src)
    obj = os.path.join(OUT, src + ".o")
    flags = COMMON + (CU_FLAGS if src.endswith(".cu") else ["-x", "cu"] + CU_FLAGS)
    cmd = [NVCC] + flags + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    deps = _headers()
    todo = [s for s in SOURCES if force or _stale(os.path.join(OUT, s + ".o"), os.path.join(CSRC, s), deps)]
    if todo:
        with ThreadPoolExecutor(max_workers=min(len(todo), os.cpu_count() or 4)) as ex:
            for obj in ex.map(_compile, todo):
                if verbose:
                    print("built", obj)
    objs = [os.path.join(OUT, s + ".o") for s in SOURCES]
    if todo or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
