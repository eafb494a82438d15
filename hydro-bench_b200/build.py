"""Build ``hydrob200/libhydrob200.so`` (sm_100a) in-tree with nvcc.

    python hydro-bench_b200/build.py [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT_DIR = os.path.join(HERE, "hydrob200")
LIB = os.path.join(OUT_DIR, "libhydrob200.so")
OBJ_DIR = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["hb_solver.cu", "hb_tiles.cu", "hb_ref_layout.cu", "hb_adjoint.cu"]
CPP_SOURCES = ["hb_deck.cpp"]


def _sources():
    srcs = [os.path.join(CSRC, f) for f in CU_SOURCES + CPP_SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h", ".hpp"))]
    deps += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return srcs, deps


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    _, deps = _sources()
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = True) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    objs = []
    common = ["-O3", "-std=c++17", "-I", INCLUDE, "-I", CSRC]
    # the translation units compile in parallel
    from concurrent.futures import ThreadPoolExecutor
    jobs = []
    for f in CU_SOURCES:
        o = os.path.join(OBJ_DIR, f + ".o")
        cmd = [NVCC, *ARCH, "-lineinfo", *common, "-Xcompiler", "-fPIC", "-Xptxas", "-v", "-c",
               os.path.join(CSRC, f), "-o", o]
        jobs.append((cmd, os.path.join(OBJ_DIR, f + ".ptxas.txt")))
        objs.append(o)
    with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        for fut in [ex.submit(_run, cmd, verbose, log) for cmd, log in jobs]:
            fut.result()
    for f in CPP_SOURCES:
        o = os.path.join(OBJ_DIR, f + ".o")
        # host arithmetic of the deck reader must round every operation like the reference's host code
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I", INCLUDE, "-I", CSRC,
               "-I", "/usr/local/cuda/include", "-c", os.path.join(CSRC, f), "-o", o]
        _run(cmd, verbose)
        objs.append(o)
    tmp = LIB + ".tmp"
    _run([NVCC, *ARCH, "-shared", "-o", tmp, *objs], verbose)
    os.replace(tmp, LIB)
    return LIB


def _run(cmd, verbose, log=None):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if log:
        with open(log, "w") as f:
            f.write(r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")


if __name__ == "__main__":
    build(force="--force" in sys.argv)
