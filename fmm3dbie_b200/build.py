"""Build libfmm3dbie_b200.so in-tree (host C++ + CUDA for sm_100a).

    python -m fmm3dbie_b200.build [--force] [--reference DIR]

The node tables for triangular patches are parsed from a reference checkout
(DIR/src/tria_routs/koorn-*.txt) into fmm3dbie_b200/_data/ when they are not
there yet (see tables.py); DIR comes from --reference or FMM3DBIE_REFERENCE.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libfmm3dbie_b200.so")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-march=x86-64-v3", "-Wall",
            "-Wno-unknown-pragmas"]
# -ftz=true: single-precision denormals flush to zero (the FP32 far-field pair
# function then needs no denormal fix-ups around rsqrtf); FP64 is unaffected.
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-ftz=true", "-Xcompiler", "-fPIC,-fopenmp",
                  "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _headers():
    return glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True) + \
        glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True) + \
        [os.path.join(ROOT, "include", "fmm3dbie_b200.h")]


def _stale(obj, src, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(force: bool = False, reference: str | None = None, verbose: bool = False) -> str:
    from . import tables
    if not os.path.exists(tables.TABLE_PATH):
        ref = reference or os.environ.get("FMM3DBIE_REFERENCE")
        if not ref or not os.path.isdir(ref):
            raise RuntimeError(
                f"{tables.TABLE_PATH} is missing and no reference checkout was given to parse "
                "the Vioreanu-Rokhlin node tables from: pass --reference DIR or set "
                "FMM3DBIE_REFERENCE")
        tables.generate(ref)
    os.makedirs(BUILD, exist_ok=True)
    deps = _headers()
    jobs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _stale(obj, src, deps):
            jobs.append([CXX] + CXXFLAGS + ["-c", src, "-o", obj])
    for src in sorted(glob.glob(os.path.join(CSRC, "cuda", "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _stale(obj, src, deps):
            jobs.append([NVCC] + NVFLAGS + ["-c", src, "-o", obj])
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    objs = sorted(glob.glob(os.path.join(BUILD, "*.o")))
    if jobs or force or not os.path.exists(LIB):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs +
             ["-Xcompiler", "-fopenmp", "-cudart", "static", "-ldl"])
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--reference", default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    sys.path.insert(0, ROOT)
    from fmm3dbie_b200 import build as _b  # noqa: E402
    print(_b.build(force=a.force, reference=a.reference, verbose=a.verbose))
