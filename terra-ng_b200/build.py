"""Build libterra_b200.so (CUDA kernels for sm_100a + C++ host runtime + C ABI).

    python terra-ng_b200/build.py [--force] [--verbose]

Objects go to terra-ng_b200/_build/, the shared library to
terra-ng_b200/libterra_b200.so (in-tree, so it travels with the repository
snapshot). Host C++ is compiled with -ffp-contract=off so the mesh generator
rounds exactly like the reference's default host build.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libterra_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
CXX = "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
                     "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra", "-I" + INCLUDE, "-I" + CSRC,
             "-I/usr/local/cuda/include"]


def _sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith(".cu") or f.endswith(".cpp"):
            out.append(os.path.join(CSRC, f))
    return out


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return hs


def _compile(src, force, verbose):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest_dep = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in _headers()])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj, None
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
    else:
        cmd = [CXX] + CXX_FLAGS + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, r.stdout + r.stderr
    return obj, None


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    errors = [e for _, e in results if e]
    if errors:
        raise RuntimeError("compilation failed:\n" + "\n".join(errors))
    objs = [o for o, _ in results]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    try:
        print(build(a.force, a.verbose))
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
