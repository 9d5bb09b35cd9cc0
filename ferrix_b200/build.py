"""Builds ferrix_b200/libferrix_b200.so (sm_100a) in-tree with nvcc.

    python -m ferrix_b200.build [--force] [--debug]

All sources are compiled by nvcc for `-gencode arch=compute_100a,code=sm_100a`
with line info, linked against the static CUDA runtime, so the library needs
no PyTorch and no JIT cache. Objects are rebuilt when a source or header is
newer than the object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libferrix_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _flags(debug: bool):
    f = ["-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo", "-I", os.path.join(ROOT, "include"),
         "--expt-relaxed-constexpr"]
    f += ["-O0", "-g", "-G"] if debug else ["-O3"]
    return f


def _headers():
    return glob.glob(os.path.join(CSRC, "*.hpp")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(ROOT, "include", "ferrix_b200.h")]


def _compile(src: str, debug: bool, force: bool, hdr_mtime: float, verbose: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime):
        return obj
    cmd = [NVCC] + ARCH + _flags(debug) + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd[1:1] = ["-x", "cu"]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        sys.stderr.write(res.stderr)
    return obj


def build(force: bool = False, debug: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    hdr = max(os.path.getmtime(h) for h in _headers())
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile(s, debug, force, hdr, verbose), srcs))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-cudart", "static"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="pass -Xptxas -v")
    a = ap.parse_args()
    print(build(a.force, a.debug, a.verbose))
