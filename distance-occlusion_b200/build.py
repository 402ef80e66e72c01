"""Build libdol_b200.so in-tree with nvcc for sm_100a.

Usage:  python distance-occlusion_b200/build.py [--force] [--verbose]

Every .cu file under csrc/ (and the C++ host interface in shim/) is compiled for sm_100a (-gencode
arch=compute_100a,code=sm_100a) with -lineinfo and linked with the static CUDA
runtime into distance-occlusion_b200/libdol_b200.so.  The object files go to
distance-occlusion_b200/_build/ and are rebuilt only when a source or header
is newer.  No torch, no JIT cache: the .so next to this file is what loads.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "libdol_b200.so")
BUILD = os.path.join(PKG, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
]


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu"))) + sorted(glob.glob(os.path.join(PKG, "shim", "*.cpp")))
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h")) + glob.glob(os.path.join(PKG, "shim", "*.h"))
    hdr_time = _newest(headers)
    objs = []
    jobs = []
    for src in sources:
        obj = os.path.join(BUILD, os.path.splitext(os.path.basename(src))[0] + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr_time):
            cmd = [NVCC] + FLAGS + ["-Xptxas", "-v"] * bool(verbose) + ["-c", src, "-o", obj]
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        return r.stdout + r.stderr

    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for log in ex.map(run, jobs):
                if verbose and log.strip():
                    print(log)
    if force or jobs or not os.path.exists(OUT) or os.path.getmtime(OUT) < _newest(objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", OUT] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
