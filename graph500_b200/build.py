"""Build recipe for libg500.so: every CUDA source under csrc/ compiled for
sm_100a with nvcc and linked into one shared library next to this file.

Also builds g500_main, the main.cc-style benchmark driver (driver/g500_main.cc).

Usage: python -m graph500_b200.build [-v] [--force]
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
LIB = os.path.join(HERE, "libg500.so")
DRIVER = os.path.join(HERE, "g500_main")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
              "--expt-relaxed-constexpr", "-I" + INCLUDE] + ARCH


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return hs + [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith((".h", ".hpp"))]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    env = dict(os.environ)
    # the system gcc is nvcc's host compiler (CC/CXX may point at a toolchain without OpenMP specs)
    env.pop("CC", None)
    env.pop("CXX", None)
    nv = nvcc()
    hdrs = headers()
    objs, jobs = [], []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            cmd = [nv, "-c", src, "-o", obj] + NVCC_FLAGS
            if verbose:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True, env=env)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for cmd, r in ex.map(run, jobs):
            if verbose or r.returncode:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode:
                raise RuntimeError("nvcc failed: " + " ".join(cmd))
    if force or jobs or _stale(LIB, objs):
        cmd = [nv, "-shared", "-o", LIB] + objs + ARCH + ["-lcuda"]
        r = subprocess.run(cmd, capture_output=True, text=True, env=env)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    # the main.cc-style driver: host C++ over the C ABI, next to the library
    drv = os.path.join(HERE, "driver", "g500_main.cc")
    if force or _stale(DRIVER, [drv, LIB] + hdrs):
        cmd = ["g++", "-O2", "-std=c++17", "-I" + INCLUDE, drv, "-o", DRIVER, "-L" + HERE, "-lg500",
               "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True, env=env)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("driver build failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.force))
