"""Builds libgpair_b200.so (sm_100a) in-tree from gpair_b200/csrc.

CUDA sources are compiled by nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a); the host-side C (OIFITS indexer,
setup) by gcc with floating-point contraction off so that its float/double
arithmetic matches the reference's. Objects go to gpair_b200/_build, the
library to gpair_b200/libgpair_b200.so. Rebuilds only what changed.

    python -m gpair_b200.build [--force] [-j N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgpair_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    cu = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
    c = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".c"))
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "gpair_b200.h"))
    return cu, c, headers


def _stale(obj: str, src: str, headers) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src, *headers])


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stderr


def build(force: bool = False, jobs: int = 8, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    cu, c, headers = _sources()
    cmds, objs = [], []
    for src in cu:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, src, headers):
            cmds.append([nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
                         "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj])
    for src in c:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, src, headers):
            cmds.append(["gcc", "-O2", "-std=gnu99", "-fPIC", "-ffp-contract=off", "-Wall", "-I", INCLUDE, "-c",
                         src, "-o", obj])
    if cmds:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            for err in ex.map(_compile, cmds):
                if verbose and err:
                    print(err, file=sys.stderr)
    if force or cmds or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        tmp = LIB + ".tmp"
        _compile([nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcuda"])
        os.replace(tmp, LIB)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.j, a.v))


if __name__ == "__main__":
    main()
