"""Builds libscrna_cle.so (CUDA, sm_100a) in-tree with nvcc.

Used by __graft_entry__.build() and by the package on first import when the
library is missing.  nvcc cross-compiles for sm_100a without a GPU.  Each .cu
file is compiled to an object in parallel, then linked into one shared library.
"""
from __future__ import annotations

import glob
import os
import re
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libscrna_cle.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


_INCLUDE_RE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps(src):
    """Local headers that src includes, directly or through other local headers."""
    seen, todo = set(), [src]
    while todo:
        with open(todo.pop()) as f:
            text = f.read()
        for name in _INCLUDE_RE.findall(text):
            for d in (CSRC, INCLUDE):
                path = os.path.join(d, name)
                if os.path.exists(path) and path not in seen:
                    seen.add(path)
                    todo.append(path)
                    break
    return sorted(seen)


def _stale(target, srcs) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in srcs)


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found; the CUDA library cannot be built")
    return exe


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    jobs = []
    objs = []
    for src in sources():
        obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + _deps(src)):
            cmd = [nvcc()] + NVCC_FLAGS + ["-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            logs = list(ex.map(lambda c: _run(c, verbose), jobs))
        if ptxas_info:
            print("\n".join(logs))
    if jobs or force or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        _run([nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcublasLt", "-ldl"], verbose)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    import sys
    build(force="-f" in sys.argv, verbose=True, ptxas_info="-v" in sys.argv)
