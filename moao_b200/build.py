"""Builds the in-tree shared library ``moao_b200/libmoao_b200.so`` for sm_100a.

Run ``python -m moao_b200.build`` (or ``__graft_entry__.build()``). Objects go
to ``moao_b200/_build/`` and are rebuilt only when a source or header changed.
nvcc cross-compiles for sm_100a, so this works on a machine without a GPU.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmoao_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
          "-I" + INCLUDE, "-I" + CSRC, "--expt-relaxed-constexpr"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h*"))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, jobs: int = 8) -> str:
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    objs, cmds = [], []
    for src in _sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(obj, [src] + headers):
            flags = list(COMMON)
            if src.endswith(".cpp"):
                cmd = [NVCC, "-x", "cu"] + ARCH + flags + ["-c", src, "-o", obj]
            else:
                cmd = [NVCC] + ARCH + flags + ["-c", src, "-o", obj]
            cmds.append(cmd)
    # compile in parallel
    procs = []
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        if len(procs) >= jobs:
            _drain(procs)
    _drain(procs)
    if cmds or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        link = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + [
            "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcuda",
            "-Xlinker", "--exclude-libs,ALL", "-Xlinker", "-rpath," + os.path.join(CUDA_HOME, "lib64")]
        if verbose:
            print(" ".join(link))
        r = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout)
        shutil.move(tmp, LIB)
    return LIB


def _drain(procs):
    errs = []
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            errs.append(" ".join(cmd) + "\n" + out.decode(errors="replace"))
    procs.clear()
    if errs:
        raise RuntimeError("compilation failed:\n" + "\n".join(errs))


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
