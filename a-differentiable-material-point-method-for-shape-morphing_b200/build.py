"""Build recipe for libdmpm.so (sm_100a) -- run by __graft_entry__.build().

    nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3 -std=c++17 \
         -Xcompiler -fPIC -shared -I include -o <pkg>/libdmpm.so <pkg>/csrc/*.cu

The library is built in-tree so it travels with the repository snapshot.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
LIB = os.path.join(PKG_DIR, "libdmpm.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cu", ".cuh", ".h"))] + [
        os.path.join(REPO, "include", "dmpm.h")]


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(force: bool = False, verbose: bool = False) -> str:
    srcs = _sources()
    if force or _stale(LIB, srcs):
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
               "-I", os.path.join(REPO, "include"), "-o", LIB + ".tmp",
               *[os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith(".cu")]]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
