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


COMPAT = os.path.join(PKG_DIR, "compat")
COMPAT_LIB = os.path.join(PKG_DIR, "libdmpm_compat.so")
COMPAT_EIGEN_LIB = os.path.join(PKG_DIR, "libdmpm_compat_eigen.so")


def _compat_sources():
    return [os.path.join(COMPAT, "dmpm_compat.cpp")] + [os.path.join(COMPAT, "DiffMPMLib3D", f)
                                                        for f in os.listdir(os.path.join(COMPAT, "DiffMPMLib3D"))]


def _build_compat_lib(target, flags, force, verbose):
    srcs = _compat_sources() + [LIB]
    if force or _stale(target, srcs):
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", *flags, "-I", COMPAT, "-I",
               os.path.join(REPO, "include"), "-o", target + ".tmp", os.path.join(COMPAT, "dmpm_compat.cpp"), "-L",
               PKG_DIR, "-ldmpm", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
        os.replace(target + ".tmp", target)
    return target


def build_compat(force: bool = False, verbose: bool = False) -> str:
    """The DiffMPMLib3D-compatible C++ API over libdmpm.so with its own value
    types (libdmpm_compat.so), for callers built without Eigen."""
    build(force=force, verbose=verbose)
    return _build_compat_lib(COMPAT_LIB, ["-DDMPM_COMPAT_NO_EIGEN"], force, verbose)


def build_compat_eigen(eigen_include: str, force: bool = False, verbose: bool = False) -> str:
    """The same API with Vec3 / Mat3 = Eigen::Vector3f / Matrix3f
    (libdmpm_compat_eigen.so), for callers that do Eigen arithmetic on the
    reference's types; eigen_include is the directory holding Eigen/Dense."""
    build(force=force, verbose=verbose)
    return _build_compat_lib(COMPAT_EIGEN_LIB, ["-DDMPM_COMPAT_EIGEN", "-I", eigen_include], force, verbose)


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
    print(build_compat(force="--force" in sys.argv, verbose=True))
