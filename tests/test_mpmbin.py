"""The .mpmbin on-disk format (a cereal binary archive of the reference's
PointCloud, PointCloud.cpp:334-362) pinned against a file written by the
reference's own writer (tests/golden/cloud_ref.mpmbin, made by
tests/golden/make_golden.py): the Python writer reproduces it byte for byte
and the compat C++ PointCloud reads and rewrites it unchanged.  Host IO only."""
import os
import subprocess

import numpy as np
import pytest

from tests.golden.make_golden import mpmbin_scene
from tests.helpers import GOLDEN, write_mpmbin

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "a-differentiable-material-point-method-for-shape-morphing_b200")


def test_python_writer_matches_reference_bytes(tmp_path):
    sc = mpmbin_scene()
    out = tmp_path / "cloud.mpmbin"
    write_mpmbin(out, sc.x, sc.v, sc.F, sc.C, np.zeros((sc.n, 3, 3)), sc.m, sc.vol, sc.lam, sc.mu, sc.dFc)
    assert out.read_bytes() == open(os.path.join(GOLDEN, "cloud_ref.mpmbin"), "rb").read()


def test_compat_pointcloud_roundtrip(tmp_path):
    import build as pkg_build

    lib = pkg_build.build_compat()
    exe = tmp_path / "roundtrip"
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-I", os.path.join(PKG, "compat"), "-I",
                           os.path.join(REPO, "include"), os.path.join(REPO, "tests", "cpp", "mpmbin_roundtrip.cpp"),
                           "-L", PKG, "-ldmpm_compat", "-ldmpm", "-Wl,-rpath," + PKG, "-o", str(exe)])
    src = os.path.join(GOLDEN, "cloud_ref.mpmbin")
    dst = tmp_path / "back.mpmbin"
    out = subprocess.run([str(exe), src, str(dst)], capture_output=True, text=True, check=True).stdout
    assert int(out.strip()) == mpmbin_scene().n
    assert dst.read_bytes() == open(src, "rb").read()
