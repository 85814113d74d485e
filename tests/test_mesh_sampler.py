"""Mesh-to-point-cloud sampling (the reference's
GeneratePointCloudFromWatertightTriangleMesh, GeometryLoading.cpp:10-83, as
LoadMPMPointCloudFromObj calls it).  Golden vectors: the points the
reference's own sampler, compiled with its vendored libigl
(oracle/build_ref_mesh.sh, tests/golden/make_mesh_golden.py), keeps for three
seeded meshes (sphere, non-convex bumpy sphere, tilted torus).  The CPU
restatement (oracle/mesh.py) is pinned to them on the sphere; the GPU sampler
(dmpm_mesh_lattice_points) must reproduce every point, bit for bit and in
order, on all three."""
import os

import numpy as np
import pytest

import dmpm
from oracle import mesh as omesh
from tests.helpers import GOLDEN

MESHES = ("sphere", "bumpy", "torus")


def _golden(name):
    g = np.load(os.path.join(GOLDEN, "mesh_%s_points.npz" % name))
    return os.path.join(GOLDEN, "mesh_%s.obj" % name), float(g["point_dx"]), g["points"]


def test_oracle_matches_reference_sampler():
    obj, dx, ref = _golden("sphere")
    V, F = omesh.read_obj(obj)
    assert np.array_equal(omesh.lattice_points(V, F, dx), ref)


def test_obj_reader_matches_oracle_reader():
    obj, _, _ = _golden("torus")
    V, F = dmpm.read_obj(obj)
    V2, F2 = omesh.read_obj(obj)
    assert np.array_equal(V, V2) and np.array_equal(F, F2.astype(np.int32))


@pytest.mark.gpu
@pytest.mark.parametrize("name", MESHES)
def test_gpu_sampler_matches_reference_bit_exactly(gpu_ready, name):
    obj, dx, ref = _golden(name)
    V, F = dmpm.read_obj(obj)
    pts = dmpm.mesh_lattice_points(V, F, dx)
    assert pts.shape == ref.shape
    assert np.array_equal(pts, ref)


@pytest.mark.gpu
def test_point_cloud_from_obj_and_errors(gpu_ready):
    obj, dx, ref = _golden("bumpy")
    pc = dmpm.point_cloud_from_obj(obj, dx, 40.0, 58333.0, 38888.9)
    assert np.array_equal(pc["x"], ref.astype(np.float64))
    assert pc["m"][0] == pytest.approx(float(np.float32(dx)) ** 3 * 40.0, rel=1e-6)
    V, F = dmpm.read_obj(obj)
    bad = F.copy()
    bad[0, 0] = len(V)  # vertex index out of range
    with pytest.raises(dmpm.DmpmError):
        dmpm.mesh_lattice_points(V, bad, dx)
    with pytest.raises(dmpm.DmpmError):
        dmpm.mesh_lattice_points(V, F, -1.0)


@pytest.mark.gpu
def test_compat_cpp_geometry_loading(gpu_ready, tmp_path):
    """GeometryLoading::GeneratePointCloudFromWatertightTriangleMesh of the
    C++ compat API, called as LoadMPMPointCloudFromObj calls it."""
    import subprocess

    import build as pkg_build

    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    pkg = os.path.join(repo, "a-differentiable-material-point-method-for-shape-morphing_b200")
    pkg_build.build_compat()
    exe = str(tmp_path / "mesh_check")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(pkg, "compat"), "-I",
                           os.path.join(repo, "include"), os.path.join(repo, "tests", "cpp", "mesh_check.cpp"),
                           "-L", pkg, "-ldmpm_compat", "-ldmpm", "-Wl,-rpath," + pkg, "-o", exe])
    obj, dx, ref = _golden("torus")
    out = tmp_path / "pts.bin"
    subprocess.check_call([exe, obj, repr(dx), str(out)])
    pts = np.fromfile(out, dtype=np.float32).reshape(-1, 3)
    assert np.array_equal(pts, ref)
