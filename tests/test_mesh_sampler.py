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


@pytest.mark.gpu
def test_input_file_and_mesh_drive_a_gradient(gpu_ready, tmp_path):
    """An OptInput file naming OBJ meshes, turned into a context the way the
    reference's animator sets up its CompGraph (LoadMPMPointCloudFromObj for
    the input and target meshes, grid from the file, volumes, target mass
    raster, simulation parameters), runs forward + loss + backward."""
    import optinput

    obj, _, _ = _golden("sphere")
    opt = optinput.OptInput(mpm_input_mesh_path=obj, mpm_target_mesh_path=obj, grid_dx=0.05,
                            grid_min_point=(-1.0, -1.0, -1.0), grid_max_point=(1.0, 1.0, 1.0), dt=1e-4,
                            num_timesteps=4, control_stride=2)
    path = str(tmp_path / "input.json")
    optinput.save(opt, path)
    opt = optinput.load(path)
    pc = dmpm.point_cloud_from_obj(opt.mpm_input_mesh_path, optinput.point_dx(opt), opt.p_density, opt.lam, opt.mu)
    assert abs(pc["m"][0] - optinput.point_mass(opt)) <= 1e-6 * optinput.point_mass(opt)
    with dmpm.Context("fp32") as c:
        c.set_grid(optinput.grid_dims(opt), opt.grid_dx, opt.grid_min_point)
        c.set_particles(pc["x"], pc["m"], pc["lam"], pc["mu"], v=pc["v"], F=pc["F"])
        c.compute_volumes()  # CalculatePointCloudVolumes, as LoadCompGraph does
        tpc = dmpm.point_cloud_from_obj(opt.mpm_target_mesh_path, optinput.point_dx(opt), opt.p_density, opt.lam,
                                        opt.mu)
        c.rasterize_target(tpc["x"], optinput.point_mass(opt))
        c.set_params(**optinput.params(opt), adjoint="exact")
        c.setup(opt.num_timesteps + 1)
        assert c.forward(0) == dmpm.OK
        loss = c.loss()
        assert c.backward(0) == dmpm.OK
        g = c.control_grad(0)
    assert np.isfinite(loss) and loss > 0
    assert g.shape == (len(pc["x"]), 3, 3) and np.all(np.isfinite(g)) and np.abs(g).max() > 0


def test_oracle_jittered_points_stratified():
    """The restated jittered sampler: every kept point lies in its own sub-cell
    (one per sub-cell) and the count matches the sphere's volume."""
    obj, _, _ = _golden("sphere")
    V, F = omesh.read_obj(obj)
    cdx, per = 0.09, 2
    pts, dims = omesh.jittered_points(V, F, cdx, per, seed=1234)
    mn = V.min(axis=0).astype(np.float32)
    sdx = np.float32(cdx / per)
    cell = np.floor((pts - mn) / sdx).astype(np.int64)
    q = (cell[:, 0] * dims[1] + cell[:, 1]) * dims[2] + cell[:, 2]
    assert len(np.unique(q)) == len(q)
    r = (V.max(axis=0) - V.min(axis=0)).mean() / 2
    vol = 4 / 3 * np.pi * r ** 3
    assert abs(len(pts) * sdx ** 3 - vol) < 0.05 * vol


@pytest.mark.gpu
@pytest.mark.parametrize("name,per,seed", [("sphere", 2, 7), ("torus", 3, 2 ** 63 + 5)])
def test_gpu_jittered_points_match_oracle(gpu_ready, name, per, seed):
    obj, _, _ = _golden(name)
    V, F = dmpm.read_obj(obj)
    want, _ = omesh.jittered_points(V, F, 0.07, per, seed)
    got = dmpm.mesh_jittered_points(V, F, 0.07, per, seed)
    assert got.shape == want.shape and np.array_equal(got, want)
