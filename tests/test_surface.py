"""Headless surfacing (include/dmpm.h "surfaces") against the reference's own
code: MarchingCubesPointCloud's P2G_Mass / G2G_Mass fields and mesh, and
SphereUnionMarchingCubesSurfaceFromPointCloud's field and mesh, for the torus
point cloud (tests/golden/make_surface_golden.py runs the reference).

The oracle (oracle/surface.py) reproduces the reference's fields bit for bit:
its P2G_Mass and G2G_Mass masses equal the reference's, and libigl's marching
cubes of its sphere field gives the reference's mesh exactly (checked when the
goldens were made; the field's digest is stored).  The GPU fields must match:
G2G_Mass and the sphere field bit for bit, P2G_Mass up to the rounding of its
atomic sums.  The GPU extractor (marching tetrahedra) triangulates the same
level set as the reference's marching cubes differently, so the meshes are
compared geometrically: closed, consistently oriented, the same enclosed
volume within 1.5 % and area within 4 % (tetrahedral facets add about 2 %),
every vertex of each mesh within one grid spacing of the other mesh's
vertices."""
import hashlib
import os

import numpy as np
import pytest

import dmpm
from oracle import surface as osurf
from tests.helpers import GOLDEN


@pytest.fixture(scope="module")
def gold():
    g = dict(np.load(os.path.join(GOLDEN, "surface_torus.npz")))
    g["points"] = np.load(os.path.join(GOLDEN, "mesh_torus_points.npz"))["points"].astype(np.float32)
    g["fine_dx"] = np.float32(g["grid_dx"] / g["quality"])
    return g


def test_oracle_p2g_mass_matches_reference(gold):
    m = osurf.p2g_mass(gold["points"], 1.0, tuple(gold["coarse_dims"]), gold["grid_dx"], gold["box_min"])
    assert np.array_equal(m, gold["coarse_mass"])


def test_oracle_g2g_mass_matches_reference(gold):
    m = osurf.g2g_mass(gold["coarse_mass"], tuple(gold["coarse_dims"]), gold["grid_dx"], gold["box_min"],
                       tuple(gold["fine_dims"]), gold["fine_dx"], gold["box_min"])
    assert np.array_equal(m, gold["fine_mass"])


def test_oracle_sphere_field_is_the_pinned_field(gold):
    f = osurf.sphere_field(gold["points"], gold["sphere_radius"], gold["sphere_dx"], int(gold["blur"]),
                           gold["box_min"], tuple(gold["sphere_dims"]))
    assert hashlib.sha256(f.astype(np.float32).tobytes()).hexdigest() == str(gold["sphere_field_sha256"])


def _mesh_stats(V, F):
    V = np.asarray(V, dtype=np.float64)
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    cr = np.cross(b - a, c - a)
    area = 0.5 * np.linalg.norm(cr, axis=1).sum()
    vol = np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0
    return area, vol


def _closed_and_oriented(F):
    """Every directed edge once and its reverse once: a closed, consistently oriented surface."""
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
    key = e[:, 0].astype(np.int64) * (1 << 32) + e[:, 1]
    rev = e[:, 1].astype(np.int64) * (1 << 32) + e[:, 0]
    return len(np.unique(key)) == len(key) and np.array_equal(np.sort(key), np.sort(rev))


def _compare_meshes(V, F, Vr, Fr, dx):
    from scipy.spatial import cKDTree

    assert len(F) > 0 and _closed_and_oriented(F)
    area, vol = _mesh_stats(V, F)
    area_r, vol_r = _mesh_stats(Vr, Fr)
    d1, _ = cKDTree(Vr).query(V)
    d2, _ = cKDTree(V).query(Vr)
    stats = dict(area=area, area_ref=area_r, vol=vol, vol_ref=vol_r, d_to_ref=d1.max(), d_from_ref=d2.max(), dx=dx)
    assert vol > 0, stats  # normals point out of {field > iso}
    # the tetrahedral facets add a little area over the same level set (about 2 % here)
    assert abs(area - area_r) <= 0.04 * area_r, stats
    assert abs(vol - abs(vol_r)) <= 0.015 * abs(vol_r), stats
    assert d1.max() <= dx and d2.max() <= dx, stats


@pytest.mark.gpu
def test_gpu_mass_fields(gpu_ready, gold):
    dims = dmpm.surface_grid_dims(gold["box_min"], gold["box_max"], gold["grid_dx"])
    assert dims == tuple(gold["coarse_dims"])
    m = dmpm.p2g_mass(gold["points"], 1.0, dims, gold["grid_dx"], gold["box_min"])
    ref = gold["coarse_mass"]
    assert np.abs(m - ref).max() <= 2e-6 * ref.max()
    fine = dmpm.g2g_mass(ref, dims, gold["grid_dx"], gold["box_min"], tuple(gold["fine_dims"]), gold["fine_dx"],
                         gold["box_min"])
    assert np.array_equal(fine, gold["fine_mass"])


@pytest.mark.gpu
def test_gpu_sphere_field_bit_exact(gpu_ready, gold):
    f = dmpm.sphere_field(gold["points"], gold["sphere_radius"], int(gold["blur"]), tuple(gold["sphere_dims"]),
                          gold["sphere_dx"], gold["box_min"])
    assert hashlib.sha256(f.tobytes()).hexdigest() == str(gold["sphere_field_sha256"])


@pytest.mark.gpu
def test_gpu_marching_cubes_point_cloud_matches_reference_mesh(gpu_ready, gold, tmp_path):
    V, F = dmpm.marching_cubes_point_cloud(gold["points"], gold["iso_mass"], gold["grid_dx"], gold["quality"],
                                           gold["box_min"], gold["box_max"])
    _compare_meshes(V, F, gold["mass_V"].reshape(-1, 3), gold["mass_F"].reshape(-1, 3), gold["fine_dx"])
    path = str(tmp_path / "mass.obj")
    dmpm.write_obj(path, V, F)
    V2, F2 = dmpm.read_obj(path)
    assert np.allclose(V2, V) and np.array_equal(F2, F)


@pytest.mark.gpu
def test_gpu_sphere_union_surface_matches_reference_mesh(gpu_ready, gold):
    V, F = dmpm.sphere_union_surface(gold["points"], gold["sphere_radius"], gold["sphere_dx"], gold["sphere_iso"],
                                     int(gold["blur"]), gold["box_min"], gold["box_max"])
    _compare_meshes(V, F, gold["sphere_V"].reshape(-1, 3), gold["sphere_F"].reshape(-1, 3), gold["sphere_dx"])


@pytest.mark.gpu
def test_gpu_extract_small_cases(gpu_ready):
    """A ball's field: closed oriented mesh close to the sphere; empty and full fields give nothing."""
    n, dx = 24, 0.1
    mn = np.float32([-1.2, -1.2, -1.2])
    P = osurf.node_positions((n, n, n), dx, mn).astype(np.float64)
    f = (0.8 - np.linalg.norm(P, axis=1)).astype(np.float32)
    V, F = dmpm.extract_surface(f, (n, n, n), dx, mn, 0.0)
    assert _closed_and_oriented(F)
    r = np.linalg.norm(V.astype(np.float64), axis=1)
    assert np.abs(r - 0.8).max() < 0.02
    area, vol = _mesh_stats(V, F)
    assert abs(vol - 4 / 3 * np.pi * 0.8 ** 3) < 0.03 * vol
    for c in (-1.0, 1.0):
        V0, F0 = dmpm.extract_surface(np.full(n ** 3, c, np.float32), (n, n, n), dx, mn, 0.0)
        assert len(V0) == 0 and len(F0) == 0
    with pytest.raises(dmpm.DmpmError):
        dmpm.extract_surface(f, (n, n, n), -1.0, mn, 0.0)
    # output buffers too small: DMPM_ERR_TOO_LARGE with the sizes needed
    import ctypes

    lib = dmpm.load_library()
    d = np.int32([n, n, n])
    nv, nf = ctypes.c_int64(), ctypes.c_int64()
    Vs = np.empty((4, 3), np.float32)
    Fs = np.empty((4, 3), np.int32)
    st = lib.dmpm_surface_extract(f.ctypes.data, d.ctypes.data, dx, mn.ctypes.data, 0.0, Vs.ctypes.data, 4,
                                  Fs.ctypes.data, 4, ctypes.byref(nv), ctypes.byref(nf))
    assert st == dmpm.ERR_TOO_LARGE and (nv.value, nf.value) == (len(V), len(F))


@pytest.mark.gpu
def test_compat_cpp_surfacing(gpu_ready, gold, tmp_path):
    """SingleThreadMPM::P2G_Mass / G2G_Mass and SphereUnionMarchingCubesSurfaceFromPointCloud
    of the C++ compat API (tests/cpp/surface_check.cpp), called as the reference's GUI calls them."""
    import subprocess

    import build as pkg_build

    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    pkg = os.path.join(repo, "a-differentiable-material-point-method-for-shape-morphing_b200")
    pkg_build.build_compat()
    exe = str(tmp_path / "surface_check")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(pkg, "compat"), "-I",
                           os.path.join(repo, "include"), os.path.join(repo, "tests", "cpp", "surface_check.cpp"),
                           "-L", pkg, "-ldmpm_compat", "-ldmpm", "-Wl,-rpath," + pkg, "-o", exe])
    pf = tmp_path / "pts.f32"
    gold["points"].tofile(pf)
    out = tmp_path / "out.bin"
    subprocess.check_call([exe, str(pf), repr(float(gold["grid_dx"])), repr(float(gold["quality"])),
                           repr(float(gold["sphere_radius"])), repr(float(gold["sphere_dx"])),
                           repr(float(gold["sphere_iso"])), str(int(gold["blur"])), str(out)])
    fine, V, F = osurf.read_blocks(str(out), "ffi")
    ref = gold["fine_mass"]
    assert np.abs(fine - ref).max() <= 2e-6 * ref.max()  # P2G_Mass sums with float atomics
    Vp, Fp = dmpm.sphere_union_surface(gold["points"], gold["sphere_radius"], gold["sphere_dx"], gold["sphere_iso"],
                                       int(gold["blur"]), gold["box_min"], gold["box_max"])
    assert np.array_equal(V.reshape(-1, 3), Vp) and np.array_equal(F.reshape(-1, 3), Fp)
