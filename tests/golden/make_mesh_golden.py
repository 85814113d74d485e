"""Golden vectors of the mesh sampler: seeded watertight test meshes (OBJ)
and the points the reference's own GeneratePointCloudFromWatertightTriangleMesh
(GeometryLoading.cpp:10-83, built by oracle/build_ref_mesh.sh) keeps for them.

    bash oracle/build_ref_mesh.sh && python tests/golden/make_mesh_golden.py

Sizes are deliberately not round numbers, so no lattice point lies on the
surface (there the reference's result depends on the rounding of its
float closest-point search).
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_MESH = os.path.join(REPO, "oracle", "_ref", "ref_mesh")


def uv_sphere(center, radius_fn, n_lat=18, n_lon=28):
    """Closed, outward-oriented triangle mesh of a star-shaped surface r(theta, phi)."""
    verts = [np.asarray(center) + np.array([0.0, 0.0, radius_fn(0.0, 0.0)])]
    for i in range(1, n_lat):
        th = np.pi * i / n_lat
        for j in range(n_lon):
            ph = 2 * np.pi * j / n_lon
            r = radius_fn(th, ph)
            verts.append(np.asarray(center) + r * np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)]))
    verts.append(np.asarray(center) + np.array([0.0, 0.0, -radius_fn(np.pi, 0.0)]))
    V = np.array(verts)
    F = []
    ring = lambda i, j: 1 + (i - 1) * n_lon + (j % n_lon)
    for j in range(n_lon):
        F.append((0, ring(1, j), ring(1, j + 1)))
    for i in range(1, n_lat - 1):
        for j in range(n_lon):
            a, b, c, d = ring(i, j), ring(i, j + 1), ring(i + 1, j), ring(i + 1, j + 1)
            F.append((a, c, b))
            F.append((b, c, d))
    last = len(V) - 1
    for j in range(n_lon):
        F.append((last, ring(n_lat - 1, j + 1), ring(n_lat - 1, j)))
    return V, np.array(F)


def torus(center, R, r, n_u=36, n_v=16, tilt=0.37):
    V = []
    for i in range(n_u):
        u = 2 * np.pi * i / n_u
        for j in range(n_v):
            v = 2 * np.pi * j / n_v
            V.append([(R + r * np.cos(v)) * np.cos(u), (R + r * np.cos(v)) * np.sin(u), r * np.sin(v)])
    V = np.array(V)
    c, s = np.cos(tilt), np.sin(tilt)
    V = V @ np.array([[1, 0, 0], [0, c, -s], [0, s, c]]).T + np.asarray(center)
    idx = lambda i, j: (i % n_u) * n_v + (j % n_v)
    F = []
    for i in range(n_u):
        for j in range(n_v):
            a, b, cc, d = idx(i, j), idx(i + 1, j), idx(i, j + 1), idx(i + 1, j + 1)
            F.append((a, b, d))
            F.append((a, d, cc))
    return V, np.array(F)


def oriented(V, F):
    """Flip every face if the signed volume is negative (outward normals)."""
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    vol = np.sum(np.einsum("ij,ij->i", a, np.cross(b, c))) / 6.0
    return F if vol > 0 else F[:, ::-1].copy()


def write_obj(path, V, F):
    with open(path, "w") as f:
        for v in V:
            f.write("v %.9g %.9g %.9g\n" % tuple(v))
        for t in F:
            f.write("f %d %d %d\n" % tuple(t + 1))


def meshes():
    out = {}
    V, F = uv_sphere((0.1037, -0.2113, 0.0519), lambda th, ph: 0.3137)
    out["sphere"] = (V, oriented(V, F), 0.0213)
    V, F = uv_sphere((0.0, 0.0, 0.0), lambda th, ph: 0.2971 * (1.0 + 0.3 * np.sin(3 * th) * np.sin(2 * ph)))
    out["bumpy"] = (V, oriented(V, F), 0.0187)
    V, F = torus((0.0213, 0.0117, -0.0371), 0.4119, 0.1307)
    out["torus"] = (V, oriented(V, F), 0.0231)
    return out


if __name__ == "__main__":
    if not os.path.exists(REF_MESH):
        sys.exit("build the reference sampler first: bash oracle/build_ref_mesh.sh")
    for name, (V, F, dx) in meshes().items():
        obj = os.path.join(HERE, "mesh_%s.obj" % name)
        write_obj(obj, V, F)
        tmp = os.path.join(HERE, "mesh_%s.tmp" % name)
        subprocess.check_call([REF_MESH, obj, "%.9g" % dx, tmp], stdout=subprocess.DEVNULL)
        pts = np.fromfile(tmp, dtype=np.float32).reshape(-1, 3)
        os.remove(tmp)
        np.savez_compressed(os.path.join(HERE, "mesh_%s_points.npz" % name), points=pts, point_dx=np.float32(dx))
        print(name, len(V), "vertices", len(F), "faces", len(pts), "points")
