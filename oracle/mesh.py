"""CPU restatement of the reference's mesh-to-point-cloud sampler (test
infrastructure only): LoadMPMPointCloudFromObj (MPMPolyscope.cpp:10-60) reads
an OBJ, takes the float bounding box of its vertices, and
GeneratePointCloudFromWatertightTriangleMesh (GeometryLoading.cpp:10-83) keeps
every point of the lattice min + point_dx (i, j, k), i < ceil((max - min) /
point_dx) + 1 per axis, whose signed distance to the mesh is <= 0 with the
winding-number sign of libigl's signed_distance: s = 1 - 2 w, S = s |d|, so a
point is kept when its winding number w >= 1/2 or it lies on the surface.

The winding number is the sum of the triangles' solid angles / 4 pi, each by
the formula of Van Oosterom and Strackee (1983):
tan(Omega / 2) = a.(b x c) / (|a||b||c| + (a.b)|c| + (b.c)|a| + (c.a)|b|),
a, b, c the vertices relative to the point, evaluated in float64.
Pinned against the reference's own sampler in tests/test_mesh_sampler.py.
"""
from __future__ import annotations

import numpy as np


def read_obj(path):
    """Vertices (float32, as the reference's Eigen::MatrixXf) and triangles of
    the 'v' and 'f' lines of an OBJ file (1-based indices, v/vt/vn forms)."""
    V, F = [], []
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            if t[0] == "v":
                V.append([float(x) for x in t[1:4]])
            elif t[0] == "f":
                idx = [int(x.split("/")[0]) for x in t[1:]]
                idx = [i - 1 if i > 0 else len(V) + i for i in idx]
                for k in range(1, len(idx) - 1):  # fan for polygons
                    F.append([idx[0], idx[k], idx[k + 1]])
    return np.asarray(V, dtype=np.float32), np.asarray(F, dtype=np.int64)


def lattice(V, point_dx):
    """Float32 lattice of the reference: bounding box, dims, coordinates."""
    dx = np.float32(point_dx)
    mn = V.min(axis=0).astype(np.float32)
    mx = V.max(axis=0).astype(np.float32)
    dims = [int(np.ceil(np.float32(mx[i] - mn[i]) / dx)) + 1 for i in range(3)]
    axes = [np.float32(mn[i]) + np.arange(dims[i], dtype=np.float32) * dx for i in range(3)]
    return mn, dims, axes


def winding_numbers(P, V, F, chunk=1024):
    a0 = V[F[:, 0]].astype(np.float64)
    b0 = V[F[:, 1]].astype(np.float64)
    c0 = V[F[:, 2]].astype(np.float64)
    w = np.empty(len(P))
    for s in range(0, len(P), chunk):
        p = P[s:s + chunk, None, :].astype(np.float64)
        a, b, c = a0[None] - p, b0[None] - p, c0[None] - p
        la, lb, lc = (np.linalg.norm(x, axis=2) for x in (a, b, c))
        num = np.einsum("ijk,ijk->ij", a, np.cross(b, c))
        den = la * lb * lc + np.einsum("ijk,ijk->ij", a, b) * lc + np.einsum("ijk,ijk->ij", b, c) * la + \
            np.einsum("ijk,ijk->ij", c, a) * lb
        w[s:s + chunk] = np.sum(2.0 * np.arctan2(num, den), axis=1) / (4.0 * np.pi)
    return w


def lattice_points(V, F, point_dx):
    """The points the reference keeps, in its lattice order (i, then j, then k)."""
    mn, dims, axes = lattice(V, point_dx)
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    P = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    keep = winding_numbers(P, V, F) >= 0.5
    return P[keep]


_M64 = 0xFFFFFFFFFFFFFFFF


def splitmix64(z):
    """SplitMix64's finaliser (Steele, Lea and Flood 2014) on uint64 arrays."""
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def jittered_points(V, F, cell_dx, per_axis, seed, min_point=None, max_point=None):
    """dmpm_mesh_jittered_points restated: one point per sub-cell at
    min + (index + u) * sdx (float32), u from splitmix64(seed + 3 q + axis),
    kept where the winding number is >= 1/2, in sub-cell order."""
    V = np.asarray(V, dtype=np.float32)
    mn = np.asarray(V.min(axis=0) if min_point is None else min_point, dtype=np.float32)
    mx = np.asarray(V.max(axis=0) if max_point is None else max_point, dtype=np.float32)
    cdx = np.float32(cell_dx)
    dims = [int(np.ceil(np.float32(mx[a] - mn[a]) / cdx)) * per_axis for a in range(3)]
    sdx = np.float32(cdx / np.float32(per_axis))
    I, J, K = np.meshgrid(*(np.arange(d, dtype=np.int64) for d in dims), indexing="ij")
    idx = np.stack([I.ravel(), J.ravel(), K.ravel()], axis=1)
    q = ((idx[:, 0] * dims[1] + idx[:, 1]) * dims[2] + idx[:, 2]).astype(np.uint64)
    P = np.empty((len(q), 3), dtype=np.float32)
    with np.errstate(over="ignore"):
        base = np.uint64(int(seed) & _M64) + np.uint64(3) * q
        for a in range(3):
            u = (splitmix64(base + np.uint64(a)) >> np.uint64(40)).astype(np.float32) * np.float32(1.0 / 16777216.0)
            P[:, a] = mn[a] + (idx[:, a].astype(np.float32) + u) * sdx
    keep = winding_numbers(P, V, F) >= 0.5
    return P[keep], dims
