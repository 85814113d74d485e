"""Oracle (test infrastructure only): CPU restatement of the reference's
headless surfacing fields, in float32 with the reference's operation order so
the results are bit-identical to its serial build.

  p2g_mass      SingleThreadMPM::P2G_Mass (ForwardSimulation.cpp:292-327)
  g2g_mass      SingleThreadMPM::G2G_Mass (ForwardSimulation.cpp:329-367)
  sphere_field  the scalar field of SphereUnionMarchingCubesSurfaceFromPointCloud
                (SphereUnionSurfacing.cpp:7-106): max over points of radius - |x - p|
                inside each sphere, then `blur_iterations` passes of the 27-node box
                sum divided by 9 on interior nodes (border nodes keep their values)
  grid_dims     the reference's ceil((max_x - min_x) / dx) on every axis
                (SphereUnionSurfacing.cpp:13-16, DiffMPMAnimator3D.cpp:494-497)

Grid arrays are flat in the reference's node order (i * dim_y + j) * dim_z + k,
node (i, j, k) at min + (i, j, k) * dx (Grid.cpp:21, SphereUnionSurfacing.cpp:62).
"""
from __future__ import annotations

import math
from typing import Sequence, Tuple

import numpy as np

F32 = np.float32


def cubic_bspline(x: np.ndarray) -> np.ndarray:
    """CubicBSpline (Interpolation.h:5-17) elementwise in float32."""
    x = np.abs(np.asarray(x, dtype=F32))
    inner = (F32(0.5) * x * x * x - x * x) + F32(2.0 / 3.0)
    t = F32(2.0) - x
    outer = t * t * t / F32(6.0)
    return np.where(x < F32(1.0), inner, np.where(x < F32(2.0), outer, F32(0.0))).astype(F32)


def grid_dims(min_point: Sequence[float], max_point: Sequence[float], dx: float) -> Tuple[int, int, int]:
    d = int(math.ceil(float((F32(max_point[0]) - F32(min_point[0])) / F32(dx))))
    return (d, d, d)


def node_positions(dims, dx, min_point) -> np.ndarray:
    """(prod(dims), 3) float32 node positions min + (i, j, k) * dx."""
    dx = F32(dx)
    mn = np.asarray(min_point, dtype=F32)
    axes = [mn[c] + np.arange(dims[c], dtype=F32) * dx for c in range(3)]
    I, J, K = np.meshgrid(axes[0], axes[1], axes[2], indexing="ij")
    return np.stack([I.ravel(), J.ravel(), K.ravel()], axis=1).astype(F32)


def _stencil(xp: np.ndarray, dims, dx, min_point):
    """For query points xp (n, 3) float32: the 64 stencil node offsets in the
    reference's order (Grid.cpp:40-79), as (flat node index (n, 64), valid mask,
    weight (n, 64)) with weights CubicBSpline((xg - xp) / dx) multiplied over axes."""
    dx = F32(dx)
    mn = np.asarray(min_point, dtype=F32)
    rel = (xp - mn).astype(F32)
    base = np.floor(rel / dx).astype(np.int64) - 1
    idx = np.empty((len(xp), 64), dtype=np.int64)
    ok = np.empty((len(xp), 64), dtype=bool)
    w = np.empty((len(xp), 64), dtype=F32)
    o = 0
    for i in range(4):
        for j in range(4):
            for k in range(4):
                n = base + np.array([i, j, k])
                valid = np.all((n >= 0) & (n < np.asarray(dims)), axis=1)
                xg = (mn + n.astype(F32) * dx).astype(F32)
                d = ((xg - xp) / dx).astype(F32)
                b = cubic_bspline(d)
                w[:, o] = (b[:, 0] * b[:, 1]) * b[:, 2]
                idx[:, o] = (n[:, 0] * dims[1] + n[:, 1]) * dims[2] + n[:, 2]
                ok[:, o] = valid
                o += 1
    return idx, ok, w


def p2g_mass(points, mp_m: float, dims, dx: float, min_point) -> np.ndarray:
    """Node masses sum_p w(x_g - x_p) mp_m, accumulated point by point in stencil order."""
    xp = np.asarray(points, dtype=F32).reshape(-1, 3)
    idx, ok, w = _stencil(xp, dims, dx, min_point)
    m = np.zeros(int(np.prod(dims)), dtype=F32)
    contrib = (w * F32(mp_m)).astype(F32)
    np.add.at(m, idx[ok], contrib[ok])  # sequential, in (point, stencil) order
    return m


def g2g_mass(m1, dims1, dx1: float, min1, dims2, dx2: float, min2) -> np.ndarray:
    """Masses of grid 2's nodes: sum over grid 1's stencil of w * m1 (weights with dx1)."""
    m1 = np.asarray(m1, dtype=F32)
    xq = node_positions(dims2, dx2, min2)
    idx, ok, w = _stencil(xq, dims1, dx1, min1)
    acc = np.zeros(len(xq), dtype=F32)
    for o in range(64):
        term = np.where(ok[:, o], w[:, o] * m1[np.where(ok[:, o], idx[:, o], 0)], F32(0.0)).astype(F32)
        acc = (acc + term).astype(F32)
    return acc


def sphere_field(points, radius: float, dx: float, blur_iterations: int, min_point, dims) -> np.ndarray:
    pts = np.asarray(points, dtype=F32).reshape(-1, 3)
    r = F32(radius)
    dx = F32(dx)
    mn = np.asarray(min_point, dtype=F32)
    n0, n1, n2 = dims
    g = np.zeros(dims, dtype=F32)
    for p in pts:
        lo = np.ceil(((p - r) - mn) / dx).astype(np.int64)
        hi = np.ceil(((p + r) - mn) / dx).astype(np.int64)
        lo = np.maximum(lo, 0)
        hi = np.minimum(hi, np.asarray(dims) - 1)
        if np.any(hi < lo):
            continue
        ax = [mn[c] + np.arange(lo[c], hi[c] + 1).astype(F32) * dx for c in range(3)]
        d0 = (ax[0] - p[0])[:, None, None]
        d1 = (ax[1] - p[1])[None, :, None]
        d2 = (ax[2] - p[2])[None, None, :]
        # Eigen's squaredNorm of a 3-vector sums its unrolled halves: d0^2 + (d1^2 + d2^2)
        sq = (d0 * d0 + (d1 * d1 + d2 * d2)).astype(F32)
        val = np.where(sq <= r * r, (r - np.sqrt(sq)).astype(F32), F32(0.0))
        sl = g[lo[0]:hi[0] + 1, lo[1]:hi[1] + 1, lo[2]:hi[2] + 1]
        np.maximum(sl, np.where(sq <= r * r, val, sl), out=sl)
    blurred = g.copy()
    for _ in range(blur_iterations):
        acc = np.zeros((n0 - 2, n1 - 2, n2 - 2), dtype=F32)
        for a in (-1, 0, 1):
            for b in (-1, 0, 1):
                for c in (-1, 0, 1):
                    acc = (acc + g[1 + a:n0 - 1 + a, 1 + b:n1 - 1 + b, 1 + c:n2 - 1 + c]).astype(F32)
        blurred[1:-1, 1:-1, 1:-1] = (acc.astype(np.float64) / 9.0).astype(F32)
        g = blurred.copy()
    return g.ravel()


def read_blocks(path: str, kinds: Sequence[str]):
    """Blocks <int64 count><count values> of the reference driver's output files."""
    out = []
    with open(path, "rb") as f:
        for kind in kinds:
            n = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
            dt = {"f": np.float32, "i": np.int32, "l": np.int64}[kind]
            out.append(np.frombuffer(f.read(n * np.dtype(dt).itemsize), dtype=dt).copy())
    return out
