"""Seeded synthetic morphing scenes in lattice units.

The reference builds its scenes from OBJ meshes (MPMPolyscope.cpp:11-55,
59-167): points on a regular sub-cell lattice inside a watertight mesh, mass
density * point_dx^3, F = I, Lame parameters from (E, nu), a grid of
ceil((max-min)/dx) nodes per axis, particle volumes from
CalculatePointCloudVolumes and a target grid rasterised by a mass-only P2G of
target sample points.  The meshes themselves are not part of the reference
tree, so scenes here are analytic shapes (sphere, ellipsoid, box, torus,
capsule, unions) sampled the same way.

Units.  The reference computes a particle volume as m_p / sum_g w m_g
(ForwardSimulation.cpp:262-290), which is a volume only when dx = 1.  Scenes
are therefore expressed in lattice units: x' = x / dx, dx' = 1, grid minimum
0, E' = E * dx; masses stay rho * (dx / r)^3 for r^3 particles per cell and dt
is unchanged.  These are the same dynamics as the physical scene.

Sampling is jittered stratified: each cell is split into r x r x r sub-cells and
every sub-cell receives one uniformly jittered point, kept when it falls inside
the shape.  Target samples are the un-jittered sub-cell centres.

All matrices here are numpy (N, 3, 3) arrays indexed [p, row, col]; the C ABI
takes them column-major, see `to_colmajor`.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np

Shape = Callable[[np.ndarray], np.ndarray]  # (K, 3) unit-box coords -> bool mask


# ---------------------------------------------------------------- shapes
def sphere(c, r) -> Shape:
    c = np.asarray(c, dtype=np.float64)
    return lambda p: np.sum((p - c) ** 2, axis=1) <= r * r


def ellipsoid(c, axes) -> Shape:
    c = np.asarray(c, dtype=np.float64)
    a = np.asarray(axes, dtype=np.float64)
    return lambda p: np.sum(((p - c) / a) ** 2, axis=1) <= 1.0


def box(c, half) -> Shape:
    c = np.asarray(c, dtype=np.float64)
    h = np.broadcast_to(np.asarray(half, dtype=np.float64), (3,))
    return lambda p: np.all(np.abs(p - c) <= h, axis=1)


def cube(c, side) -> Shape:
    return box(c, 0.5 * side)


def torus(c, R, r, axis=2) -> Shape:
    c = np.asarray(c, dtype=np.float64)

    def f(p):
        q = p - c
        ax = q[:, axis]
        rad = np.sqrt(np.sum(np.delete(q, axis, axis=1) ** 2, axis=1))
        return (rad - R) ** 2 + ax ** 2 <= r * r

    return f


def capsule(c, length, r, axis=0) -> Shape:
    c = np.asarray(c, dtype=np.float64)

    def f(p):
        q = p - c
        t = np.clip(q[:, axis], -0.5 * length, 0.5 * length)
        d = q.copy()
        d[:, axis] -= t
        return np.sum(d * d, axis=1) <= r * r

    return f


def union(*shapes: Shape) -> Shape:
    def f(p):
        m = np.zeros(len(p), dtype=bool)
        for s in shapes:
            m |= s(p)
        return m

    return f


# ---------------------------------------------------------------- sampling
def sample_points(shape: Shape, res: int, ppc_root: int, rng: Optional[np.random.Generator],
                  bbox: Tuple[np.ndarray, np.ndarray] = None) -> np.ndarray:
    """Jittered (rng given) or centred (rng None) stratified samples in lattice units."""
    lo = np.zeros(3) if bbox is None else np.floor(np.asarray(bbox[0]) * res).astype(int)
    hi = np.full(3, res) if bbox is None else np.ceil(np.asarray(bbox[1]) * res).astype(int)
    lo = np.clip(lo, 0, res)
    hi = np.clip(hi, 0, res)
    r = ppc_root
    out: List[np.ndarray] = []
    sub = np.stack(np.meshgrid(np.arange(r), np.arange(r), np.arange(r), indexing="ij"), -1).reshape(-1, 3)
    for i in range(lo[0], hi[0]):  # one x-slab of cells at a time bounds memory
        jj, kk = np.meshgrid(np.arange(lo[1], hi[1]), np.arange(lo[2], hi[2]), indexing="ij")
        cells = np.stack([np.full(jj.size, i), jj.ravel(), kk.ravel()], -1)
        if cells.size == 0:
            continue
        pts = (cells[:, None, :] * r + sub[None, :, :]).reshape(-1, 3).astype(np.float64)
        if rng is None:
            pts += 0.5
        else:
            pts += rng.random(pts.shape)
        pts /= r
        keep = shape(pts / res)
        out.append(pts[keep])
    return np.concatenate(out, 0) if out else np.zeros((0, 3))


def lame(E: float, nu: float) -> Tuple[float, float]:
    """CalculateLameParameters (Elasticity.cpp:231-235)."""
    return E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), E / (2.0 + 2.0 * nu)


# ---------------------------------------------------------------- scene
@dataclasses.dataclass
class Scene:
    name: str
    x: np.ndarray           # (N, 3) lattice units
    v: np.ndarray           # (N, 3)
    F: np.ndarray           # (N, 3, 3)
    C: np.ndarray           # (N, 3, 3)
    dFc: np.ndarray         # (N, 3, 3)
    m: np.ndarray           # (N,)
    lam: np.ndarray         # (N,)
    mu: np.ndarray          # (N,)
    vol: np.ndarray         # (N,) zeros until computed (CalculatePointCloudVolumes)
    dims: Tuple[int, int, int]
    dx: float
    min_point: np.ndarray   # (3,)
    target_points: np.ndarray  # (M, 3) lattice units
    target_mp: float
    dt: float
    steps: int
    drag: float = 0.0
    f_ext: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(3))
    smoothing: float = 0.0
    checkpoint_every: int = 0
    meta: Dict = dataclasses.field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    @property
    def num_nodes(self) -> int:
        return int(np.prod(self.dims))

    def float32_inputs(self) -> "Scene":
        """A copy whose per-particle inputs are float32-representable (each
        value rounded to the nearest float).  The FP32-mixed path rounds its
        inputs so on upload; giving the FP64 path this copy too makes the two
        paths compute from identical inputs."""
        r = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
        out = dataclasses.replace(self)
        for k in ("x", "v", "F", "C", "dFc", "m", "lam", "mu", "vol"):
            setattr(out, k, r(getattr(self, k)))
        return out

    def cfl_dt(self) -> float:
        """Explicit P-wave limit dx / c_p in these (lattice) units."""
        rho = float(self.m.mean()) / (1.0 / self.meta.get("ppc", 8))  # lattice density
        c = math.sqrt((float(self.lam.mean()) + 2.0 * float(self.mu.mean())) / rho)
        return self.dx / c


def make_scene(name: str, shape: Shape, target: Shape, res: int, ppc_root: int, E: float, nu: float,
               dt: float, steps: int, seed: int, rho: float = 1.0, dfc_std: float = 1e-3,
               drag: float = 0.0, smoothing: float = 0.0, f_ext=(0.0, 0.0, 0.0),
               checkpoint_every: int = 0, bbox=None, target_bbox=None, dims=None) -> Scene:
    rng = np.random.default_rng(seed)
    x = sample_points(shape, res, ppc_root, rng, bbox)
    n = x.shape[0]
    dx_phys = 1.0 / res
    lam, mu = lame(E * dx_phys, nu)
    mp = rho * (dx_phys / ppc_root) ** 3
    F = np.broadcast_to(np.eye(3), (n, 3, 3)).copy()
    dFc = rng.normal(0.0, dfc_std, size=(n, 3, 3)) if dfc_std > 0 else np.zeros((n, 3, 3))
    tp = sample_points(target, res, ppc_root, None, target_bbox)
    d = tuple(dims) if dims is not None else (res, res, res)
    return Scene(name=name, x=x, v=np.zeros((n, 3)), F=F, C=np.zeros((n, 3, 3)), dFc=dFc,
                 m=np.full(n, mp), lam=np.full(n, lam), mu=np.full(n, mu), vol=np.zeros(n),
                 dims=d, dx=1.0, min_point=np.zeros(3), target_points=tp, target_mp=mp, dt=dt,
                 steps=steps, drag=drag, f_ext=np.asarray(f_ext, dtype=np.float64), smoothing=smoothing,
                 checkpoint_every=checkpoint_every,
                 meta={"res": res, "ppc": ppc_root ** 3, "E": E, "nu": nu, "seed": seed})


def _bb(c, h):
    c = np.asarray(c, dtype=np.float64)
    h = np.asarray(h, dtype=np.float64)
    return (c - h, c + h)


# Density of the 128^3 and 256^3 scenes: the reference's default p_density
# (DiffMPMAnimator3D/MPMPolyscope.h:37).  With density 1, the value the small
# scenes use, a fully covered node of a 256^3 unit box holds 1/256^3 = 6e-8,
# below the FLT_EPSILON node-mass threshold of the grid update
# (ForwardSimulation.cpp:55, BackPropagation.cpp:55) and of the volume
# estimate (ForwardSimulation.cpp:288): every node would count as empty, every
# volume would be zero and the rollout would not move.  At 128^3 a full node
# holds 4.8e-7, so the partly covered surface nodes cross the threshold from
# step to step: the 500-step gradient of the three-sphere scene then changes
# by 1e-6 (relative) between two FP64 runs that differ only in atomic
# summation order, against 2e-11 at density 40.
LARGE_SCENE_DENSITY = 40.0


def config_scene(config: int, instance: int = 0, ppc_root: Optional[int] = None) -> Scene:
    """The five benchmark configurations as seeded scenes (seed = 1000*config + instance)."""
    seed = 1000 * config + instance
    c = (0.5, 0.5, 0.5)
    if config == 0:
        return make_scene("sphere_r0.2_32^3", sphere(c, 0.2), cube(c, 0.35), 32, ppc_root or 2, 1e4, 0.3,
                          1e-3, 100, seed, bbox=_bb(c, 0.2), target_bbox=_bb(c, 0.175))
    if config == 1:
        return make_scene("ellipsoid_0.3x0.2x0.15_64^3", ellipsoid(c, (0.3, 0.2, 0.15)), torus(c, 0.25, 0.08),
                          64, ppc_root or 3, 1e4, 0.3, 5e-4, 200, seed, bbox=_bb(c, (0.3, 0.2, 0.15)),
                          target_bbox=_bb(c, (0.33, 0.33, 0.08)))
    if config == 2:
        rng = np.random.default_rng(seed + 7)
        cs = rng.uniform(0.25, 0.75, size=(3, 3))
        rs = rng.uniform(0.1, 0.2, size=3)
        shp = union(*[sphere(cs[k], rs[k]) for k in range(3)])
        lo = np.min(cs - rs[:, None], 0)
        hi = np.max(cs + rs[:, None], 0)
        return make_scene("3spheres_128^3", shp, capsule(c, 0.5, 0.15), 128, ppc_root or 2, 5e4, 0.35,
                          2.5e-4, 500, seed, rho=LARGE_SCENE_DENSITY, checkpoint_every=25, bbox=(lo, hi),
                          target_bbox=_bb(c, (0.4, 0.15, 0.15)))
    if config == 4:
        return make_scene("sphere_r0.2423_256^3", sphere(c, 0.2423), torus(c, 0.3, 0.1), 256, ppc_root or 2,
                          1e4, 0.3, 1.25e-4, 400, seed, rho=LARGE_SCENE_DENSITY, checkpoint_every=20,
                          bbox=_bb(c, 0.2423),
                          target_bbox=_bb(c, (0.4, 0.4, 0.1)))
    raise ValueError("config %d is not a single-instance scene; see batch_scenes" % config)


def batch_scenes(count: int = 48, seed_base: int = 3000) -> List[Scene]:
    """Config 3: seeded sphere / ellipsoid / box instances with particle counts
    log-uniform in [5k, 150k], grids 32^3 or 64^3, 100-300 steps, dt = 5e-4."""
    out = []
    for inst in range(count):
        rng = np.random.default_rng(seed_base + inst)
        res = int(rng.choice([32, 64]))
        kind = int(rng.integers(0, 3))
        n_target = math.exp(rng.uniform(math.log(5e3), math.log(1.5e5)))
        ppc_root = 2 if n_target / 8 <= 0.3 * res ** 3 else 3
        vol_frac = n_target / (ppc_root ** 3 * res ** 3)
        c = (0.5, 0.5, 0.5)
        if kind == 0:
            r = min((3 * vol_frac / (4 * math.pi)) ** (1 / 3), 0.4)
            shp, bb = sphere(c, r), _bb(c, r)
            tgt, tbb = sphere(c, 0.8 * r), _bb(c, 0.8 * r)
        elif kind == 1:
            s = min((3 * vol_frac / (4 * math.pi * 0.3 * 0.2 * 0.15)) ** (1 / 3), 1.3)
            ax = (0.3 * s, 0.2 * s, 0.15 * s)
            shp, bb = ellipsoid(c, ax), _bb(c, ax)
            tgt, tbb = ellipsoid(c, ax[::-1]), _bb(c, ax[::-1])
        else:
            h = min(0.5 * vol_frac ** (1 / 3), 0.4)
            shp, bb = box(c, h), _bb(c, h)
            tgt, tbb = box(c, (1.2 * h, 0.8 * h, h)), _bb(c, (1.2 * h, 0.8 * h, h))
        steps = int(rng.integers(100, 301))
        sc = make_scene("batch%02d" % inst, shp, tgt, res, ppc_root, 1e4, 0.3, 5e-4, steps, seed_base + inst,
                        bbox=bb, target_bbox=tbb)
        out.append(sc)
    return out


def small_scene(seed: int = 0, res: int = 16, radius: float = 0.2, ppc_root: int = 2, E: float = 1e4,
                nu: float = 0.3, dt: float = 2e-4, steps: int = 4, dfc_std: float = 1e-3,
                drag: float = 0.0, smoothing: float = 0.0, f_ext=(0.0, 0.0, 0.0), v_std: float = 0.0,
                offset=(0.0, 0.0, 0.0)) -> Scene:
    """Small sphere-to-cube scene for parity tests (a few hundred particles)."""
    c = tuple(0.5 + o for o in offset)
    sc = make_scene("small_s%d" % seed, sphere(c, radius), cube(c, 1.6 * radius), res, ppc_root, E, nu, dt,
                    steps, seed, dfc_std=dfc_std, drag=drag, smoothing=smoothing, f_ext=f_ext,
                    bbox=_bb(c, radius), target_bbox=_bb(c, 0.8 * radius))
    if v_std > 0:
        rng = np.random.default_rng(seed + 99)
        sc.v = rng.normal(0.0, v_std, size=(sc.n, 3))
    return sc


# ---------------------------------------------------------------- layout helpers
def to_colmajor(M: np.ndarray) -> np.ndarray:
    """(N, 3, 3) [p, row, col] -> (N, 9) column-major (Eigen::Matrix3f storage)."""
    return np.ascontiguousarray(np.asarray(M).transpose(0, 2, 1).reshape(-1, 9))


def from_colmajor(a: np.ndarray) -> np.ndarray:
    return np.asarray(a).reshape(-1, 3, 3).transpose(0, 2, 1)
