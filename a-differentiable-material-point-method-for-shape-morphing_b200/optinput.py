"""The reference's optimisation input file (OptInput, DiffMPMAnimator3D/
MPMPolyscope.h:16-83) read and written in the layout cereal's JSON archive
gives it (DiffMPMAnimator3D.cpp:252-281): one top-level object "value0"
holding the fields in declaration order, each Vec3 as
{"value0": 3, "value1": x, "value2": y, "value3": z} (the reference's
cereal_eigen.h writes the row count, then the coefficients).

A caller holding an input.json of the reference sets up an engine context
from it with grid_dims / point_mass / params below, and turns the OBJ meshes
it names into point clouds with dmpm.point_cloud_from_obj(path, point_dx(opt),
opt.p_density, opt.lam, opt.mu) (the GPU lattice sampler); .mpmbin point
clouds are read and written by the C++ PointCloud of compat/.
"""
from __future__ import annotations

import dataclasses
import json
import math
from typing import Tuple

import numpy as np

Vec3 = Tuple[float, float, float]


@dataclasses.dataclass
class OptInput:
    """OptInput with the reference's defaults (MPMPolyscope.h:18-53)."""
    mpm_input_mesh_path: str = "experiments\\big_sca_demo\\input\\bob.obj"
    mpm_target_mesh_path: str = "experiments\\big_sca_demo\\input\\spot.obj"
    grid_dx: float = 1.0
    points_per_cell_cuberoot: int = 2
    grid_min_point: Vec3 = (-16.0, -16.0, -16.0)
    grid_max_point: Vec3 = (16.0, 16.0, 16.0)
    lam: float = 58333.0
    mu: float = 38888.9
    p_density: float = 40.0
    dt: float = 1.0 / 120.0
    drag: float = 0.5
    f_ext: Vec3 = (0.0, 0.0, 0.0)
    num_animations: int = 40
    num_timesteps: int = 30
    control_stride: int = 10
    max_gd_iters: int = 25
    max_ls_iters: int = 15
    initial_alpha: float = 0.1
    gd_tol: float = 1e-3
    smoothing_factor: float = 0.1


_VEC3 = ("grid_min_point", "grid_max_point", "f_ext")
_INT = ("points_per_cell_cuberoot", "num_animations", "num_timesteps", "control_stride", "max_gd_iters",
        "max_ls_iters")
_STR = ("mpm_input_mesh_path", "mpm_target_mesh_path")


def _f32(x: float) -> float:
    """The value a float member of the reference holds."""
    return float(np.float32(x))


def load(path: str) -> OptInput:
    """Read an OptInput written by the reference (or by save)."""
    with open(path) as f:
        doc = json.load(f)
    obj = doc["value0"] if "value0" in doc and isinstance(doc["value0"], dict) else doc
    kw = {}
    for fld in dataclasses.fields(OptInput):
        if fld.name not in obj:
            continue  # cereal's reader needs every field; a missing one keeps its default here
        v = obj[fld.name]
        if fld.name in _VEC3:
            if not (isinstance(v, dict) and v.get("value0") == 3):
                raise ValueError("%s: expected a cereal Vec3 object" % fld.name)
            kw[fld.name] = tuple(_f32(v["value%d" % i]) for i in (1, 2, 3))
        elif fld.name in _INT:
            kw[fld.name] = int(v)
        elif fld.name in _STR:
            kw[fld.name] = str(v)
        else:
            kw[fld.name] = _f32(v)
    return OptInput(**kw)


def save(opt: OptInput, path: str) -> None:
    """Write opt in cereal's JSON layout, readable by the reference."""
    body = {}
    for fld in dataclasses.fields(OptInput):
        v = getattr(opt, fld.name)
        if fld.name in _VEC3:
            body[fld.name] = {"value0": 3, "value1": _f32(v[0]), "value2": _f32(v[1]), "value3": _f32(v[2])}
        elif fld.name in _INT:
            body[fld.name] = int(v)
        elif fld.name in _STR:
            body[fld.name] = str(v)
        else:
            body[fld.name] = _f32(v)
    with open(path, "w") as f:
        json.dump({"value0": body}, f, indent=4)
        f.write("\n")


def grid_dims(opt: OptInput) -> Tuple[int, int, int]:
    """Grid nodes per axis as the reference computes them (MPMPolyscope.cpp:96-99):
    every axis uses the x extent, ceil((max[0] - min[0]) / grid_dx)."""
    d = int(math.ceil((_f32(opt.grid_max_point[0]) - _f32(opt.grid_min_point[0])) / _f32(opt.grid_dx)))
    return (d, d, d)


def point_dx(opt: OptInput) -> float:
    """Particle spacing grid_dx / points_per_cell_cuberoot (MPMPolyscope.cpp:64)."""
    return _f32(opt.grid_dx) / opt.points_per_cell_cuberoot


def point_mass(opt: OptInput) -> float:
    """Particle mass point_dx^3 * p_density (MPMPolyscope.cpp:51)."""
    pdx = point_dx(opt)
    return pdx * pdx * pdx * _f32(opt.p_density)


def params(opt: OptInput) -> dict:
    """Keyword arguments of dmpm.Context.set_params for this input: the
    simulation parameters OptimizeDefGradControlSequence receives
    (CompGraph.cpp:280-300) and its control stride as control frames."""
    return {"dt": _f32(opt.dt), "drag": _f32(opt.drag), "f_ext": tuple(_f32(x) for x in opt.f_ext),
            "smoothing": _f32(opt.smoothing_factor), "control": "per_layer",
            "control_stride": int(opt.control_stride)}
