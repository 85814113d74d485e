"""Compensated positions of the FP32-mixed engine (kernels.cuh: load_xd,
stencil_coord): every position coordinate is kept as two floats hi + lo, the
stencil of a particle is formed from its lattice coordinate in FP64, and G2P
advances x in FP64 before splitting it again.  Positions therefore go in and
come back at double-float precision, and a scene far from the grid origin --
where a float32 position is rounded to a large fraction of a cell -- matches
the FP64 oracle (the CPU restatement of the reference's ForwardTimeStep /
EndLayerMassLoss / Back_Timestep) as closely as one near it."""
import dataclasses

import numpy as np
import pytest

import dmpm
import scenes
from oracle.lib import OracleGraph
from tests.helpers import normrel, relerr
from tests.test_gpu_parity import make_ctx

pytestmark = pytest.mark.gpu

OFFSET = (3000.0, -2000.0, 1000.0)  # lattice units (cells of dx = 1)


def _scene(offset):
    """A 2,146-particle sphere on a 16^3 grid, with the grid and everything in
    it moved by offset."""
    sc = scenes.small_scene(seed=31, res=16, radius=0.25, steps=12, v_std=0.5, drag=0.1, smoothing=0.05,
                            f_ext=(0.0, -1.0, 0.0))
    off = np.asarray(offset, dtype=np.float64)
    sc = dataclasses.replace(sc, x=sc.x + off, target_points=sc.target_points + off,
                             min_point=np.asarray(sc.min_point, dtype=np.float64) + off)
    sc.vol = OracleGraph(sc, "f64").calc_volumes()
    return sc


def _oracle(sc, L):
    o = OracleGraph(sc, "f64")
    o.setup(L, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
    o.forward(0)
    loss = o.loss()
    o.backward(0, 1)
    return o, loss


def _fp32(sc, target, L, **params):
    with make_ctx(sc, "fp32", target, adjoint="exact", control="tied", **params) as c:
        c.setup(L)
        assert c.forward(0) == dmpm.OK
        lo = c.loss()
        assert c.backward(0) == dmpm.OK
        return {"loss": lo, "x0": c.get(0, "x"), "x": c.get(L - 1, "x"), "F": c.get(L - 1, "F"),
                "dLdx": c.get(0, "dLdx"), "grad": c.control_grad()}


def test_positions_round_trip_at_double_float_precision(gpu_ready):
    """Uploaded FP64 positions read back to ~2^-48 of their size, far below the
    float32 rounding of the same values; set_layer stores them the same way."""
    sc = _scene(OFFSET)
    with make_ctx(sc, "fp32", np.zeros(int(np.prod(sc.dims)))) as c:
        c.setup(3)
        x0 = c.get(0, "x")
        scale = np.abs(sc.x).max()
        f32 = np.abs(sc.x.astype(np.float32).astype(np.float64) - sc.x).max()
        assert np.abs(x0 - sc.x).max() <= 2.0 ** -47 * scale
        assert np.abs(x0 - sc.x).max() < 1e-6 * f32
        shifted = sc.x + 1.234567891e-3
        c.set_layer(0, "x", shifted)
        assert np.abs(c.get(0, "x") - shifted).max() <= 2.0 ** -47 * scale


@pytest.mark.parametrize("brick", [0, 2])
def test_scene_far_from_the_origin_matches_fp64_oracle(gpu_ready, brick):
    """A scene 3,000 cells from the origin: a float32 position there is
    rounded to up to 1.2e-4 of a cell (2.4e-4 apart).  The displacement,
    strain, loss and gradient still meet the FP32 path's bars against the FP64
    oracle, and agree with the same scene at the origin to float rounding."""
    L = 13
    far = _scene(OFFSET)
    o, loss = _oracle(far, L)
    r = _fp32(far, o.target, L, brick_cells=brick)
    assert relerr(r["x"] - far.x, o.get(L - 1, "x") - far.x) < 1e-4
    assert relerr(r["F"], o.get(L - 1, "F")) < 1e-4
    assert abs(r["loss"] - loss) / abs(loss) < 1e-4
    assert normrel(r["dLdx"], o.get(0, "dLdx")) < 1e-3
    near = _scene((0.0, 0.0, 0.0))
    on, _ = _oracle(near, L)
    rn = _fp32(near, on.target, L, brick_cells=brick)
    assert normrel(r["grad"], rn["grad"]) < 1e-4
    assert relerr(r["x"] - far.x, rn["x"] - near.x) < 1e-4
