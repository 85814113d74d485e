"""The deterministic mode of the FP32-mixed path (dmpm_params::deterministic):
P2G, the adjoint scatter and the mass rasters sum each node as 64-bit integer
multiples of a per-pass power of two (csrc/fixpoint.cuh) -- through each
brick unit's shared-memory node tile when the epoch has units (brick_cells 2
or 4), straight into global memory otherwise (0) -- so two runs on the same
inputs give bit-identical states, losses and gradients, and so do the
checkpointed, eager and graph-replayed evaluations of one gradient.  The
mode computes the same quantities, so it is held to the FP32 path's bars
against the FP64 oracle (the CPU restatement of the reference's
ForwardTimeStep / EndLayerMassLoss / Back_Timestep)."""
import numpy as np
import pytest

import dmpm
import scenes
from oracle.lib import OracleGraph
from tests.helpers import normrel, relerr
from tests.test_gpu_parity import make_ctx

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stirred():
    """A 24^3 cloud that drifts about two cells along x over 24 steps and is
    stirred by random velocities, so particles leave their cells between sorts
    (items whose particles no longer share a stencil take the per-lane path)."""
    sc = scenes.small_scene(seed=41, res=24, radius=0.25, steps=24, v_std=30.0, drag=0.1, smoothing=0.05,
                            f_ext=(0.0, -2.0, 0.0), dt=2e-4)
    sc.v[:, 0] += 400.0
    sc.vol = OracleGraph(sc, "f64").calc_volumes()
    L = 25
    o = OracleGraph(sc, "f64")
    o.setup(L, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
    o.forward(0)
    loss = o.loss()
    o.backward(0, 1)
    return sc, o, loss, L


def _gradient(sc, target, L, **params):
    with make_ctx(sc, "fp32", target, adjoint="exact", control="tied", **params) as c:
        c.setup(L)
        assert c.forward(0) == dmpm.OK
        lo = c.loss()
        assert c.backward(0) == dmpm.OK
        return {"loss": lo, "grad": c.control_grad(), "x": c.get(L - 1, "x"), "F": c.get(L - 1, "F"),
                "m": c.get_grid(L // 2, "grid_m"), "dLdx": c.get(0, "dLdx"), "m0": c.get_grid(0, "grid_m"),
                "v0": c.get_grid(0, "grid_v")}


@pytest.mark.parametrize("general", [False, True])
@pytest.mark.parametrize("brick", [0, 2, 4])
def test_deterministic_runs_are_bit_identical(gpu_ready, stirred, brick, general):
    sc, o, loss, L = stirred
    kw = dict(deterministic=True, brick_cells=brick, warp_general=general, sort_every=8)
    a = _gradient(sc, o.target, L, **kw)
    b = _gradient(sc, o.target, L, **kw)
    assert a["loss"] == b["loss"]
    for k in ("grad", "x", "F", "m", "dLdx"):
        assert np.array_equal(a[k], b[k]), k
    if brick:
        # the first P2G (before any G2P, whose kernel brick_cells also picks) through the
        # unit tiles and straight into global memory: the same integers, added elsewhere first
        w = _gradient(sc, o.target, L, **dict(kw, brick_cells=0))
        assert np.array_equal(a["m0"], w["m0"]) and np.array_equal(a["v0"], w["v0"])


@pytest.mark.parametrize("brick", [0, 2, 4])
def test_deterministic_mode_matches_fp64_oracle(gpu_ready, stirred, brick):
    sc, o, loss, L = stirred
    r = _gradient(sc, o.target, L, deterministic=True, brick_cells=brick)
    assert relerr(r["x"], o.get(L - 1, "x")) < 1e-5
    assert relerr(r["F"], o.get(L - 1, "F")) < 1e-4
    assert abs(r["loss"] - loss) / abs(loss) < 1e-4
    assert normrel(r["dLdx"], o.get(0, "dLdx")) < 1e-3
    # and the float-atomic mode on the same inputs: the same quantities, summed in another order
    f = _gradient(sc, o.target, L, brick_cells=brick)
    assert normrel(r["grad"], f["grad"]) < 1e-4
    assert abs(r["loss"] - f["loss"]) / abs(f["loss"]) < 1e-5


def test_deterministic_checkpointing_and_graphs_give_the_same_bits(gpu_ready, stirred):
    """Store-all replayed as CUDA graphs, eager store-all and checkpoint-every-3
    (segments recomputed during the backward pass) run the same kernels on the
    same inputs, so in this mode their gradients agree bit for bit."""
    sc, o, loss, L = stirred
    ref = None
    for kw in (dict(), dict(eager=True), dict(checkpoint_every=3)):
        r = _gradient(sc, o.target, L, deterministic=True, **kw)
        if ref is None:
            ref = r
            continue
        assert r["loss"] == ref["loss"], kw
        assert np.array_equal(r["grad"], ref["grad"]), kw


def test_deterministic_volumes_and_target_raster(gpu_ready):
    """dmpm_compute_volumes and dmpm_rasterize_target in this mode: the same
    bits on every call, and within float rounding of the float-atomic mode."""
    sc = scenes.small_scene(seed=23, res=32, radius=0.3, ppc_root=3)
    out = []
    for det in (True, True, False):
        with dmpm.Context("fp32") as c:
            c.set_grid(sc.dims, sc.dx, sc.min_point)
            c.set_particles(sc.x, sc.m, sc.lam, sc.mu)
            c.set_params(dt=1e-4, deterministic=det)
            c.compute_volumes()
            c.rasterize_target(sc.target_points, sc.target_mp)
            c.setup(1)
            out.append((c.get(0, "vol"), c.target_mass()))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert relerr(out[0][0], out[2][0]) < 1e-5
    assert relerr(out[0][1], out[2][1]) < 1e-5


def _edge_scene(case):
    """The boundary and few-particle scenes of tests/test_gpu_parity.py: a cloud
    partly outside the grid's low corner (clamped cell keys), and 1 or 37
    particles on a 16 x 12 x 10 grid."""
    if case == "boundary":
        sc = scenes.small_scene(seed=13, res=16, radius=0.2, steps=5, v_std=0.4, drag=0.1, smoothing=0.05,
                                f_ext=(0.0, -1.0, 0.0), offset=(-0.42, -0.42, 0.0))
        sc.x = sc.x - np.array([1.3, 0.7, 0.0])
        sc.v[:, 0] -= 0.5
        return sc, 6
    count = 1 if case == "one" else 37
    sc = scenes.small_scene(seed=17, res=16, radius=0.2, steps=4, v_std=0.3, drag=0.1, f_ext=(0.0, -1.0, 0.0))
    keep = np.argsort(np.linalg.norm(sc.x - sc.x.mean(axis=0), axis=1))[:count]
    for f in ("x", "v", "F", "C", "dFc", "m", "lam", "mu", "vol"):
        setattr(sc, f, np.ascontiguousarray(getattr(sc, f)[keep]))
    sc.dims = (16, 12, 10)
    if count == 1:
        sc.F = np.eye(3)[None].copy()
        sc.dFc = np.zeros((1, 3, 3))
    return sc, 5


@pytest.mark.parametrize("case", ["boundary", "one", "few37"])
def test_deterministic_mode_at_the_grid_boundary_and_with_few_particles(gpu_ready, case):
    sc, L = _edge_scene(case)
    o = OracleGraph(sc, "f64")
    sc.vol = o.calc_volumes()
    o = OracleGraph(sc, "f64")
    o.setup(L, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
    o.forward(0)
    loss = o.loss()
    o.backward(0, 1)
    runs = []
    for _ in range(2):
        with make_ctx(sc, "fp32", o.target, adjoint="exact", keep_adjoints=True, deterministic=True) as c:
            c.setup(L)
            assert c.forward(0) == dmpm.OK
            lo = c.loss()
            assert c.backward(0) == dmpm.OK
            runs.append((c.get(L - 1, "x"), lo, c.get(0, "dLdFe"), c.get(0, "dLdx")))
    x, lo, dfe, dlx = runs[0]
    assert relerr(x, o.get(L - 1, "x")) < 1e-5
    assert abs(lo - loss) / abs(loss) < 1e-4
    assert normrel(dfe, o.get(0, "dLdFe")) < 1e-3
    assert normrel(dlx, o.get(0, "dLdx")) < 1e-3
    assert runs[1][1] == lo
    for a, b in zip(runs[0], runs[1]):
        assert np.array_equal(np.asarray(a), np.asarray(b))
