"""The brick G2P of the FP32-mixed path (brick_cells = 2, the default, or 4):
one thread per particle over the node tile of a brick of cells staged in shared
memory.  It computes what the warp-item G2P (brick_cells = 0) computes, summed
in another order, so it is held to the same bars against the FP64 oracle (the
CPU restatement of the reference's ForwardTimeStep / EndLayerMassLoss /
Back_Timestep) and to the warp-item kernel's results on the same inputs.
Particles that leave their brick between cell sorts take the kernel's
global-memory path; the long sort interval and fast cloud below make many of
them."""
import numpy as np
import pytest

import dmpm
import scenes
from oracle.lib import OracleGraph
from tests.helpers import normrel, relerr
from tests.test_gpu_parity import make_ctx

pytestmark = pytest.mark.gpu

BRICKS = [2, 4]


def _oracle(sc, L, prec="f64"):
    o = OracleGraph(sc, prec)
    o.setup(L, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
    o.forward(0)
    loss = o.loss()
    o.backward(0, 1)
    return o, loss


@pytest.fixture(scope="module")
def case():
    sc = scenes.small_scene(seed=5, res=16, steps=6, v_std=0.4, drag=0.2, smoothing=0.1, f_ext=(0.0, -1.0, 0.0),
                            dt=2e-4)
    sc.vol = OracleGraph(sc, "f64").calc_volumes()
    L = 7
    o, loss = _oracle(sc, L)
    return sc, o, loss, L


@pytest.fixture(scope="module")
def fast_case():
    """A 24^3 cloud that drifts about two cells along x over its 24 steps (and
    is stirred by random velocities), so it crosses brick faces between sorts."""
    sc = scenes.small_scene(seed=41, res=24, radius=0.25, steps=24, v_std=30.0, drag=0.1, smoothing=0.05,
                            f_ext=(0.0, -2.0, 0.0), dt=2e-4)
    sc.v[:, 0] += 400.0
    sc.vol = OracleGraph(sc, "f64").calc_volumes()
    L = 25
    o, loss = _oracle(sc, L)
    return sc, o, loss, L


def _run(sc, target, L, **params):
    with make_ctx(sc, "fp32", target, adjoint="exact", keep_adjoints=True, **params) as c:
        c.setup(L)
        c.forward(0)
        lo = c.loss()
        c.backward(0)
        return {"x": c.get(L - 1, "x"), "F": c.get(L - 1, "F"), "v": c.get(L - 1, "v"), "loss": lo,
                "grid_m": c.get_grid(0, "grid_m"), "dLdFe": c.get(0, "dLdFe"), "dLdx": c.get(0, "dLdx"),
                "dLdv": c.get(0, "dLdv"), "dLdC": c.get(0, "dLdC")}


@pytest.mark.parametrize("brick", BRICKS)
def test_brick_kernels_match_fp64_oracle(gpu_ready, case, brick):
    sc, o, loss, L = case
    r = _run(sc, o.target, L, brick_cells=brick)
    assert relerr(r["x"], o.get(L - 1, "x")) < 1e-5
    assert relerr(r["F"], o.get(L - 1, "F")) < 1e-4
    assert relerr(r["v"], o.get(L - 1, "v")) < 2e-3
    assert relerr(r["grid_m"], o.get(0, "grid_m")) < 1e-5
    assert abs(r["loss"] - loss) / abs(loss) < 1e-4
    assert normrel(r["dLdFe"], o.get(0, "dLdFe")) < 1e-3
    assert normrel(r["dLdx"], o.get(0, "dLdx")) < 1e-3


@pytest.mark.parametrize("brick", BRICKS)
def test_brick_kernels_match_warp_items(gpu_ready, case, brick):
    """Same inputs, same FP32 arithmetic per term: the two kernel families differ
    only by float summation order."""
    sc, o, loss, L = case
    w = _run(sc, o.target, L, brick_cells=0)
    b = _run(sc, o.target, L, brick_cells=brick)
    assert relerr(b["x"], w["x"]) < 1e-5
    assert relerr(b["F"], w["F"]) < 1e-5
    assert abs(b["loss"] - w["loss"]) / abs(w["loss"]) < 1e-5
    for k in ("dLdFe", "dLdx", "dLdv", "dLdC"):
        assert normrel(b[k], w[k]) < 1e-3, k


@pytest.mark.parametrize("adjoint", ["exact", "refcompat"])
@pytest.mark.parametrize("brick", BRICKS)
def test_brick_grid_fields_and_adjoints_match_warp_items(gpu_ready, case, brick, adjoint):
    """Layer grids, grid adjoints and the first layer's dLdx of the brick G2P
    and the warp-item G2P on the same inputs, in both adjoint modes (the grid
    momentum is left out: it is recovered from the stored velocity as
    (v - dt f) m, which cancels where |v| is close to dt |f| and so magnifies
    the float-order differences)."""
    sc, o, loss, L = case
    out = {}
    for b in (0, brick):
        with make_ctx(sc, "fp32", o.target, adjoint=adjoint, keep_intermediates=True, brick_cells=b) as c:
            c.setup(L)
            c.forward(0)
            c.loss()
            c.backward(0)
            out[b] = {(lay, k): c.get_grid(lay, k) for lay in (0, L // 2, L - 2)
                      for k in ("grid_m", "grid_v", "grid_dLdv", "grid_dLdp", "grid_dLdm")}
            out[b]["dLdx"] = c.get(0, "dLdx")
    for key, w in out[0].items():
        adj = key == "dLdx" or key[1].startswith("grid_dLd")
        assert normrel(out[brick][key], w) < (1e-3 if adj else 1e-4), key  # float summation orders differ


@pytest.mark.parametrize("sort_every", [1, 100])
@pytest.mark.parametrize("brick", BRICKS)
def test_brick_kernels_with_particles_leaving_their_bricks(gpu_ready, fast_case, brick, sort_every):
    """sort_every 100: the cloud is sorted once and crosses brick faces during the
    rollout, so its particles mix the tile and global-memory paths."""
    sc, o, loss, L = fast_case
    r = _run(sc, o.target, L, brick_cells=brick, sort_every=sort_every)
    assert relerr(r["x"], o.get(L - 1, "x")) < 1e-5
    assert abs(r["loss"] - loss) / abs(loss) < 1e-4
    assert normrel(r["dLdFe"], o.get(0, "dLdFe")) < 1e-3
    assert normrel(r["dLdx"], o.get(0, "dLdx")) < 1e-3


@pytest.mark.parametrize("brick", BRICKS)
def test_brick_kernels_at_and_outside_the_grid_boundary(gpu_ready, brick):
    """A cloud straddling the grid's low corner, partly outside it: clamped cell
    keys put such particles into border bricks whose tiles reach outside the
    grid (zeros there, nothing flushed)."""
    sc = scenes.small_scene(seed=13, res=16, radius=0.2, steps=5, v_std=0.4, drag=0.1, smoothing=0.05,
                            f_ext=(0.0, -1.0, 0.0), offset=(-0.42, -0.42, 0.0))
    sc.x = sc.x - np.array([1.3, 0.7, 0.0])
    sc.v[:, 0] -= 0.5
    sc.vol = OracleGraph(sc, "f64").calc_volumes()
    L = 6
    o, loss = _oracle(sc, L)
    r = _run(sc, o.target, L, brick_cells=brick)
    assert relerr(r["x"], o.get(L - 1, "x")) < 1e-5
    assert relerr(r["F"], o.get(L - 1, "F")) < 1e-4
    assert abs(r["loss"] - loss) / abs(loss) < 1e-4
    assert normrel(r["dLdFe"], o.get(0, "dLdFe")) < 1e-3
    assert normrel(r["dLdx"], o.get(0, "dLdx")) < 1e-3


@pytest.mark.parametrize("brick", BRICKS)
def test_brick_kernels_with_checkpointing_and_graphs(gpu_ready, case, brick):
    """Checkpoint every 3 layers (segments recomputed in the backward pass) and
    store-all replayed as CUDA graphs give the eager store-all gradient."""
    sc, o, loss, L = case
    ref = None
    for kw in (dict(eager=True), dict(checkpoint_every=3), dict()):
        with make_ctx(sc, "fp32", o.target, adjoint="exact", control="tied", brick_cells=brick, **kw) as c:
            c.setup(L)
            c.forward(0)
            c.loss()
            c.backward(0)
            g = c.control_grad()
        if ref is None:
            ref = g
        else:
            assert normrel(g, ref) < 1e-4, kw  # float atomics: summation order differs run to run


@pytest.mark.parametrize("ckpt", [1, 3])
@pytest.mark.parametrize("brick", [0] + BRICKS)
def test_stress_stage_formed_by_g2p_matches_oracle(gpu_ready, case, brick, ckpt):
    """With the brick G2P (brick_cells 2 or 4) each step's G2P also forms the next
    step's stress stage (P, the polar factors and G), which the next step then
    does not recompute; with warp items (0) a separate kernel forms it.  The
    per-layer P (keep_intermediates) of every layer against the FP64 oracle,
    store-all and checkpointed (segments recomputed during the backward pass)."""
    sc, o, loss, L = case
    with make_ctx(sc, "fp32", o.target, adjoint="exact", keep_intermediates=True, brick_cells=brick,
                  checkpoint_every=ckpt) as c:
        c.setup(L)
        assert c.forward(0) == dmpm.OK
        c.loss()
        assert c.backward(0) == dmpm.OK
        for lay in range(L - 1):
            assert normrel(c.get(lay, "P"), o.get(lay, "P")) < 1e-3, lay
        assert normrel(c.get(0, "dLdFe"), o.get(0, "dLdFe")) < 1e-3
