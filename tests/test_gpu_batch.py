"""Batched instances (dmpm_batch_*) against the one-scene FP32-mixed path.

Three seeded scenes with different grids and numbers of time steps (listed
out of step order, so the batch's internal longest-first ordering differs from
the caller's) run in one batch; every instance's loss, final positions and
tied control gradient must match the same scene run alone through a
dmpm_ctx, whose own parity against the oracle is covered by
test_gpu_parity.py.  Both paths are FP32 with atomic accumulation, so they
agree to summation-order noise (tolerances below).
"""
import numpy as np
import pytest

import dmpm
import scenes
from tests.helpers import relerr
from oracle.lib import OracleGraph

pytestmark = pytest.mark.gpu

DT, DRAG, SMOOTH, FEXT = 2e-4, 0.1, 0.05, (0.0, -1.0, 0.0)


def _scenes():
    out = []
    for seed, res, steps, radius in ((21, 12, 3, 0.22), (22, 16, 6, 0.2), (23, 14, 4, 0.25)):
        sc = scenes.small_scene(seed=seed, res=res, radius=radius, steps=steps, v_std=0.3, drag=DRAG,
                                smoothing=SMOOTH, f_ext=FEXT, dt=DT)
        og = OracleGraph(sc, "f64")
        sc.vol = og.calc_volumes()
        sc.target = OracleGraph(sc, "f64").target
        out.append(sc)
    return out


@pytest.fixture(scope="module")
def batch_case(gpu_ready):
    scs = _scenes()
    singles = []
    for sc in scs:
        with dmpm.Context("fp32") as c:
            c.set_grid(sc.dims, sc.dx, sc.min_point)
            c.set_particles(sc.x, sc.m, sc.lam, sc.mu, v=sc.v, F=sc.F, C=sc.C, dFc=sc.dFc, vol=sc.vol)
            c.set_target_mass(sc.target)
            c.set_params(dt=DT, drag=DRAG, f_ext=FEXT, smoothing=SMOOTH, adjoint="exact", control="tied")
            c.setup(sc.steps + 1)
            c.forward(0)
            loss = c.loss()
            c.backward(0)
            singles.append((loss, c.control_grad(), c.get(sc.steps, "x")))
    return scs, singles


def _batch(scs):
    b = dmpm.Batch([{"n": sc.n, "dims": sc.dims, "dx": sc.dx, "min_point": sc.min_point, "steps": sc.steps}
                    for sc in scs])
    b.set_params(dt=DT, drag=DRAG, f_ext=FEXT, smoothing=SMOOTH, adjoint="exact")
    for i, sc in enumerate(scs):
        b.set_particles(i, sc.x, sc.m, sc.lam, sc.mu, v=sc.v, F=sc.F, C=sc.C, dFc=sc.dFc, vol=sc.vol)
        b.set_target_mass(i, sc.target)
    return b


def _check(b, scs, singles, losses):
    for i, sc in enumerate(scs):
        lo, g, x = singles[i]
        assert abs(losses[i] - lo) <= 1e-6 * abs(lo), (i, losses[i], lo)
        assert relerr(b.get(i, sc.steps, "x"), x) < 1e-5, i
        assert relerr(b.control_grad(i), g) < 1e-4, i


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_matches_single_scene_runs(batch_case, use_graph):
    scs, singles = batch_case
    with _batch(scs) as b:
        b.set_launch(use_graph=use_graph)
        b.setup()
        for _ in range(2):  # a graph is captured on the first call and replayed on the second
            losses = b.gradient()
            _check(b, scs, singles, losses)
        info = b.info()
        assert info["instances"] == 3 and info["particles"] == sum(sc.n for sc in scs)
        assert info["graph"] == use_graph and info["launches_per_gradient"] > 0


@pytest.mark.parametrize("sort_every,ctas", [(1, 1), (3, 2), (100, 8)])
def test_batch_launch_settings_do_not_change_results(batch_case, sort_every, ctas):
    scs, singles = batch_case
    with _batch(scs) as b:
        b.set_launch(sort_every=sort_every, ctas_per_sm=ctas, particle_block=128, use_graph=True)
        b.setup()
        _check(b, scs, singles, b.gradient())


def test_batch_autotune_then_gradient(batch_case):
    scs, singles = batch_case
    with _batch(scs) as b:
        b.setup()
        ms = b.autotune(reps=1)
        assert ms > 0
        cfg = b.launch()
        assert cfg["sort_every"] in (4, 8, 16) and cfg["ctas_per_sm"] in (2, 3, 4, 6)
        assert cfg["particle_block"] in (128, 256)
        _check(b, scs, singles, b.gradient())


def test_batch_errors(batch_case):
    scs, _ = batch_case
    with pytest.raises(dmpm.DmpmError):
        dmpm.Batch([{"n": 10, "dims": (8, 8, 8), "steps": 0}])
    with pytest.raises(dmpm.DmpmError):
        dmpm.Batch([{"n": 10, "dims": (8, 8, 8), "steps": 2, "dx": 1.0},
                    {"n": 10, "dims": (8, 8, 8), "steps": 2, "dx": 0.5}])
    with _batch(scs) as b:
        with pytest.raises(dmpm.DmpmError):
            b.gradient()  # before setup
        b.setup()
        with pytest.raises(dmpm.DmpmError):
            b.control_grad(0)  # before a gradient
        with pytest.raises(dmpm.DmpmError):
            b.set_target_mass(7, scs[0].target)
        with pytest.raises(dmpm.DmpmError):
            b.set_launch(particle_block=100)
