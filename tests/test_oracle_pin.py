"""Pin the CPU oracle (oracle/dmpm_oracle.cpp) to the reference's own outputs.

The golden vectors come from the reference sources compiled here
(tests/golden/make_golden.py).  FP64: the oracle restates the FP64-retyped
reference to ~1e-10 relative.  FP32: the shipped float reference computes its
polar decomposition with a 1024*FLT_EPSILON stopping tolerance, so its stress
carries ~1e-3 relative noise; the FP32 comparison is correspondingly loose.
"""
import numpy as np
import pytest

import scenes
from tests.helpers import relerr
from oracle.lib import Elementary, OracleGraph


def test_elementary_fp64(golden):
    g = golden("elementary_f64")
    e = Elementary("oracle", "f64")
    for F, dF, R, S, P, d2 in zip(g["F"], g["dF"], g["R"], g["S"], g["P"], g["d2"]):
        r, s = e.polar(F)
        assert relerr(r, R) < 1e-9 and relerr(s, S) < 1e-9
        assert relerr(e.pk(F, float(g["lam"]), float(g["mu"])), P) < 1e-8
        assert relerr(e.d2(F, float(g["lam"]), float(g["mu"]), dF), d2) < 1e-8
    for x, b, bs in zip(g["bx"], g["b"], g["bs"]):
        assert e.bspline(x) == b and e.bspline_slope(x) == bs


def test_elementary_fp32(golden):
    g = golden("elementary_f32")
    e = Elementary("oracle", "f32")
    for x, b, bs in zip(g["bx"], g["b"], g["bs"]):
        assert abs(e.bspline(x) - b) <= 1e-7 and abs(e.bspline_slope(x) - bs) <= 1e-6
    # CheckGradients fixture: F = 0.8 Rx(45deg) is a scaled rotation, R exact
    r, _ = e.polar(g["F"][0])
    assert relerr(r, g["R"][0]) < 1e-5


def _oracle_rollout(prec, golden_name):
    from tests.golden.make_golden import ROLLOUT_LAYERS, rollout_scene

    g = golden_name
    sc = rollout_scene()
    o = OracleGraph(sc, prec, target_m=g["target"])
    vol = o.calc_volumes()
    sc.vol = np.asarray(g["vol"], dtype=np.float64)
    o = OracleGraph(sc, prec, target_m=g["target"])
    o.setup(ROLLOUT_LAYERS, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
    o.forward(0)
    loss = o.loss()
    o.backward(0, 0)
    return o, vol, loss, ROLLOUT_LAYERS


def test_rollout_fp64(golden):
    g = golden("rollout_f64")
    o, vol, loss, L = _oracle_rollout("f64", g)
    assert relerr(vol, g["vol"]) < 1e-12
    tgt = g["target"]
    for lay in range(L):
        for k in ("x", "v", "F", "C"):
            assert relerr(o.get(lay, k), g["%s_%d" % (k, lay)]) < 1e-10, (k, lay)
        if lay < L - 1:
            assert relerr(o.get(lay, "P"), g["P_%d" % lay]) < 1e-10
            assert relerr(o.get(lay, "grid_m"), g["grid_m_%d" % lay]) < 1e-12
            assert relerr(o.get(lay, "grid_v"), g["grid_v_%d" % lay]) < 1e-10
    assert abs(loss - float(g["loss"])) / abs(float(g["loss"])) < 1e-12
    for lay in range(L - 1):
        for k in ("dLdF", "dLdx", "dLdv", "dLdC", "dLdP", "dLdv_next", "dLdC_next"):
            assert relerr(o.get(lay, k), g["%s_%d" % (k, lay)]) < 1e-10, (k, lay)
        for k in ("grid_dLdv", "grid_dLdp", "grid_dLdm"):
            assert relerr(o.get(lay, k), g["%s_%d" % (k, lay)]) < 1e-10, (k, lay)
    assert tgt.shape == (16 ** 3,)


def test_rollout_fp32(golden):
    g = golden("rollout_f32")
    o, vol, loss, L = _oracle_rollout("f32", g)
    assert relerr(vol, g["vol"]) < 1e-6
    for lay in range(L):
        assert relerr(o.get(lay, "x"), g["x_%d" % lay]) < 1e-5
        assert relerr(o.get(lay, "F"), g["F_%d" % lay]) < 1e-4
        assert relerr(o.get(lay, "v"), g["v_%d" % lay]) < 3e-2
    assert abs(loss - float(g["loss"])) / abs(float(g["loss"])) < 1e-4
    assert relerr(o.get(0, "dLdF"), g["dLdF_0"]) < 1e-2
    assert relerr(o.get(0, "dLdx"), g["dLdx_0"]) < 1e-3


@pytest.mark.parametrize("steps", [1, 10, 30, 100])
def test_long_rollouts_fp64(golden, steps):
    """RefCompat rollouts of 1 to 100 steps against the reference's FP64 build:
    the last layer's state, the loss and the layer-0 adjoint (which the
    reference's adjoint grows to ~1e21 over 100 steps).  Measured: loss
    <= 2.1e-16, x and F <= 7.3e-14, v <= 4.6e-12 (the grid velocity p/m of
    nearly empty nodes), adjoint <= 1.1e-10 (at 100 steps)."""
    from tests.golden.make_golden import long_scene

    g = golden("rollout_long_f64")
    sc = long_scene()
    sc.vol = np.asarray(g["vol"], dtype=np.float64)
    o = OracleGraph(sc, "f64", target_m=g["target"])
    o.setup(steps + 1, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
    o.forward(0)
    loss = o.loss()
    o.backward(0, 0)
    assert abs(loss - float(g["loss_%d" % steps])) / abs(float(g["loss_%d" % steps])) < 1e-12
    for k in ("x", "v", "F"):
        assert relerr(o.get(steps, k), g["%s_%d" % (k, steps)]) < 1e-10, k
    for k in ("dLdx", "dLdv", "dLdF", "dLdC"):
        assert relerr(o.get(0, k), g["%s0_%d" % (k, steps)]) < 1e-9, k


@pytest.mark.parametrize("mode", ["layer0", "tied"])
def test_exact_adjoint_matches_central_fd(mode):
    """The oracle's exact adjoint against central differences in FP64."""
    sc = scenes.small_scene(seed=2, res=12, steps=4, v_std=0.5, drag=0.3, smoothing=0.1, f_ext=(0.0, -2.0, 0.5))
    sc.vol = OracleGraph(sc, "f64").calc_volumes()
    L = 5

    def run(dfc_layer0=None, dfc_all=None):
        s2 = scenes.Scene(**{**sc.__dict__})
        if dfc_all is not None:
            s2.dFc = dfc_all
        g = OracleGraph(s2, "f64")
        g.setup(L, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
        if dfc_layer0 is not None:
            g.set(0, "dFc", dfc_layer0)
        g.forward(0)
        return g

    g = run()
    g.loss()
    g.backward(0, 1)
    rng = np.random.default_rng(7)
    h = 1e-5
    for _ in range(3):
        D = rng.normal(size=(sc.n, 3, 3))
        if mode == "layer0":
            fd = (run(dfc_layer0=sc.dFc + h * D).loss() - run(dfc_layer0=sc.dFc - h * D).loss()) / (2 * h)
            an = float(np.sum(g.get(0, "dLdFe") * D))
        else:
            fd = (run(dfc_all=sc.dFc + h * D).loss() - run(dfc_all=sc.dFc - h * D).loss()) / (2 * h)
            an = float(sum(np.sum(g.get(k, "dLdFe") * D) for k in range(L - 1)))
        assert abs(fd - an) <= 1e-5 * abs(fd) + 1e-14, (fd, an)


def _config0_bars():
    """Bars for the full-size config-0 comparison.  The reference's adjoint
    takes d(J F^-T)/dF by central differences with delta = 1e-6
    (Elasticity.cpp:7-72), which turns rounding-level input differences into
    ~1e-10 differences of the adjoint: the FP64 build against itself with every
    position multiplied by (1 + 2^-52) moves dLdF by 1.3e-10 max-abs relative
    (7.5e-11 norm-relative).  The bars sit a few times above that floor."""
    return {"x": 1e-12, "loss": 1e-11, "adj_maxabs": 1e-9, "adj_norm": 5e-10}


def test_config0_full_size_fp64(golden):
    """The oracle against the reference's FP64 build on the small benchmark
    configuration at full size (8,778 particles, 32^3, 100 steps, the
    reference's own adjoint): final positions, loss, layer-0 dLdF and dLdx."""
    from tests.golden.make_golden import config0_scene
    from tests.helpers import normrel

    g = golden("config0_f64")
    sc = config0_scene()
    assert abs(sc.dt - float(g["dt"])) == 0.0
    sc.vol = np.asarray(g["vol"], dtype=np.float64)
    o = OracleGraph(sc, "f64", target_m=np.asarray(g["target"], dtype=np.float64))
    L = sc.steps + 1
    o.setup(L, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
    o.forward(0)
    loss = o.loss()
    o.backward(0, 0)
    bar = _config0_bars()
    assert relerr(o.get(L - 1, "x"), g["x_last"]) < bar["x"]
    assert abs(loss - float(g["loss"])) / abs(float(g["loss"])) < bar["loss"]
    for k in ("dLdF", "dLdx"):
        assert relerr(o.get(0, k), g[k + "_0"]) < bar["adj_maxabs"], k
        assert normrel(o.get(0, k), g[k + "_0"]) < bar["adj_norm"], k
