"""dmpm_params::reorder_particles: dmpm_setup stores the cloud in the order of
its cell keys, and every particle array crossing the C ABI stays in the
caller's order.  A cloud handed over in random order must give, field by
field in the caller's order, what the same cloud gives without reordering (to
the summation-order noise of float atomics) and match the FP64 oracle (the CPU
restatement of the reference's ForwardTimeStep / EndLayerMassLoss /
Back_Timestep) at the FP32 path's bars."""
import numpy as np
import pytest

import dmpm
import scenes
from oracle.lib import OracleGraph
from tests.helpers import normrel, relerr
from tests.test_gpu_parity import _cpu_cell_keys, make_ctx

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def shuffled():
    sc = scenes.small_scene(seed=43, res=24, radius=0.25, steps=16, v_std=30.0, drag=0.1, smoothing=0.05,
                            f_ext=(0.0, -2.0, 0.0), dt=2e-4)
    perm = np.random.default_rng(5).permutation(sc.n)
    for f in ("x", "v", "F", "C", "dFc", "m", "lam", "mu"):
        setattr(sc, f, np.ascontiguousarray(getattr(sc, f)[perm]))
    sc.vol = OracleGraph(sc, "f64").calc_volumes()
    L = 17
    o = OracleGraph(sc, "f64")
    o.setup(L, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
    o.forward(0)
    loss = o.loss()
    o.backward(0, 1)
    return sc, o, loss, L


def _run(sc, target, L, reorder, **params):
    with make_ctx(sc, "fp32", target, adjoint="exact", control="tied", keep_adjoints=True,
                  reorder_particles=reorder, **params) as c:
        c.setup(L)
        x0 = c.get(0, "x")
        assert c.forward(0) == dmpm.OK
        lo = c.loss()
        assert c.backward(0) == dmpm.OK
        keys, order, _ = c.cell_sort(L - 1)
        return {"loss": lo, "x0": x0, "x": c.get(L - 1, "x"), "F": c.get(L - 1, "F"), "v": c.get(L - 1, "v"),
                "grad": c.control_grad(), "dLdx": c.get(0, "dLdx"), "dLdF": c.get(3, "dLdF"),
                "m": c.get(0, "m"), "keys": keys, "order": order, "norm": c.dldf_norm(0)}


@pytest.mark.parametrize("params", [dict(), dict(checkpoint_every=4), dict(brick_cells=0), dict(deterministic=True)])
def test_reordered_cloud_reads_back_in_the_callers_order(gpu_ready, shuffled, params):
    sc, o, loss, L = shuffled
    r = _run(sc, o.target, L, True, **params)
    p = _run(sc, o.target, L, False, **params)
    # inputs come back exactly as given (positions as float pairs, m as float)
    assert np.abs(r["x0"] - sc.x).max() <= 2.0 ** -46 * np.abs(sc.x).max()
    assert np.array_equal(r["m"], np.asarray(sc.m, dtype=np.float32).astype(np.float64))
    # the same results as the caller's order, field by field
    assert abs(r["loss"] - p["loss"]) <= 1e-6 * abs(p["loss"])
    for k, bar in (("x", 1e-6), ("F", 1e-5), ("v", 1e-4)):
        assert relerr(r[k], p[k]) < bar, k
    for k in ("grad", "dLdx", "dLdF"):
        assert normrel(r[k], p[k]) < 1e-4, k
    assert abs(r["norm"] - p["norm"]) <= 1e-5 * abs(p["norm"])
    # and the oracle's
    assert relerr(r["x"], o.get(L - 1, "x")) < 1e-5
    assert abs(r["loss"] - loss) / abs(loss) < 1e-4
    assert normrel(r["dLdx"], o.get(0, "dLdx")) < 1e-3
    # the cell sort reports positions in the caller's indices: sorted keys of the caller's particles
    want = _cpu_cell_keys(r["x"], sc.dims)
    assert np.array_equal(r["keys"], want[r["order"]])
    assert np.all(np.diff(r["keys"].astype(np.int64)) >= 0)
    assert np.array_equal(np.sort(r["order"]), np.arange(sc.n, dtype=np.uint32))


def test_reorder_set_and_get_per_layer_fields(gpu_ready, shuffled):
    """Per-layer uploads (dFc of a control frame, positions of a stored layer)
    land on the right particles after the cloud was reordered."""
    sc, o, loss, L = shuffled
    with make_ctx(sc, "fp32", o.target, adjoint="exact", control="per_layer", reorder_particles=True) as c:
        c.setup(L)
        dfc = np.random.default_rng(9).normal(0.0, 1e-3, size=(sc.n, 3, 3))
        c.set_layer(0, "dFc", dfc)
        assert relerr(c.get(0, "dFc"), dfc) < 1e-6
        x = sc.x + 1e-3
        c.set_layer(0, "x", x)
        assert np.abs(c.get(0, "x") - x).max() <= 2.0 ** -46 * np.abs(x).max()
