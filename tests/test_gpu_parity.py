"""GPU parity: the engine through its C ABI against the reference's golden
vectors (FP64 retyped reference) and the CPU oracle.

Tolerances (relative, max-abs over the field / max-abs of the reference):
  FP64 plain path vs FP64 reference:  1e-10 forward state, loss, volumes;
                                      1e-9 for adjoint fields (float atomics
                                      reorder sums; the reference's own polar
                                      stops at 1024 eps).
  FP32 mixed path vs FP64 oracle:     positions 1e-5, deformation 1e-4,
                                      velocities/grid 1e-3, loss 1e-4,
                                      exact control gradient 1e-3 (norm-relative).
  Long RefCompat rollouts (1-100 steps):  FP64 1e-10 state, 1e-9 adjoint;
                                      FP32-mixed adjoint 3e-4 norm-relative.
"""
import numpy as np
import pytest

import dmpm
import scenes
from oracle.lib import OracleGraph, RefGraph
from tests.golden.make_golden import ROLLOUT_LAYERS, rollout_scene
from tests.helpers import load_golden, normrel, relerr

pytestmark = pytest.mark.gpu


def make_ctx(sc, prec, target, **params):
    c = dmpm.Context(prec)
    c.set_grid(sc.dims, sc.dx, sc.min_point)
    c.set_particles(sc.x, sc.m, sc.lam, sc.mu, v=sc.v, F=sc.F, C=sc.C, dFc=sc.dFc, vol=sc.vol)
    c.set_target_mass(target)
    kw = dict(dt=sc.dt, drag=sc.drag, f_ext=sc.f_ext, smoothing=sc.smoothing)
    kw.update(params)
    c.set_params(**kw)
    return c


@pytest.fixture(scope="module")
def g64():
    return load_golden("rollout_f64")


@pytest.fixture(scope="module")
def golden_scene(g64):
    sc = rollout_scene()
    sc.vol = np.asarray(g64["vol"], dtype=np.float64)
    return sc


def test_volumes_and_target_raster(gpu_ready, g64):
    sc = rollout_scene()
    for prec, tol in (("fp64", 1e-12), ("fp32", 1e-5)):
        with dmpm.Context(prec) as c:
            c.set_grid(sc.dims, sc.dx, sc.min_point)
            c.set_particles(sc.x, sc.m, sc.lam, sc.mu, v=sc.v, F=sc.F, C=sc.C, dFc=sc.dFc)
            c.compute_volumes()
            c.rasterize_target(sc.target_points, sc.target_mp)
            # the target grid: the reference's mass-only P2G of the target samples
            # (LoadCompGraph, MPMPolyscope.cpp:142-160), from its FP64 build
            assert relerr(c.target_mass(), g64["target"]) < tol
            c.set_params(dt=sc.dt)
            c.setup(2)
            assert relerr(c.get(0, "vol"), g64["vol"]) < tol
            c.forward(0)
            c.loss()
            assert np.all(np.isfinite(c.get_grid(1, "grid_dLdm")))


@pytest.mark.parametrize("brick", [0, 2, 4])
def test_fp32_grid_fields_match_reference(gpu_ready, g64, golden_scene, brick):
    """dmpm_get_grid on the FP32-mixed path, whose grid update overwrites the
    momentum with the velocity in place: v as stored, p recovered from v and m,
    both against the reference's grids of the first layers (FP32 tolerances),
    with either G2P kernel (warp items, or bricks of 2^3 or 4^3 cells)."""
    sc = golden_scene
    with make_ctx(sc, "fp32", g64["target"], brick_cells=brick) as c:
        c.setup(ROLLOUT_LAYERS)
        assert c.forward(0) == dmpm.OK
        for lay in range(3):
            m = c.get_grid(lay, "grid_m")
            assert relerr(m, g64["grid_m_%d" % lay]) < 1e-5, lay
            assert normrel(c.get_grid(lay, "grid_v"), g64["grid_v_%d" % lay]) < 1e-4, lay
            occ = np.abs(m) > 1.1920929e-07
            assert normrel(c.get_grid(lay, "grid_p")[occ], g64["grid_p_%d" % lay][occ]) < 1e-4, lay


def test_fp64_forward_matches_reference(gpu_ready, g64, golden_scene):
    sc = golden_scene
    with make_ctx(sc, "fp64", g64["target"], keep_intermediates=True) as c:
        c.setup(ROLLOUT_LAYERS)
        assert c.forward(0) == dmpm.OK
        for lay in range(ROLLOUT_LAYERS):
            for k in ("x", "v", "F", "C"):
                assert relerr(c.get(lay, k), g64["%s_%d" % (k, lay)]) < 1e-10, (k, lay)
            if lay < ROLLOUT_LAYERS - 1:
                assert relerr(c.get(lay, "P"), g64["P_%d" % lay]) < 1e-10, lay
                assert relerr(c.get_grid(lay, "grid_m"), g64["grid_m_%d" % lay]) < 1e-12, lay
                assert relerr(c.get_grid(lay, "grid_p"), g64["grid_p_%d" % lay]) < 1e-10, lay
                assert relerr(c.get_grid(lay, "grid_v"), g64["grid_v_%d" % lay]) < 1e-10, lay
        L = c.loss()
        assert abs(L - float(g64["loss"])) / abs(float(g64["loss"])) < 1e-10
        last = ROLLOUT_LAYERS - 1
        assert relerr(c.get_grid(last, "grid_m"), g64["grid_m_%d" % last]) < 1e-12
        assert relerr(c.get_grid(last, "grid_dLdm"), g64["grid_dLdm_%d" % last]) < 1e-10


def test_fp64_refcompat_adjoint_matches_reference(gpu_ready, g64, golden_scene):
    sc = golden_scene
    with make_ctx(sc, "fp64", g64["target"], keep_adjoints=True, keep_intermediates=True) as c:
        c.setup(ROLLOUT_LAYERS)
        c.forward(0)
        c.loss()
        assert c.backward(0) == dmpm.OK
        for lay in range(ROLLOUT_LAYERS):
            for k in ("dLdx", "dLdv", "dLdF", "dLdC"):
                assert relerr(c.get(lay, k), g64["%s_%d" % (k, lay)]) < 1e-9, (k, lay)
        for lay in range(ROLLOUT_LAYERS - 1):
            for k in ("dLdP", "dLdv_next", "dLdC_next"):
                assert relerr(c.get(lay, k), g64["%s_%d" % (k, lay)]) < 1e-9, (k, lay)
            for k in ("grid_dLdv", "grid_dLdp", "grid_dLdm"):
                assert relerr(c.get_grid(lay, k), g64["%s_%d" % (k, lay)]) < 1e-9, (k, lay)
        assert abs(c.dldf_norm(0) - np.linalg.norm(g64["dLdF_0"])) / np.linalg.norm(g64["dLdF_0"]) < 1e-9


@pytest.mark.parametrize("steps", [1, 10, 30, 100])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_long_rollouts_match_reference(gpu_ready, prec, steps):
    """RefCompat rollouts of 1 to 100 steps against the reference's FP64 build
    (rollout_long_f64): the last layer's state, the loss and the layer-0 adjoint,
    which the reference's adjoint grows about twofold per step (to ~1e21).
    Measured on a B200: FP64 loss 2e-14, state <= 5.1e-12, adjoint <= 1.3e-10;
    FP32-mixed loss <= 2.1e-8, x <= 1.0e-6, F <= 4.8e-6, v <= 4.7e-5, adjoint
    <= 4.4e-5 norm-relative (at 100 steps)."""
    from tests.golden.make_golden import long_scene

    g = load_golden("rollout_long_f64")
    sc = long_scene()
    sc.vol = np.asarray(g["vol"], dtype=np.float64)
    fp64 = prec == "fp64"
    with make_ctx(sc, prec, g["target"], keep_adjoints=True) as c:
        c.setup(steps + 1)
        assert c.forward(0) == dmpm.OK
        loss = c.loss()
        assert c.backward(0) == dmpm.OK
        want = float(g["loss_%d" % steps])
        assert abs(loss - want) / abs(want) < (1e-12 if fp64 else 1e-6)
        for k, tol32 in (("x", 1e-5), ("F", 1e-4), ("v", 1e-3)):
            assert relerr(c.get(steps, k), g["%s_%d" % (k, steps)]) < (1e-10 if fp64 else tol32), k
        for k in ("dLdx", "dLdv", "dLdF", "dLdC"):
            got, ref = c.get(0, k), g["%s0_%d" % (k, steps)]
            if fp64:
                assert relerr(got, ref) < 1e-9, k
            else:
                assert normrel(got, ref) < 3e-4, k


def test_config0_full_size_fp64_matches_reference(gpu_ready):
    """The plain FP64 GPU path on the small benchmark configuration at full size
    (8,778 particles, 32^3, 100 steps, the reference's own adjoint with
    per-layer controls) against the reference's FP64 build (config0_f64):
    final positions, loss, layer-0 dLdF and dLdx, at the bars of
    tests/test_oracle_pin.py (the reference's finite-difference d(J F^-T)/dF
    makes its adjoint move by ~1e-10 under rounding-level input changes)."""
    from tests.golden.make_golden import config0_scene
    from tests.test_oracle_pin import _config0_bars

    g = load_golden("config0_f64")
    sc = config0_scene()
    sc.vol = np.asarray(g["vol"], dtype=np.float64)
    L = sc.steps + 1
    bar = _config0_bars()
    with make_ctx(sc, "fp64", g["target"], adjoint="refcompat", control="per_layer") as c:
        c.setup(L)
        assert c.forward(0) == dmpm.OK
        loss = c.loss()
        assert c.backward(0) == dmpm.OK
        assert relerr(c.get(L - 1, "x"), g["x_last"]) < bar["x"]
        assert abs(loss - float(g["loss"])) / abs(float(g["loss"])) < bar["loss"]
        for k in ("dLdF", "dLdx"):
            assert relerr(c.get(0, k), g[k + "_0"]) < bar["adj_maxabs"], k
            assert normrel(c.get(0, k), g[k + "_0"]) < bar["adj_norm"], k


@pytest.mark.parametrize("steps", [1, 10, 30, 100])
def test_fp32_mixed_drifts_less_than_the_shipped_float_reference(gpu_ready, steps):
    """On the same rollouts the shipped FP32 reference build (rollout_long_f32)
    drifts from its FP64 build by 7e-6 to 8e-6 in the loss and 9e-6 to 3.4e-2 in
    the layer-0 adjoint (norm-relative, growing with the steps).  The FP32-mixed
    path keeps the loss and the adjoint at least ten times closer to the FP64
    build, and the final state no further from it (or within 1e-6)."""
    from tests.golden.make_golden import long_scene

    g = load_golden("rollout_long_f64")
    r32 = load_golden("rollout_long_f32")
    sc = long_scene()
    sc.vol = np.asarray(g["vol"], dtype=np.float64)
    with make_ctx(sc, "fp32", g["target"], keep_adjoints=True) as c:
        c.setup(steps + 1)
        assert c.forward(0) == dmpm.OK
        loss = c.loss()
        assert c.backward(0) == dmpm.OK
        want = float(g["loss_%d" % steps])
        assert abs(loss - want) <= 0.1 * abs(float(r32["loss_%d" % steps]) - want)
        for k in ("x", "v", "F"):
            ref = g["%s_%d" % (k, steps)]
            # (one float step leaves both at rounding level, ~1e-7)
            assert normrel(c.get(steps, k), ref) <= max(normrel(r32["%s_%d" % (k, steps)], ref), 1e-6), k
        for k in ("dLdx", "dLdv", "dLdF", "dLdC"):
            ref = g["%s0_%d" % (k, steps)]
            assert normrel(c.get(0, k), ref) <= 0.1 * normrel(r32["%s0_%d" % (k, steps)], ref), k


def test_fp32_refcompat_inspection_fields(gpu_ready, g64, golden_scene):
    """The FP32-mixed path's inspection copies (keep_intermediates / keep_adjoints):
    every particle and grid adjoint field of the first two adjoint steps against the
    reference's FP64 values, at FP32 tolerances (norm-relative)."""
    sc = golden_scene
    with make_ctx(sc, "fp32", g64["target"], keep_adjoints=True, keep_intermediates=True) as c:
        c.setup(ROLLOUT_LAYERS)
        c.forward(0)
        c.loss()
        assert c.backward(0) == dmpm.OK
        def close(got, want, what):
            if not np.any(want):  # e.g. dLdC_next of the top step: the loss zeroes the last layer's dLdC, dLdF
                assert not np.any(got), what
            else:
                assert normrel(got, want) < 2e-3, what

        for lay in (ROLLOUT_LAYERS - 2, ROLLOUT_LAYERS - 3):
            for k in ("dLdx", "dLdv", "dLdF", "dLdC", "dLdP", "dLdv_next", "dLdC_next"):
                close(c.get(lay, k), g64["%s_%d" % (k, lay)], (k, lay))
            for k in ("grid_dLdv", "grid_dLdp", "grid_dLdm"):
                close(c.get_grid(lay, k), g64["%s_%d" % (k, lay)], (k, lay))


def _oracle(sc, L, mode, prec="f64", target=None, control="per_layer"):
    o = OracleGraph(sc, prec, target_m=target)
    o.setup(L, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
    o.forward(0)
    loss = o.loss()
    o.backward(0, mode)
    return o, loss


@pytest.fixture(scope="module")
def exact_case():
    sc = scenes.small_scene(seed=5, res=16, steps=6, v_std=0.4, drag=0.2, smoothing=0.1, f_ext=(0.0, -1.0, 0.0),
                            dt=2e-4)
    o = OracleGraph(sc, "f64")
    sc.vol = o.calc_volumes()
    L = 7
    o, loss = _oracle(sc, L, 1)
    return sc, o, loss, L


def test_fp64_exact_adjoint_matches_oracle(gpu_ready, exact_case):
    sc, o, loss, L = exact_case
    with make_ctx(sc, "fp64", o.target, adjoint="exact", keep_adjoints=True) as c:
        c.setup(L)
        c.forward(0)
        assert abs(c.loss() - loss) / abs(loss) < 1e-10
        c.backward(0)
        for lay in range(L - 1):
            assert relerr(c.get(lay, "dLdFe"), o.get(lay, "dLdFe")) < 1e-9, lay
            assert relerr(c.get(lay, "dLdF"), o.get(lay, "dLdF")) < 1e-9, lay
            assert relerr(c.get(lay, "dLdx"), o.get(lay, "dLdx")) < 1e-9, lay


def test_fp32_mixed_matches_fp64_oracle(gpu_ready, exact_case):
    sc, o, loss, L = exact_case
    with make_ctx(sc, "fp32", o.target, adjoint="exact", keep_adjoints=True) as c:
        c.setup(L)
        c.forward(0)
        for lay in (1, L - 1):
            assert relerr(c.get(lay, "x"), o.get(lay, "x")) < 1e-5
            assert relerr(c.get(lay, "F"), o.get(lay, "F")) < 1e-4
            assert relerr(c.get(lay, "v"), o.get(lay, "v")) < 2e-3
        assert relerr(c.get_grid(0, "grid_m"), o.get(0, "grid_m")) < 1e-5
        assert abs(c.loss() - loss) / abs(loss) < 1e-4
        c.backward(0)
        assert normrel(c.get(0, "dLdFe"), o.get(0, "dLdFe")) < 1e-3
        assert normrel(c.get(0, "dLdx"), o.get(0, "dLdx")) < 1e-3


def test_particles_at_and_outside_the_grid_boundary(gpu_ready):
    """A cloud straddling the grid's low corner, some particles up to 1.3 cells
    outside it, moving outward: stencil nodes outside the grid are skipped, as the
    reference does (ForwardSimulation.cpp:27-30; Grid.cpp:66-69), and the FP32
    path's cell keys clamp such particles into border cells.  Both GPU paths
    against the FP64 oracle, forward and exact adjoint."""
    sc = scenes.small_scene(seed=13, res=16, radius=0.2, steps=5, v_std=0.4, drag=0.1, smoothing=0.05,
                            f_ext=(0.0, -1.0, 0.0), offset=(-0.42, -0.42, 0.0))
    sc.x = sc.x - np.array([1.3, 0.7, 0.0])
    sc.v[:, 0] -= 0.5
    assert np.sum(sc.x[:, 0] < 0) > 20 and np.sum(sc.x[:, 0] < -1.0) > 0
    o = OracleGraph(sc, "f64")
    sc.vol = o.calc_volumes()
    L = 6
    o, loss = _oracle(sc, L, 1)
    with make_ctx(sc, "fp64", o.target, adjoint="exact", keep_adjoints=True) as c:
        c.setup(L)
        assert c.forward(0) == dmpm.OK
        assert relerr(c.get(L - 1, "x"), o.get(L - 1, "x")) < 1e-10
        assert relerr(c.get(L - 1, "F"), o.get(L - 1, "F")) < 1e-10
        assert abs(c.loss() - loss) / abs(loss) < 1e-10
        assert c.backward(0) == dmpm.OK
        assert normrel(c.get(0, "dLdFe"), o.get(0, "dLdFe")) < 1e-8
        assert normrel(c.get(0, "dLdx"), o.get(0, "dLdx")) < 1e-8
    with make_ctx(sc, "fp32", o.target, adjoint="exact", keep_adjoints=True) as c:
        c.setup(L)
        assert c.forward(0) == dmpm.OK
        assert relerr(c.get(L - 1, "x"), o.get(L - 1, "x")) < 1e-5
        assert relerr(c.get(L - 1, "F"), o.get(L - 1, "F")) < 1e-4
        assert abs(c.loss() - loss) / abs(loss) < 1e-4
        assert c.backward(0) == dmpm.OK
        assert normrel(c.get(0, "dLdFe"), o.get(0, "dLdFe")) < 1e-3
        assert normrel(c.get(0, "dLdx"), o.get(0, "dLdx")) < 1e-3


@pytest.mark.parametrize("count", [1, 37])
def test_few_particles_on_a_non_cubic_grid(gpu_ready, count):
    """One particle, and a count that fills no warp, on a 16 x 12 x 10 grid (the
    reference's Grid takes any dims; part of the sphere lies beyond z = 10):
    both GPU paths against the FP64 oracle, forward and exact adjoint."""
    sc = scenes.small_scene(seed=17, res=16, radius=0.2, steps=4, v_std=0.3, drag=0.1, f_ext=(0.0, -1.0, 0.0))
    # a compact cluster around the cloud's centre (sparse particles get large volumes
    # and explode, in the reference as here)
    keep = np.argsort(np.linalg.norm(sc.x - sc.x.mean(axis=0), axis=1))[:count]
    for f in ("x", "v", "F", "C", "dFc", "m", "lam", "mu", "vol"):
        setattr(sc, f, np.ascontiguousarray(getattr(sc, f)[keep]))
    sc.dims = (16, 12, 10)
    if count == 1:  # undeformed, so that the lone particle's large volume makes no explosive stress
        sc.F = np.eye(3)[None].copy()
        sc.dFc = np.zeros((1, 3, 3))
    o = OracleGraph(sc, "f64")
    sc.vol = o.calc_volumes()
    L = 5
    o, loss = _oracle(sc, L, 1)
    for prec, tx, tl, tg in (("fp64", 1e-10, 1e-10, 1e-8), ("fp32", 1e-5, 1e-4, 1e-3)):
        with make_ctx(sc, prec, o.target, adjoint="exact", keep_adjoints=True) as c:
            c.setup(L)
            assert c.forward(0) == dmpm.OK
            assert relerr(c.get(L - 1, "x"), o.get(L - 1, "x")) < tx, prec
            assert abs(c.loss() - loss) / abs(loss) < tl, prec
            assert c.backward(0) == dmpm.OK
            assert normrel(c.get(0, "dLdFe"), o.get(0, "dLdFe")) < tg, prec
            assert normrel(c.get(0, "dLdx"), o.get(0, "dLdx")) < tg, prec


def test_fp32_general_path_matches_same_cell_reduction(gpu_ready, exact_case):
    """warp_general disables the same-cell warp reduce-scatter; both paths agree."""
    sc, o, loss, L = exact_case
    res = []
    for general in (False, True):
        with make_ctx(sc, "fp32", o.target, adjoint="exact", warp_general=general) as c:
            c.setup(L)
            c.forward(0)
            lo = c.loss()
            c.backward(0)
            res.append((c.get(L - 1, "x"), lo, c.get(0, "dLdFe")))
    assert relerr(res[0][0], res[1][0]) < 1e-5
    assert abs(res[0][1] - res[1][1]) / abs(res[1][1]) < 1e-5
    assert normrel(res[0][2], res[1][2]) < 1e-3


@pytest.mark.parametrize("sort_every", [1, 3, 100])
def test_fp32_sort_interval_does_not_change_results(gpu_ready, exact_case, sort_every):
    sc, o, loss, L = exact_case
    with make_ctx(sc, "fp32", o.target, adjoint="exact", sort_every=sort_every, keep_adjoints=True) as c:
        c.setup(L)
        c.forward(0)
        assert relerr(c.get(L - 1, "x"), o.get(L - 1, "x")) < 1e-5
        assert abs(c.loss() - loss) / abs(loss) < 1e-4
        c.backward(0)
        assert normrel(c.get(0, "dLdFe"), o.get(0, "dLdFe")) < 1e-3


def _cpu_cell_keys(x, dims, dx=1.0, mn=(0.0, 0.0, 0.0)):
    """Cell keys exactly as the engine defines them, on the CPU: the stencil
    base floor((x - mn) / dx) - 1 of each position in FP64 (the FP32 engine
    keeps positions as float pairs hi + lo, which c.get returns summed)."""
    x64 = np.asarray(x, dtype=np.float64)
    q = np.floor((x64 - np.asarray(mn, dtype=np.float64)) * (1.0 / dx)).astype(np.int64)
    b = np.clip(np.clip(q, -8, np.asarray(dims) + 8) - 1, -4, np.asarray(dims))
    c = b + 5
    nb = (np.asarray(dims) + 5) // 4 + 1
    br, lo = c >> 2, c & 3
    brick = (br[:, 0] * nb[1] + br[:, 1]) * nb[2] + br[:, 2]
    morton = ((lo[:, 0] >> 1) << 5) | ((lo[:, 1] >> 1) << 4) | ((lo[:, 2] >> 1) << 3) | ((lo[:, 0] & 1) << 2) \
        | ((lo[:, 1] & 1) << 1) | (lo[:, 2] & 1)
    return (brick * 64 + morton).astype(np.uint32)


@pytest.mark.parametrize("shuffle", [False, True])
def test_cell_sort_is_bit_exact_stable_sort(gpu_ready, shuffle):
    """Keys from the reference's floor division and the permutation of a stable
    sort, bit-exact against numpy (argsort kind='stable'); items are runs of
    at most 8 equal keys covering the sorted order."""
    sc = scenes.small_scene(seed=21, res=24, radius=0.3, steps=4, v_std=2.0, dt=2e-4)
    if shuffle:
        perm = np.random.default_rng(3).permutation(sc.n)
        for k in ("x", "v", "F", "C", "dFc", "m", "lam", "mu"):
            setattr(sc, k, getattr(sc, k)[perm])
    sc.vol = OracleGraph(sc, "f64").calc_volumes()
    with make_ctx(sc, "fp32", np.zeros(int(np.prod(sc.dims))), sort_every=2) as c:
        c.setup(5)
        c.forward(0)
        for layer in (0, 4):
            keys, order, items = c.cell_sort(layer)
            want_keys = _cpu_cell_keys(c.get(layer, "x"), sc.dims)
            want_order = np.argsort(want_keys, kind="stable")
            assert np.array_equal(order, want_order.astype(np.uint32))
            assert np.array_equal(keys, want_keys[want_order])
            assert items[0] == 0 and items[-1] == sc.n
            sizes = np.diff(items.astype(np.int64))
            assert np.all(sizes >= 1) and np.all(sizes <= 8)
            for a, b in zip(items[:-1], items[1:]):
                assert np.all(keys[a:b] == keys[a])
            # an item boundary falls on every key change
            changes = np.nonzero(np.diff(keys.astype(np.int64)))[0] + 1
            assert set(changes.tolist()) <= set(items.tolist())


def test_tied_controls_gradient_is_sum_over_layers(gpu_ready, exact_case):
    sc, o, loss, L = exact_case
    with make_ctx(sc, "fp64", o.target, adjoint="exact", control="tied") as c:
        c.setup(L)
        c.forward(0)
        c.loss()
        c.backward(0)
        g = c.control_grad()
    want = sum(o.get(k, "dLdFe") for k in range(L - 1))
    assert relerr(g, want) < 1e-9


@pytest.mark.parametrize("k", [2, 3])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_checkpointing_matches_store_all(gpu_ready, exact_case, prec, k):
    """Checkpoints every k layers: the backward pass recomputes each segment, and
    reading a layer that is not stored (layer 3) recomputes it from the segment's
    checkpoint.  Against the FP64 oracle's store-all run (FP32-mixed at its own
    tolerances: recomputation reorders its float atomics)."""
    sc, o, loss, L = exact_case
    with make_ctx(sc, prec, o.target, adjoint="exact", control="tied", checkpoint_every=k) as c:
        c.setup(L)
        assert c.info()["checkpoint_every"] == k
        c.forward(0)
        lo = c.loss()
        c.backward(0)
        g = c.control_grad()
        x3 = c.get(3, "x")
        F3 = c.get(3, "F")
    want = sum(o.get(j, "dLdFe") for j in range(L - 1))
    if prec == "fp64":
        assert abs(lo - loss) / abs(loss) < 1e-10
        assert relerr(g, want) < 1e-9
        assert relerr(x3, o.get(3, "x")) < 1e-10
        assert relerr(F3, o.get(3, "F")) < 1e-10
    else:
        assert abs(lo - loss) / abs(loss) < 1e-4
        assert normrel(g, want) < 1e-3
        assert relerr(x3, o.get(3, "x")) < 1e-5
        assert relerr(F3, o.get(3, "F")) < 1e-4


def test_fd_gradient_on_gpu_fp64(gpu_ready):
    """Central differences (h = 1e-5) of the GPU FP64 loss along seeded random
    directions in tied-dFc space against the exact adjoint."""
    sc = scenes.small_scene(seed=8, res=12, steps=5, v_std=0.3, drag=0.1, smoothing=0.05, dt=2e-4)
    sc.vol = OracleGraph(sc, "f64").calc_volumes()
    L = 6
    tgt = OracleGraph(sc, "f64").target

    def loss_at(dfc):
        s2 = scenes.Scene(**{**sc.__dict__})
        s2.dFc = dfc
        with make_ctx(s2, "fp64", tgt, adjoint="exact", control="tied") as c:
            c.setup(L)
            c.forward(0)
            return c.loss()

    with make_ctx(sc, "fp64", tgt, adjoint="exact", control="tied") as c:
        c.setup(L)
        c.forward(0)
        c.loss()
        c.backward(0)
        g = c.control_grad()
    rng = np.random.default_rng(123)
    h = 1e-5
    for _ in range(4):
        D = rng.normal(size=(sc.n, 3, 3))
        fd = (loss_at(sc.dFc + h * D) - loss_at(sc.dFc - h * D)) / (2 * h)
        an = float(np.sum(g * D))
        assert abs(fd - an) <= 1e-5 * abs(fd) + 1e-14, (fd, an)


def test_reference_layout_upload_and_download(gpu_ready, golden_scene, g64):
    sc = golden_scene
    pts = np.zeros((sc.n, 118), dtype=np.float32)
    pts[:, 0:3] = sc.x
    pts[:, 3:6] = sc.v
    pts[:, 6:15] = sc.F.transpose(0, 2, 1).reshape(-1, 9)
    pts[:, 15:24] = sc.C.transpose(0, 2, 1).reshape(-1, 9)
    pts[:, 33] = sc.m
    pts[:, 34] = sc.vol
    pts[:, 35] = sc.lam
    pts[:, 36] = sc.mu
    pts[:, 37:46] = sc.dFc.transpose(0, 2, 1).reshape(-1, 9)
    with dmpm.Context("fp64") as c:
        c.set_grid(sc.dims, sc.dx, sc.min_point)
        c.set_points_ref(pts)
        c.set_target_mass(g64["target"])
        c.set_params(dt=sc.dt, drag=sc.drag, f_ext=sc.f_ext, smoothing=sc.smoothing)
        c.setup(3)
        c.forward(0)
        c.loss()
        c.backward(0)
        out = np.zeros_like(pts)
        c.get_points_ref(2, out)
        assert relerr(out[:, 0:3], c.get(2, "x")) < 1e-6
        out0 = np.zeros_like(pts)
        c.get_points_ref(0, out0)
        assert relerr(out0[:, 52:61].reshape(-1, 3, 3).transpose(0, 2, 1), c.get(0, "dLdF")) < 1e-6
        assert np.array_equal(out0[:, 33], pts[:, 33])


def test_errors_are_reported(gpu_ready):
    c = dmpm.Context("fp32")
    with pytest.raises(dmpm.DmpmError) as e:
        c.set_grid((0, 4, 4))
    assert e.value.status == dmpm.ERR_ARG
    c.set_grid((8, 8, 8))
    with pytest.raises(dmpm.DmpmError) as e:
        c.setup(3)
    assert e.value.status == dmpm.ERR_STATE
    sc = scenes.small_scene(seed=1, res=8, radius=0.2)
    c.set_particles(sc.x, sc.m, sc.lam, sc.mu)
    c.set_params(dt=1e-4)
    c.setup(3)
    with pytest.raises(dmpm.DmpmError) as e:
        c.backward(0)
    assert e.value.status == dmpm.ERR_STATE
    # an empty cloud is an argument error (there is nothing to differentiate) and
    # leaves the uploaded cloud and its layers in place
    z = np.zeros((0, 3))
    for call in (lambda: c.set_particles(z, z[:, 0], z[:, 0], z[:, 0]),
                 lambda: c.set_points_ref(np.zeros((0, 118), np.float32))):
        with pytest.raises(dmpm.DmpmError) as e:
            call()
        assert e.value.status == dmpm.ERR_ARG
    assert c.forward(0) == dmpm.OK
    assert np.all(np.isfinite(c.get(2, "x")))
    c.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_out_of_memory_in_setup_leaves_a_usable_context(gpu_ready, exact_case, prec):
    """Allocation failure injected on the host: a device byte limit below what
    dmpm_setup needs makes it fail with DMPM_ERR_OOM (the status a failed
    cudaMalloc gives) before any kernel runs.  The context then reads as not set
    up (forward, loss and layer reads return DMPM_ERR_STATE or DMPM_ERR_ARG, no
    fault), and once the limit is lifted the same context sets up and returns
    the gradient of a fresh context."""
    sc, o, loss, L = exact_case

    def gradient(c):
        c.setup(L)
        c.forward(0)
        lo = c.loss()
        c.backward(0)
        return lo, c.control_grad()

    with make_ctx(sc, prec, o.target, adjoint="exact", control="tied") as c:
        want = gradient(c)
    with make_ctx(sc, prec, o.target, adjoint="exact", control="tied") as c:
        c.set_device_limit(c.info()["device_bytes"] + 4096)  # the scene fits, its layers do not
        with pytest.raises(dmpm.DmpmError) as e:
            c.setup(L)
        assert e.value.status == dmpm.ERR_OOM
        assert c.lib.dmpm_forward(c.h, 0) == dmpm.ERR_STATE
        assert c.lib.dmpm_loss(c.h, None) in (dmpm.ERR_STATE, dmpm.ERR_ARG)
        with pytest.raises(dmpm.DmpmError):
            c.get(0, "x")
        c.set_device_limit(0)
        got = gradient(c)
    assert abs(got[0] - want[0]) <= 1e-6 * abs(want[0])
    assert relerr(got[1], want[1]) < (1e-12 if prec == "fp64" else 1e-4)


def test_nonfinite_is_flagged_not_faulted(gpu_ready):
    """A NaN control on one particle propagates to the grid and the cloud (as in
    the reference); the engine reports DMPM_ERR_NONFINITE from forward and
    backward, and the context stays usable."""
    sc = scenes.small_scene(seed=4, res=12, steps=3)
    sc.vol = OracleGraph(sc, "f64").calc_volumes()
    bad = sc.dFc.copy()
    bad[sc.n // 2, 0, 0] = np.nan
    s2 = scenes.Scene(**{**sc.__dict__})
    s2.dFc = bad
    for prec in ("fp32", "fp64"):
        with make_ctx(s2, prec, np.zeros(int(np.prod(sc.dims)))) as c:
            c.setup(4)
            assert c.forward(0) == dmpm.ERR_NONFINITE
            c.loss()
            assert c.backward(0) == dmpm.ERR_NONFINITE
            c.set_particles(sc.x, sc.m, sc.lam, sc.mu, dFc=sc.dFc, vol=sc.vol)
            c.setup(4)
            assert c.forward(0) == dmpm.OK
            assert np.all(np.isfinite(c.get(3, "x")))


def _reference_descent(sc, d, g, steps, lr, b1, b2, eps):
    """The reference's own PointCloud::Descend_* (its float build, compiled from
    its sources into oracle/_ref) applied to layer 0 of a CompGraph whose dFc
    is d and whose dLdF is the gradient g, with the same gradient norm: the dFc
    after each (rule, t) step of `steps`."""
    from oracle.lib import ref_available

    if not ref_available("f32"):
        pytest.skip("the reference's float build (oracle/_ref) has not been compiled")
    r = RefGraph(sc, "f32", target_m=np.zeros(int(np.prod(sc.dims))), target_from_points=False)
    r.setup(2, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
    r.set(0, "dFc", d)
    r.set(0, "dLdF", g)
    gnorm = float(np.linalg.norm(g))
    out = []
    for rule, t in steps:
        r.descend(rule, 0, lr, gnorm, b1, b2, eps, t)
        out.append(r.get(0, "dFc").astype(np.float64))
    return out


def test_device_adam_step_matches_reference_descend_adam(gpu_ready, exact_case):
    """dmpm_adam_step = PointCloud::Descend_Adam on the tied control gradient,
    with the gradient divided by its norm (PointCloud.cpp:83-99): two steps
    (the second reuses the moments) against the reference's compiled Descend_Adam."""
    sc, o, loss, L = exact_case
    with make_ctx(sc, "fp32", o.target, adjoint="exact", control="tied") as c:
        c.setup(L)
        c.forward(0)
        c.loss()
        c.backward(0)
        g = c.control_grad()
        d0 = c.get(0, "dFc")
        c.adam_step(t=1, lr=1e-2, beta1=0.9, beta2=0.999, eps=1e-5)
        d1 = c.get(0, "dFc")
        c.adam_step(t=2, lr=1e-2, beta1=0.9, beta2=0.999, eps=1e-5)
        d2 = c.get(0, "dFc")
    want1, want2 = _reference_descent(sc, d0, g, [("adam", 1), ("adam", 2)], 1e-2, 0.9, 0.999, 1e-5)
    assert relerr(d1 - d0, want1 - d0) < 1e-4
    assert relerr(d2 - d0, want2 - d0) < 1e-4


def test_control_stride_keeps_controls_on_frames_only(gpu_ready, exact_case):
    """control_stride = 3 with 7 layers: layers 0 and 3 own dFc and its gradient
    (the control frames of OptimizeDefGradControlSequence, CompGraph.cpp:352);
    the others read the uploaded dFc.  Same losses and frame gradients as
    per-layer storage of every layer, before and after editing a frame's dFc."""
    sc, o, loss, L = exact_case
    rng = np.random.default_rng(11)
    with make_ctx(sc, "fp64", o.target, adjoint="exact") as c1, \
            make_ctx(sc, "fp64", o.target, adjoint="exact", control_stride=3) as c3:
        for c in (c1, c3):
            c.setup(L)
        for it in range(2):
            res = []
            for c in (c1, c3):
                c.forward(0)
                lo = c.loss()
                c.backward(0)
                res.append((lo, c.control_grad(0), c.control_grad(3)))
            assert abs(res[0][0] - res[1][0]) <= 1e-13 * abs(res[0][0])
            assert relerr(res[1][1], res[0][1]) < 1e-12 and relerr(res[1][2], res[0][2]) < 1e-12
            if it == 0:
                assert relerr(res[1][1], o.get(0, "dLdFe")) < 1e-9
                assert relerr(res[1][2], o.get(3, "dLdFe")) < 1e-9
                d = c3.get(3, "dFc") + 1e-3 * rng.normal(size=(sc.n, 3, 3))
                c1.set_layer(3, "dFc", d)
                c3.set_layer(3, "dFc", d)
        with pytest.raises(dmpm.DmpmError):
            c3.set_layer(1, "dFc", d)
        with pytest.raises(dmpm.DmpmError):
            c3.control_grad(2)
        with pytest.raises(dmpm.DmpmError):
            c3.adam_step(t=1, layer=4)
        c3.adam_step(t=1, layer=3)


def test_graph_replay_matches_eager_launches(gpu_ready, exact_case):
    """The FP32 store-all passes are captured once and replayed as CUDA graphs;
    replays give the eager launches' results, and dmpm_set_params (here a new
    dt) drops the captured graphs so the next pass runs with the new values."""
    sc, o, loss, L = exact_case
    out = {}
    for eager in (True, False):
        with make_ctx(sc, "fp32", o.target, adjoint="exact", control="tied", eager=eager) as c:
            c.setup(L)
            res = []
            for dt in (sc.dt, sc.dt, 0.5 * sc.dt):
                c.set_params(dt=dt, drag=sc.drag, f_ext=sc.f_ext, smoothing=sc.smoothing, adjoint="exact",
                             control="tied", eager=eager)
                for _ in range(2):  # capture, then replay
                    c.forward(0)
                    lo = c.loss()
                    c.backward(0)
                    res.append((lo, c.control_grad(), c.get(L - 1, "x")))
            out[eager] = res
    for (l_e, g_e, x_e), (l_g, g_g, x_g) in zip(out[True], out[False]):
        assert abs(l_g - l_e) <= 1e-6 * abs(l_e)
        assert relerr(g_g, g_e) < 1e-4
        assert relerr(x_g, x_e) < 1e-6
    # the halved dt changed the result (the graph of the old dt was not replayed)
    assert relerr(out[False][4][2], out[False][0][2]) > 1e-6


@pytest.mark.parametrize("rules", [("amsgrad", "amsgrad"), ("lion", "lion"), ("gd", "dldf"), ("adam", "amsgrad")])
def test_device_descent_rules_match_reference_descend(gpu_ready, exact_case, rules):
    """dmpm_descend: Descend_AMSGrad / Descend_Lion / Descend_GradientDescent /
    Descend_dLdF on the tied control gradient (normalised by its norm), two
    consecutive steps sharing the moment buffers as MaterialPoint's
    momentum / vector / vector_max are shared -- against the same two calls of
    the reference's compiled PointCloud methods (PointCloud.cpp:83-204)."""
    sc, o, loss, L = exact_case
    lr, b1, b2, eps = 1e-2, 0.9, 0.999, 1e-5
    with make_ctx(sc, "fp32", o.target, adjoint="exact", control="tied") as c:
        c.setup(L)
        c.forward(0)
        c.loss()
        c.backward(0)
        g = c.control_grad()
        d = c.get(0, "dFc")
        outs = []
        for t, rule in enumerate(rules, start=1):
            if rule == "adam":
                c.adam_step(t=t, lr=lr, beta1=b1, beta2=b2, eps=eps)
            else:
                c.descend(rule, lr, t=t, beta1=b1, beta2=b2, eps=eps)
            outs.append(c.get(0, "dFc"))
        with pytest.raises(dmpm.DmpmError):
            c.descend("amsgrad", lr, t=0)
        # an unknown rule is rejected by the C ABI itself
        assert c.lib.dmpm_descend(c.h, 0, 9, lr, b1, b2, eps, 1, 1) == dmpm.ERR_ARG
    wants = _reference_descent(sc, d, g, [(r, t) for t, r in enumerate(rules, start=1)], lr, b1, b2, eps)
    for (rule, got, want) in zip(rules, outs, wants):
        step = want - d
        assert np.linalg.norm(got - d - step) <= 1e-5 * np.linalg.norm(step), rule
