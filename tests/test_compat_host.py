"""Host-side parts of the compat C++ API (no GPU): PointCloud's minibatch
variants against the reference's own Compute_dLdF_Norm_Stochastic and
Descend_Adam_Stochastic (its float build, compiled from its sources into
oracle/_ref), Grid::QueryPoint_CubicBSpline against the stencil the
reference forms (floor((p - min) / dx) - 1 by division, nodes outside the
grid left out, i outermost), flatten / unflatten and the minibatch indices."""
import os
import subprocess

import numpy as np
import pytest

import scenes
from oracle.lib import RefGraph, ref_available

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "a-differentiable-material-point-method-for-shape-morphing_b200")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    import build as pkg_build

    pkg_build.build_compat()
    out = tmp_path_factory.mktemp("cpp") / "compat_host_check"
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-DDMPM_COMPAT_NO_EIGEN", "-I", os.path.join(PKG, "compat"),
                           os.path.join(REPO, "tests", "cpp", "compat_host_check.cpp"), "-L", PKG, "-ldmpm_compat",
                           "-ldmpm", "-Wl,-rpath," + PKG, "-o", str(out)])
    return str(out)


def _cm(M):
    return np.ascontiguousarray(np.asarray(M).transpose(0, 2, 1).reshape(-1, 9))


@pytest.mark.skipif(not ref_available("f32"), reason="the reference's float build (oracle/_ref) is not compiled")
def test_stochastic_descent_and_stencil_queries(exe, tmp_path):
    sc = scenes.small_scene(seed=9, res=8, radius=0.3)
    rng = np.random.default_rng(4)
    n = sc.n
    g = rng.normal(size=(n, 3, 3)).astype(np.float32)
    d = (1e-3 * rng.normal(size=(n, 3, 3))).astype(np.float32)
    idx = rng.permutation(n)[: n // 4].astype(np.int32)
    lr, b1, b2, eps, t0 = 1e-2, 0.9, 0.999, 1e-5, 0
    dims, dx, mn = (6, 5, 7), 0.25, (-0.1, 0.2, 0.05)
    pts = rng.uniform(-0.6, 2.0, size=(40, 3)).astype(np.float32)
    pts[0] = (0.0, 0.0, 0.0)
    with open(tmp_path / "in.bin", "wb") as f:
        f.write(np.array([n, len(idx), t0], dtype=np.int32).tobytes())
        f.write(_cm(g).astype(np.float32).tobytes())
        f.write(_cm(d).astype(np.float32).tobytes())
        f.write(idx.tobytes())
        f.write(np.array([lr, b1, b2, eps], dtype=np.float32).tobytes())
        f.write(np.array(dims, dtype=np.int32).tobytes())
        f.write(np.array([dx, *mn], dtype=np.float32).tobytes())
        f.write(np.array([len(pts)], dtype=np.int32).tobytes())
        f.write(pts.tobytes())
    res = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True,
                         timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    raw = (tmp_path / "out.bin").read_bytes()
    norm = np.frombuffer(raw[:4], dtype=np.float32)[0]
    dfc = np.frombuffer(raw[4:4 + 36 * n], dtype=np.float32).reshape(n, 3, 3).transpose(0, 2, 1)
    ints = np.frombuffer(raw[4 + 36 * n:], dtype=np.int32)

    # the reference's own functions on the same points
    r = RefGraph(sc, "f32", target_m=np.zeros(int(np.prod(sc.dims))), target_from_points=False)
    r.setup(2, sc.dt)
    r.set(0, "dLdF", g.astype(np.float64))
    r.set(0, "dFc", d.astype(np.float64))
    rnorm = r.dldf_norm_stochastic(0, idx)
    assert abs(norm - rnorm) <= 1e-6 * rnorm
    for t in (t0, t0 + 1):
        r.descend_adam_stochastic(0, lr, rnorm, b1, b2, eps, t, idx)
    want = r.get(0, "dFc")
    step = want - d
    assert np.linalg.norm(dfc - want) <= 1e-5 * np.linalg.norm(step)
    untouched = np.setdiff1d(np.arange(n), idx)
    assert np.array_equal(dfc[untouched], d[untouched])

    # stencil queries
    o = 0
    for p in pts:
        cnt = ints[o]
        got = ints[o + 1:o + 1 + 3 * cnt].reshape(-1, 3)
        o += 1 + 3 * cnt
        b = np.floor((p - np.float32(mn)) / np.float32(dx)).astype(np.int64) - 1
        want_ijk = [(b[0] + i, b[1] + j, b[2] + k) for i in range(4) for j in range(4) for k in range(4)
                    if 0 <= b[0] + i < dims[0] and 0 <= b[1] + j < dims[1] and 0 <= b[2] + k < dims[2]]
        assert [tuple(x) for x in got] == want_ijk
    assert ints[o] == n // 3 and ints[o + 1] == 1
    assert ints[o + 2] == 1
