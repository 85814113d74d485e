"""The engine's device math (csrc/mat3.cuh, svd3.cuh, elasticity.cuh) compiled
for the host and compared with the reference's golden vectors and the oracle.
This exercises the exact source the kernels use, without a GPU."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from oracle.lib import Elementary
from tests.helpers import load_golden, relerr

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "native", "math_host.cu")
LIB = os.path.join(HERE, "native", "libmath_host.so")
CSRC = os.path.join(os.path.dirname(HERE), "a-differentiable-material-point-method-for-shape-morphing_b200", "csrc")
P = ctypes.c_void_p


@pytest.fixture(scope="module")
def mh():
    deps = [SRC] + [os.path.join(CSRC, f) for f in ("mat3.cuh", "svd3.cuh", "elasticity.cuh")]
    if not os.path.exists(LIB) or any(os.path.getmtime(d) > os.path.getmtime(LIB) for d in deps):
        subprocess.check_call(["/usr/local/cuda/bin/nvcc", "-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                               "-Wno-deprecated-gpu-targets", "-I", CSRC, "-o", LIB, SRC])
    lib = ctypes.CDLL(LIB)
    for s in ("f64",):
        getattr(lib, "mh_pk_" + s).argtypes = [P, ctypes.c_double, ctypes.c_double, P]
        getattr(lib, "mh_d2_" + s).argtypes = [P, ctypes.c_double, ctypes.c_double, P, ctypes.c_int, P]
        getattr(lib, "mh_bspline_" + s).restype = ctypes.c_double
        getattr(lib, "mh_bspline_" + s).argtypes = [ctypes.c_double]
        getattr(lib, "mh_bspline_slope_" + s).restype = ctypes.c_double
        getattr(lib, "mh_bspline_slope_" + s).argtypes = [ctypes.c_double]
    return lib


def cm(M):
    return np.ascontiguousarray(np.asarray(M, dtype=np.float64).T.reshape(9))


def un(a):
    return a.reshape(3, 3).T


def polar(mh, F):
    R = np.zeros(9); S = np.zeros(9)
    mh.mh_polar_f64(cm(F).ctypes.data_as(P), R.ctypes.data_as(P), S.ctypes.data_as(P))
    return un(R), un(S)


def svd(mh, F):
    U = np.zeros(9); s = np.zeros(3); V = np.zeros(9)
    a = cm(F)
    mh.mh_svd_f64(a.ctypes.data_as(P), U.ctypes.data_as(P), s.ctypes.data_as(P), V.ctypes.data_as(P))
    return un(U), s, un(V)


def test_against_golden(mh):
    g = load_golden("elementary_f64")
    lam, mu = float(g["lam"]), float(g["mu"])
    for F, dF, R, S, Pg, d2 in zip(g["F"], g["dF"], g["R"], g["S"], g["P"], g["d2"]):
        r, s = polar(mh, F)
        assert relerr(r, R) < 1e-9 and relerr(s, S) < 1e-9
        out = np.zeros(9)
        mh.mh_pk_f64(cm(F).ctypes.data_as(P), lam, mu, out.ctypes.data_as(P))
        assert relerr(un(out), Pg) < 1e-8
        mh.mh_d2_f64(cm(F).ctypes.data_as(P), lam, mu, cm(dF).ctypes.data_as(P), 0, out.ctypes.data_as(P))
        assert relerr(un(out), d2) < 1e-8
    for x, b, bs in zip(g["bx"], g["b"], g["bs"]):
        assert mh.mh_bspline_f64(x) == b and mh.mh_bspline_slope_f64(x) == bs


def test_svd_convention_and_hard_cases(mh):
    """Rotation-variant convention on random, near-rotation, repeated-sigma,
    inverted and nearly singular matrices."""
    rng = np.random.default_rng(11)
    ref = Elementary("oracle", "f64")
    for t in range(600):
        k = t % 5
        if k == 0:
            F = rng.normal(size=(3, 3))
        elif k == 1:
            Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
            Q *= np.sign(np.linalg.det(Q))
            F = Q @ np.diag([1.3, 1.3, 0.6]) @ Q.T
        elif k == 2:
            F = np.eye(3) + 0.3 * rng.normal(size=(3, 3))
            F[:, 1] *= -1
        elif k == 3:
            F = np.outer(rng.normal(size=3), rng.normal(size=3)) + 1e-9 * rng.normal(size=(3, 3))
        else:
            F = np.eye(3) + 1e-4 * rng.normal(size=(3, 3))
        U, s, V = svd(mh, F)
        assert np.allclose(U @ np.diag(s) @ V.T, F, atol=1e-12 * max(1.0, np.abs(F).max()))
        assert abs(np.linalg.det(U) - 1) < 1e-12 and abs(np.linalg.det(V) - 1) < 1e-12
        assert s[0] >= 0 and s[1] >= 0 and abs(s[0]) >= abs(s[1]) - 1e-12 and abs(s[1]) >= abs(s[2]) - 1e-12
        if k != 3:
            r, _ = polar(mh, F)
            ro, _ = ref.polar(F)
            assert relerr(r, ro) < 1e-9


def test_exact_stress_derivative_matches_fd(mh):
    rng = np.random.default_rng(5)
    ref = Elementary("oracle", "f64")
    lam, mu = 90.0, 60.0
    for _ in range(50):
        F = np.eye(3) + 0.2 * rng.normal(size=(3, 3))
        dF = rng.normal(size=(3, 3))
        out = np.zeros(9)
        mh.mh_d2_f64(cm(F).ctypes.data_as(P), lam, mu, cm(dF).ctypes.data_as(P), 1, out.ctypes.data_as(P))
        h = 1e-6
        fd = (ref.pk(F + h * dF, lam, mu) - ref.pk(F - h * dF, lam, mu)) / (2 * h)
        assert relerr(un(out), fd) < 1e-7


def test_newton_polar_matches_svd_polar(mh):
    """polar_newton (the FP32 path's k_stress, det F > 0) gives polar3's R and S
    to rounding, and declines inverted or near-singular F (left to the SVD)."""
    mh.mh_polar_newton_f64.restype = ctypes.c_int
    rng = np.random.default_rng(2024)
    cases = []
    for t in range(400):
        k = t % 4
        if k == 0:
            F = np.eye(3) + 1e-3 * rng.normal(size=(3, 3))
        elif k == 1:
            F = np.eye(3) + 0.3 * rng.normal(size=(3, 3))
        elif k == 2:
            Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
            Q *= np.sign(np.linalg.det(Q))
            F = Q @ np.diag(rng.uniform(0.2, 5.0, 3)) @ Q.T
        else:
            Q1, _ = np.linalg.qr(rng.normal(size=(3, 3)))
            Q1 *= np.sign(np.linalg.det(Q1))
            Q2, _ = np.linalg.qr(rng.normal(size=(3, 3)))
            Q2 *= np.sign(np.linalg.det(Q2))
            F = Q1 @ np.diag(rng.uniform(0.05, 20.0, 3)) @ Q2
        cases.append(F)
    used = 0
    for F in cases:
        R = np.zeros(9)
        S = np.zeros(9)
        ok = mh.mh_polar_newton_f64(cm(F).ctypes.data_as(P), R.ctypes.data_as(P), S.ctypes.data_as(P))
        if np.linalg.det(F) > 1e-3:
            assert ok == 1
        if not ok:
            continue
        used += 1
        R0, S0 = polar(mh, F)
        assert np.abs(un(R) - R0).max() < 1e-12
        assert np.abs(un(S) - S0).max() < 1e-12 * max(1.0, np.abs(S0).max())
    assert used >= 380
    for F in (np.diag([1.0, 1.0, -1.0]), np.diag([1.0, 1.0, 1e-9]), -np.eye(3)):
        R = np.zeros(9)
        S = np.zeros(9)
        assert mh.mh_polar_newton_f64(cm(F).ctypes.data_as(P), R.ctypes.data_as(P), S.ctypes.data_as(P)) == 0


def test_compat_djfit_matches_reference_fd():
    """The compat API's d_JFit_dF_FD (a host utility) against the reference's
    FP64 build on the elementary fixture's 25 matrices, and its closed-form
    d_JFit_dF against it.  The shipped float build's own central differences
    (delta = 1e-6 in float, so one float step of J F^-T near 1 moves an entry by
    0.06) stray from the FP64 build by 6 % of the largest entry at the median
    and 12.5 % at worst over these matrices."""
    import build as pkg_build

    pkg_build.build_compat()
    pkg = os.path.join(os.path.dirname(HERE), "a-differentiable-material-point-method-for-shape-morphing_b200")
    exe = os.path.join(HERE, "native", "jfit_check")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(pkg, "compat"), "-I",
                           os.path.join(os.path.dirname(HERE), "include"), os.path.join(HERE, "cpp", "jfit_check.cpp"),
                           "-L", pkg, "-ldmpm_compat", "-ldmpm", "-Wl,-rpath," + pkg, "-o", exe])
    g64, g32 = load_golden("elementary_f64"), load_golden("elementary_f32")
    Fs = g64["F"]
    stdin = "%d\n" % len(Fs) + "\n".join(" ".join("%.17g" % v for v in F.reshape(9)) for F in Fs) + "\n"
    res = subprocess.run([exe], input=stdin, capture_output=True, text=True, check=True)
    vals = np.array(res.stdout.split(), dtype=np.float64).reshape(len(Fs), 2, 3, 3, 3, 3)
    fd, closed = vals[:, 0], vals[:, 1]
    for k in range(len(Fs)):
        assert relerr(fd[k], g64["djfit"][k]) < 1e-6, k
        assert relerr(closed[k], g64["djfit"][k]) < 1e-5, k
        assert relerr(g32["djfit"][k], g64["djfit"][k]) < 0.15, k
    os.remove(exe)


def test_compat_bspline_is_the_reference_float_bspline():
    """The compat API's CubicBSpline / CubicBSplineSlope (header-only) give the
    shipped float build's values bit for bit on the elementary fixture's sweep."""
    pkg = os.path.join(os.path.dirname(HERE), "a-differentiable-material-point-method-for-shape-morphing_b200")
    exe = os.path.join(HERE, "native", "bspline_check")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(pkg, "compat"),
                           os.path.join(HERE, "cpp", "bspline_check.cpp"), "-o", exe])
    g = load_golden("elementary_f32")
    xs = np.asarray(g["bx"], dtype=np.float32)
    stdin = "%d\n" % len(xs) + "\n".join("%.9g" % x for x in xs) + "\n"
    res = subprocess.run([exe], input=stdin, capture_output=True, text=True, check=True)
    vals = np.array(res.stdout.split(), dtype=np.float32).reshape(len(xs), 2)
    os.remove(exe)
    assert np.array_equal(vals[:, 0], np.asarray(g["b"], dtype=np.float32))
    assert np.array_equal(vals[:, 1], np.asarray(g["bs"], dtype=np.float32))
