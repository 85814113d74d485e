"""The scale of the deterministic mode's integer node sums (csrc/fixscale.h),
compiled for the host: the exponent k keeps n contributions bounded by c below
2^61 after scaling (and above 2^59, so no precision is given away), the clamps
hold for zero, tiny, huge and non-finite bounds, and sums of rounded integers
are the same in every order while staying within the rounding bound of the
exact sum."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "a-differentiable-material-point-method-for-shape-morphing_b200", "csrc")
SRC = os.path.join(HERE, "cpp", "fixscale_api.cpp")
LIB = os.path.join(HERE, "native", "libfixscale.so")


@pytest.fixture(scope="module")
def fx():
    deps = [SRC, os.path.join(CSRC, "fixscale.h")]
    if not os.path.exists(LIB) or any(os.path.getmtime(d) > os.path.getmtime(LIB) for d in deps):
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", CSRC, "-o", LIB, SRC])
    lib = ctypes.CDLL(LIB)
    lib.fx_exponent.restype = ctypes.c_int
    lib.fx_exponent.argtypes = [ctypes.c_uint, ctypes.c_longlong]
    lib.fx_pow2.restype = ctypes.c_float
    lib.fx_pow2.argtypes = [ctypes.c_int]
    lib.fx_sum.restype = ctypes.c_float
    lib.fx_sum.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int,
                           ctypes.POINTER(ctypes.c_longlong)]
    return lib


def bits(c):
    return int(np.array([c], dtype=np.float32).view(np.uint32)[0])


def test_exponent_brackets_the_bound(fx):
    rng = np.random.default_rng(3)
    for _ in range(4000):
        c = np.float32(10.0 ** rng.uniform(-30, 30))
        n = int(10 ** rng.uniform(0, 9.5))
        k = fx.fx_exponent(bits(c), n)
        assert -126 <= k <= 126
        if -126 < k < 126:
            scaled = float(n) * float(c) * 2.0 ** k
            assert 2.0 ** 59 <= scaled < 2.0 ** 61, (c, n, k)


def test_exponent_clamps(fx):
    assert fx.fx_exponent(bits(0.0), 1000) == 126
    assert fx.fx_exponent(bits(1e-38), 10) == 126
    k = fx.fx_exponent(bits(3e38), 1 << 40)  # the largest floats over 2^40 particles still fit
    assert 2.0 ** 59 <= 2.0 ** k * 3e38 * 2.0 ** 40 < 2.0 ** 61
    assert fx.fx_exponent(bits(np.inf), 10) == -126
    assert fx.fx_exponent(0x7FC00000, 10) == -126  # NaN
    for k in (-126, -1, 0, 1, 126, 127):
        assert fx.fx_pow2(k) == np.float32(2.0 ** k)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_integer_sums_do_not_depend_on_order(fx, seed):
    rng = np.random.default_rng(seed)
    n = 5000
    c = np.float32(10.0 ** rng.uniform(-8, 4))
    # signed contributions with B-spline-like weights, some tiny
    x = (rng.uniform(-1, 1, n) * rng.uniform(0, 1, n) ** 6 * c).astype(np.float32)
    k = fx.fx_exponent(bits(np.float32(c * 1.001)), n)
    out = []
    for _ in range(6):
        order = rng.permutation(n).astype(np.int32)
        isum = ctypes.c_longlong()
        v = fx.fx_sum(x.ctypes.data, order.ctypes.data, n, k, ctypes.byref(isum))
        out.append((v, isum.value))
    assert len(set(out)) == 1
    exact = float(np.sum(x.astype(np.float64)))
    # n roundings of at most half a unit 2^-k each, plus the one float rounding of the result
    assert abs(out[0][0] - exact) <= n * 0.5 * 2.0 ** -k + abs(exact) * 2.0 ** -24 + 1e-45
