"""ctypes wrappers over the CPU oracle libraries (test infrastructure only).

OracleGraph wraps oracle/lib/liboracle.so (this repository's restatement of the
reference algorithm); RefGraph wraps oracle/_ref/libref_fp{32,64}.so (the
reference's own sources, built by oracle/build_ref.sh).  Both expose the same
small API so a test can compare them field by field:

    g = OracleGraph(scene, "f64"); g.setup(L); g.forward(0); L = g.loss(); g.backward(0)
    g.get(layer, "x")  -> (N, 3);  g.get(layer, "F") -> (N, 3, 3);  g.get(layer, "grid_m") -> (G,)
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "lib", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")


def reference_source_dir() -> str:
    """Where the reference's source tree lies: $DMPM_REFERENCE_DIR, else a
    directory named "reference" beside this repository's checkout.  Only the
    recipes that compile the reference (and the tests that call its tools)
    read it; nothing on the GPU side does."""
    env = os.environ.get("DMPM_REFERENCE_DIR")
    if env:
        return env
    repo = os.path.dirname(HERE)
    return os.path.join(os.path.dirname(repo), "reference")

_P = ctypes.c_void_p


def build_oracle(force: bool = False) -> str:
    """Compile oracle/dmpm_oracle.cpp into oracle/lib/liboracle.so."""
    src = os.path.join(HERE, "dmpm_oracle.cpp")
    if force or not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        os.makedirs(os.path.dirname(ORACLE_SO), exist_ok=True)
        subprocess.check_call(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-o", ORACLE_SO, src])
    return ORACLE_SO


def _np_dtype(prec: str):
    return np.float32 if prec == "f32" else np.float64


def _c_real(prec: str):
    return ctypes.c_float if prec == "f32" else ctypes.c_double


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_P)


def _cm(M):
    return np.ascontiguousarray(np.asarray(M).transpose(0, 2, 1).reshape(-1, 9))


def _from_cm(a):
    return np.asarray(a).reshape(-1, 3, 3).transpose(0, 2, 1)


_VEC3 = {"x", "v", "dLdx", "dLdv", "dLdv_next", "grid_v", "grid_p", "grid_dLdv", "grid_dLdp"}
_SCAL = {"grid_m", "grid_dLdm", "vol", "m", "lam", "mu"}


_lib_cache = {}


def load_oracle():
    if "oracle" not in _lib_cache:
        _lib_cache["oracle"] = ctypes.CDLL(build_oracle())
    return _lib_cache["oracle"]


def ref_available(prec: str = "f64") -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_fp%s.so" % prec[1:]))


def load_ref(prec: str):
    key = "ref" + prec
    if key not in _lib_cache:
        path = os.path.join(REF_DIR, "libref_fp%s.so" % prec[1:])
        if not os.path.exists(path):
            raise FileNotFoundError("reference build missing: %s (run oracle/build_ref.sh)" % path)
        _lib_cache[key] = ctypes.CDLL(path)
    return _lib_cache[key]


class _Arrays:
    def __init__(self, scene, prec):
        dt = _np_dtype(prec)
        self.keep = []
        c = lambda a: self._k(np.ascontiguousarray(a, dtype=dt))
        self.x = c(scene.x)
        self.v = c(scene.v)
        self.F = c(_cm(scene.F))
        self.C = c(_cm(scene.C))
        self.dFc = c(_cm(scene.dFc))
        self.m = c(scene.m)
        self.vol = c(scene.vol)
        self.lam = c(scene.lam)
        self.mu = c(scene.mu)
        self.mn = c(scene.min_point)

    def _k(self, a):
        self.keep.append(a)
        return a


class OracleGraph:
    """Graph over oracle/dmpm_oracle.cpp (modes: 0 = RefCompat, 1 = Exact)."""

    def __init__(self, scene, prec: str = "f64", target_m: Optional[np.ndarray] = None):
        self.prec, self.sfx = prec, prec
        self.scene = scene
        self.lib = load_oracle()
        self.dt_np = _np_dtype(prec)
        R = _c_real(prec)
        self.R = R
        a = _Arrays(scene, prec)
        self._a = a
        if target_m is None:
            target_m = oracle_p2g_mass(scene.target_points, scene.target_mp, scene.dims, scene.dx,
                                       scene.min_point, prec)
        self.target = np.ascontiguousarray(target_m, dtype=self.dt_np)
        f = getattr(self.lib, "or_graph_create_" + prec)
        f.restype = _P
        f.argtypes = [ctypes.c_int] + [_P] * 9 + [ctypes.c_int] * 3 + [R, _P, _P]
        self.h = f(scene.n, _ptr(a.x), _ptr(a.v), _ptr(a.F), _ptr(a.C), _ptr(a.dFc), _ptr(a.m), _ptr(a.vol),
                   _ptr(a.lam), _ptr(a.mu), *scene.dims, scene.dx, _ptr(a.mn), _ptr(self.target))
        self.G = int(np.prod(scene.dims))
        self.n = scene.n

    def _fn(self, name, restype=None, argtypes=None):
        f = getattr(self.lib, name + "_" + self.sfx)
        f.restype = restype
        if argtypes is not None:
            f.argtypes = argtypes
        return f

    def calc_volumes(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=self.dt_np)
        self._fn("or_graph_calc_volumes", None, [_P, _P])(self.h, _ptr(out))
        return out

    def setup(self, num_layers, dt, drag=0.0, f_ext=(0, 0, 0), smoothing=0.0):
        fe = np.ascontiguousarray(f_ext, dtype=self.dt_np)
        self._fe = fe
        self._fn("or_graph_setup", None, [_P, ctypes.c_int, self.R, self.R, _P, self.R])(
            self.h, num_layers, dt, drag, _ptr(fe), smoothing)
        self.num_layers = num_layers

    def forward(self, start=0):
        self._fn("or_graph_forward", None, [_P, ctypes.c_int])(self.h, start)

    def loss(self) -> float:
        return float(self._fn("or_graph_loss", ctypes.c_double, [_P])(self.h))

    def backward(self, control=0, mode=0):
        self._fn("or_graph_backward", None, [_P, ctypes.c_int, ctypes.c_int])(self.h, control, mode)

    def _size(self, name):
        if name.startswith("grid_"):
            return self.G * (3 if name in _VEC3 else 1)
        if name == "vol":
            return self.n
        return self.n * (3 if name in _VEC3 else 9)

    def get(self, layer, name):
        out = np.zeros(self._size(name), dtype=self.dt_np)
        r = self._fn("or_graph_get", ctypes.c_int, [_P, ctypes.c_int, ctypes.c_char_p, _P])(
            self.h, layer, name.encode(), _ptr(out))
        if r < 0:
            raise KeyError(name)
        return _shape(out, name)

    def set(self, layer, name, value):
        if name in ("F", "C", "dFc"):
            arr = np.ascontiguousarray(_cm(value), dtype=self.dt_np)
        else:
            arr = np.ascontiguousarray(value, dtype=self.dt_np)
        r = self._fn("or_graph_set", ctypes.c_int, [_P, ctypes.c_int, ctypes.c_char_p, _P])(
            self.h, layer, name.encode(), _ptr(arr))
        if r < 0:
            raise KeyError(name)

    def __del__(self):
        try:
            self._fn("or_graph_destroy", None, [_P])(self.h)
        except Exception:
            pass


def _shape(out, name):
    if name in _VEC3:
        return out.reshape(-1, 3)
    if name in _SCAL:
        return out
    return _from_cm(out)


def oracle_p2g_mass(points, mp, dims, dx, mn, prec="f64"):
    lib = load_oracle()
    dt = _np_dtype(prec)
    R = _c_real(prec)
    f = getattr(lib, "or_p2g_mass_" + prec)
    f.restype = None
    f.argtypes = [ctypes.c_int, _P, R, ctypes.c_int, ctypes.c_int, ctypes.c_int, R, _P, _P]
    x = np.ascontiguousarray(points, dtype=dt)
    m = np.ascontiguousarray(mn, dtype=dt)
    out = np.zeros(int(np.prod(dims)), dtype=dt)
    f(x.shape[0], _ptr(x), mp, dims[0], dims[1], dims[2], dx, _ptr(m), _ptr(out))
    return out


# Field codes of oracle/ref_driver.cpp
_REF_PF = {"x": 0, "v": 1, "F": 2, "C": 3, "P": 4, "m": 5, "vol": 6, "lam": 7, "mu": 8, "dFc": 9, "dLdx": 10,
           "dLdv": 11, "dLdF": 12, "dLdC": 13, "dLdP": 14, "dLdv_next": 15, "dLdC_next": 16, "momentum": 17,
           "vector": 18}
_REF_GF = {"grid_m": 0, "grid_v": 1, "grid_p": 2, "grid_dLdv": 3, "grid_dLdp": 4, "grid_dLdm": 5, "grid_x": 6}


class RefGraph:
    """Graph over the reference's own CompGraph (oracle/_ref).  RefCompat only."""

    def __init__(self, scene, prec: str = "f64", target_m: Optional[np.ndarray] = None, target_from_points=True):
        self.prec = prec
        self.lib = load_ref(prec)
        self.dt_np = _np_dtype(prec)
        R = _c_real(prec)
        self.R = R
        a = _Arrays(scene, prec)
        self._a = a
        L = self.lib
        L.ref_scene_create.restype = _P
        L.ref_scene_create.argtypes = [ctypes.c_int] + [_P] * 9 + [ctypes.c_int] * 3 + [R, _P]
        self.h = L.ref_scene_create(scene.n, _ptr(a.x), _ptr(a.v), _ptr(a.F), _ptr(a.C), _ptr(a.dFc), _ptr(a.m),
                                    _ptr(a.vol), _ptr(a.lam), _ptr(a.mu), *scene.dims, scene.dx, _ptr(a.mn))
        self.G = int(np.prod(scene.dims))
        self.n = scene.n
        if target_m is not None:
            t = np.ascontiguousarray(target_m, dtype=self.dt_np)
            L.ref_scene_set_target_mass.argtypes = [_P, _P]
            L.ref_scene_set_target_mass(self.h, _ptr(t))
        elif target_from_points:
            tp = np.ascontiguousarray(scene.target_points, dtype=self.dt_np)
            L.ref_scene_target_from_points.argtypes = [_P, ctypes.c_int, _P, R]
            L.ref_scene_target_from_points(self.h, tp.shape[0], _ptr(tp), scene.target_mp)

    def target_mass(self):
        out = np.zeros(self.G, dtype=self.dt_np)
        self.lib.ref_scene_get_target_mass.argtypes = [_P, _P]
        self.lib.ref_scene_get_target_mass(self.h, _ptr(out))
        return out

    def calc_volumes(self):
        self.lib.ref_scene_calc_volumes.argtypes = [_P]
        self.lib.ref_scene_calc_volumes(self.h)
        out = np.zeros(self.n, dtype=self.dt_np)
        self.lib.ref_scene_get_particles.argtypes = [_P, ctypes.c_int, _P]
        self.lib.ref_scene_get_particles(self.h, _REF_PF["vol"], _ptr(out))
        return out

    def setup(self, num_layers, dt, drag=0.0, f_ext=(0, 0, 0), smoothing=0.0):
        fe = np.ascontiguousarray(f_ext, dtype=self.dt_np)
        self._fe = fe
        self.lib.ref_graph_setup.argtypes = [_P, ctypes.c_int, self.R, self.R, _P, self.R]
        self.lib.ref_graph_setup(self.h, num_layers, dt, drag, _ptr(fe), smoothing)
        self.num_layers = num_layers

    def forward(self, start=0):
        self.lib.ref_graph_forward.argtypes = [_P, ctypes.c_int]
        self.lib.ref_graph_forward(self.h, start)

    def loss(self) -> float:
        self.lib.ref_graph_loss.restype = self.R
        self.lib.ref_graph_loss.argtypes = [_P]
        return float(self.lib.ref_graph_loss(self.h))

    def backward(self, control=0, mode=0):
        assert mode == 0, "the reference implements its own adjoint only"
        self.lib.ref_graph_backward.argtypes = [_P, ctypes.c_int]
        self.lib.ref_graph_backward(self.h, control)

    def get(self, layer, name):
        if name.startswith("grid_"):
            w = 3 if name in _VEC3 or name == "grid_x" else 1
            out = np.zeros(self.G * w, dtype=self.dt_np)
            self.lib.ref_graph_get_grid.argtypes = [_P, ctypes.c_int, ctypes.c_int, _P]
            self.lib.ref_graph_get_grid(self.h, layer, _REF_GF[name], _ptr(out))
            return out.reshape(-1, 3) if w == 3 else out
        code = _REF_PF[name]
        w = 3 if name in _VEC3 else (1 if name in _SCAL else 9)
        out = np.zeros(self.n * w, dtype=self.dt_np)
        self.lib.ref_graph_get_particles.argtypes = [_P, ctypes.c_int, ctypes.c_int, _P]
        self.lib.ref_graph_get_particles(self.h, layer, code, _ptr(out))
        return _shape(out, name)

    def set(self, layer, name, value):
        code = _REF_PF[name]
        matrix = name not in _VEC3 and name not in _SCAL  # 3x3 fields are stored column-major
        arr = np.ascontiguousarray(_cm(value) if matrix else value, dtype=self.dt_np)
        self._keep_set = arr
        self.lib.ref_graph_set_particles.argtypes = [_P, ctypes.c_int, ctypes.c_int, _P]
        self.lib.ref_graph_set_particles(self.h, layer, code, _ptr(arr))

    def descend(self, rule: str, layer: int, lr: float, gnorm: float, beta1: float = 0.9, beta2: float = 0.999,
                eps: float = 1e-5, t: int = 1):
        """One step of PointCloud::Descend_<rule> on a layer (PointCloud.cpp:83-204):
        adam, amsgrad, lion (beta1 as its beta), gd, dldf."""
        R, I = self.R, ctypes.c_int
        if rule in ("adam", "amsgrad"):
            fn = getattr(self.lib, "ref_graph_descend_" + rule)
            fn.argtypes = [_P, I, R, R, R, R, R, I]
            fn(self.h, layer, lr, gnorm, beta1, beta2, eps, t)
        elif rule == "lion":
            self.lib.ref_graph_descend_lion.argtypes = [_P, I, R, R, R]
            self.lib.ref_graph_descend_lion(self.h, layer, lr, beta1, gnorm)
        elif rule in ("gd", "dldf"):
            fn = getattr(self.lib, "ref_graph_descend_" + rule)
            fn.argtypes = [_P, I, R, R]
            fn(self.h, layer, lr, gnorm)
        else:
            raise ValueError(rule)

    def dldf_norm_stochastic(self, layer: int, idx) -> float:
        """PointCloud::Compute_dLdF_Norm_Stochastic over the given indices."""
        a = np.ascontiguousarray(idx, dtype=np.int32)
        fn = self.lib.ref_graph_dldf_norm_stochastic
        fn.restype = self.R
        fn.argtypes = [_P, ctypes.c_int, _P, ctypes.c_int]
        return float(fn(self.h, layer, _ptr(a), len(a)))

    def descend_adam_stochastic(self, layer: int, lr: float, gnorm: float, beta1: float, beta2: float, eps: float,
                                t: int, idx):
        """PointCloud::Descend_Adam_Stochastic on the given indices."""
        a = np.ascontiguousarray(idx, dtype=np.int32)
        R, I = self.R, ctypes.c_int
        fn = self.lib.ref_graph_descend_adam_stochastic
        fn.argtypes = [_P, I, R, R, R, R, R, I, _P, I]
        fn(self.h, layer, lr, gnorm, beta1, beta2, eps, t, _ptr(a), len(a))

    def time_forward_multithread(self, steps, threads) -> float:
        self.lib.ref_time_forward_multithread.restype = ctypes.c_double
        self.lib.ref_time_forward_multithread.argtypes = [_P, ctypes.c_int, ctypes.c_int]
        return float(self.lib.ref_time_forward_multithread(self.h, steps, threads))

    def time_loss_backward(self):
        self.lib.ref_time_loss_backward.restype = ctypes.c_double
        out = np.zeros(1, dtype=self.dt_np)
        self.lib.ref_time_loss_backward.argtypes = [_P, _P]
        t = float(self.lib.ref_time_loss_backward(self.h, _ptr(out)))
        return t, float(out[0])

    def __del__(self):
        try:
            self.lib.ref_scene_destroy.argtypes = [_P]
            self.lib.ref_scene_destroy(self.h)
        except Exception:
            pass


# ---------------------------------------------------------------- elementary functions
class Elementary:
    """Per-matrix functions of the oracle (kind='oracle') or the reference (kind='ref')."""

    def __init__(self, kind="oracle", prec="f64"):
        self.kind, self.prec = kind, prec
        self.lib = load_oracle() if kind == "oracle" else load_ref(prec)
        self.dt = _np_dtype(prec)
        self.R = _c_real(prec)

    def _f(self, oname, rname):
        return getattr(self.lib, (oname + "_" + self.prec) if self.kind == "oracle" else rname)

    def _m(self, M):
        return np.ascontiguousarray(np.asarray(M, dtype=self.dt).T.reshape(9))

    def _u(self, a):
        return a.reshape(3, 3).T.copy()

    def bspline(self, x):
        f = self._f("or_bspline", "ref_bspline"); f.restype = self.R; f.argtypes = [self.R]
        return float(f(x))

    def bspline_slope(self, x):
        f = self._f("or_bspline_slope", "ref_bspline_slope"); f.restype = self.R; f.argtypes = [self.R]
        return float(f(x))

    def polar(self, F):
        f = self._f("or_polar", "ref_polar"); f.argtypes = [_P] * 3; f.restype = None
        a = self._m(F); R = np.zeros(9, self.dt); S = np.zeros(9, self.dt)
        f(_ptr(a), _ptr(R), _ptr(S))
        return self._u(R), self._u(S)

    def svd(self, F):
        f = self._f("or_svd", "ref_svd"); f.argtypes = [_P] * 4; f.restype = None
        a = self._m(F); U = np.zeros(9, self.dt); s = np.zeros(3, self.dt); V = np.zeros(9, self.dt)
        f(_ptr(a), _ptr(U), _ptr(s), _ptr(V))
        return self._u(U), s, self._u(V)

    def djfit_fd(self, F):
        """The reference's d_JFit_dF_FD (Elasticity.cpp:7-72): T[a][b](i, j) =
        d(J F^-T)_ab / dF_ij by central differences, as an (3, 3, 3, 3) array."""
        assert self.kind == "ref", "the oracle has no standalone d_JFit_dF_FD"
        f = self.lib.ref_djfit_fd; f.argtypes = [_P, _P]; f.restype = None
        a = self._m(F); out = np.zeros(81, self.dt)
        f(_ptr(a), _ptr(out))
        return out.reshape(3, 3, 3, 3)

    def pk(self, F, lam, mu):
        f = self._f("or_pk", "ref_pk"); f.argtypes = [_P, self.R, self.R, _P]; f.restype = None
        a = self._m(F); P = np.zeros(9, self.dt)
        f(_ptr(a), lam, mu, _ptr(P))
        return self._u(P)

    def energy(self, F, lam, mu):
        f = self._f("or_energy", "ref_energy"); f.argtypes = [_P, self.R, self.R]; f.restype = self.R
        return float(f(_ptr(self._m(F)), lam, mu))

    def d2(self, F, lam, mu, dF, exact=False):
        if self.kind == "ref":
            assert not exact
            f = self.lib.ref_d2
        else:
            f = getattr(self.lib, ("or_d2_exact_" if exact else "or_d2_ref_") + self.prec)
        f.argtypes = [_P, self.R, self.R, _P, _P]; f.restype = None
        a = self._m(F); b = self._m(dF); out = np.zeros(9, self.dt)
        f(_ptr(a), lam, mu, _ptr(b), _ptr(out))
        return self._u(out)
