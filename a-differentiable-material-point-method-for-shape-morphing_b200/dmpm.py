"""Python binding of libdmpm.so (include/dmpm.h) over ctypes.

This is plumbing for tests and the benchmark; the engine and its C ABI are
the product.  There is no CPU fallback: importing works anywhere, but
creating a Context raises DmpmError when the CUDA library or a GPU is missing.

Matrices are numpy (N, 3, 3) arrays indexed [p, row, col]; they are converted
to the ABI's column-major layout here.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libdmpm.so")

# status codes / enums of include/dmpm.h
OK, ERR_ARG, ERR_OOM, ERR_CUDA, ERR_NONFINITE, ERR_STATE, ERR_TOO_LARGE = 0, 1, 2, 3, 4, 5, 6
FP64, FP32_MIXED = 0, 1
ADJ_REFCOMPAT, ADJ_EXACT = 0, 1
CTRL_PER_LAYER, CTRL_TIED = 0, 1
LOSS_REF_LOGMASS, LOSS_L2 = 0, 1
DESCEND = {"adam": 0, "amsgrad": 1, "lion": 2, "gd": 3, "dldf": 4}

FIELDS = {"x": 0, "v": 1, "F": 2, "C": 3, "P": 4, "m": 5, "vol": 6, "lam": 7, "mu": 8, "dFc": 9, "dLdx": 10,
          "dLdv": 11, "dLdF": 12, "dLdC": 13, "dLdP": 14, "dLdv_next": 15, "dLdC_next": 16, "dLdFe": 19}
WIDTH = {"x": 3, "v": 3, "F": 9, "C": 9, "P": 9, "m": 1, "vol": 1, "lam": 1, "mu": 1, "dFc": 9, "dLdx": 3,
         "dLdv": 3, "dLdF": 9, "dLdC": 9, "dLdP": 9, "dLdv_next": 3, "dLdC_next": 9, "dLdFe": 9}
GRID_FIELDS = {"grid_m": 0, "grid_v": 1, "grid_p": 2, "grid_dLdv": 3, "grid_dLdp": 4, "grid_dLdm": 5}
NUM_KERNEL_IDS = 12
GRID_WIDTH = {"grid_m": 1, "grid_v": 3, "grid_p": 3, "grid_dLdv": 3, "grid_dLdp": 3, "grid_dLdm": 1}


class DmpmError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__("dmpm status %d: %s" % (status, message))
        self.status = status


class Params(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("drag", ctypes.c_double), ("f_ext", ctypes.c_double * 3),
                ("smoothing", ctypes.c_double), ("adjoint_mode", ctypes.c_int), ("control_mode", ctypes.c_int),
                ("loss_kind", ctypes.c_int), ("checkpoint_every", ctypes.c_int), ("keep_adjoints", ctypes.c_int),
                ("keep_intermediates", ctypes.c_int), ("block_size", ctypes.c_int), ("tile_cap", ctypes.c_int),
                ("sort_every", ctypes.c_int), ("warp_general", ctypes.c_int), ("control_stride", ctypes.c_int),
                ("eager", ctypes.c_int), ("brick_cells", ctypes.c_int), ("deterministic", ctypes.c_int),
                ("reorder_particles", ctypes.c_int)]


class Instance(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("dim_x", ctypes.c_int), ("dim_y", ctypes.c_int), ("dim_z", ctypes.c_int),
                ("dx", ctypes.c_double), ("min_point", ctypes.c_double * 3), ("steps", ctypes.c_int)]


class BatchLaunch(ctypes.Structure):
    _fields_ = [("sort_every", ctypes.c_int), ("ctas_per_sm", ctypes.c_int), ("particle_block", ctypes.c_int),
                ("use_graph", ctypes.c_int)]


_P = ctypes.c_void_p
_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libdmpm.so; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise DmpmError(ERR_CUDA, "libdmpm.so not built at %s (run __graft_entry__.build())" % path)
    L = ctypes.CDLL(path)
    L.dmpm_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(_P)]
    L.dmpm_destroy.argtypes = [_P]
    L.dmpm_last_error.argtypes = [_P]
    L.dmpm_last_error.restype = ctypes.c_char_p
    L.dmpm_get_info.argtypes = [_P, ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
    L.dmpm_set_grid.argtypes = [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _P]
    L.dmpm_set_params.argtypes = [_P, ctypes.POINTER(Params)]
    L.dmpm_set_device_limit.argtypes = [_P, ctypes.c_int64]
    L.dmpm_default_params.argtypes = [ctypes.POINTER(Params)]
    L.dmpm_default_params.restype = None
    L.dmpm_set_particles.argtypes = [_P, ctypes.c_int] + [_P] * 9
    L.dmpm_set_points_ref.argtypes = [_P, _P, ctypes.c_int]
    L.dmpm_compute_volumes.argtypes = [_P]
    L.dmpm_set_target_mass.argtypes = [_P, _P]
    L.dmpm_rasterize_target.argtypes = [_P, ctypes.c_int, _P, ctypes.c_double]
    L.dmpm_get_target_mass.argtypes = [_P, _P]
    L.dmpm_setup.argtypes = [_P, ctypes.c_int]
    L.dmpm_forward.argtypes = [_P, ctypes.c_int]
    L.dmpm_loss.argtypes = [_P, ctypes.POINTER(ctypes.c_double)]
    L.dmpm_backward.argtypes = [_P, ctypes.c_int]
    L.dmpm_get_particles.argtypes = [_P, ctypes.c_int, ctypes.c_int, _P]
    L.dmpm_set_layer_particles.argtypes = [_P, ctypes.c_int, ctypes.c_int, _P]
    L.dmpm_get_grid.argtypes = [_P, ctypes.c_int, ctypes.c_int, _P]
    L.dmpm_get_control_grad.argtypes = [_P, ctypes.c_int, _P]
    L.dmpm_dldf_norm.argtypes = [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.dmpm_get_points_ref.argtypes = [_P, ctypes.c_int, _P]
    L.dmpm_adam_step.argtypes = [_P, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_int, ctypes.c_int]
    L.dmpm_descend.argtypes = [_P, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                               ctypes.c_double, ctypes.c_int, ctypes.c_int]
    L.dmpm_synchronize.argtypes = [_P]
    L.dmpm_stream.argtypes = [_P]
    L.dmpm_stream.restype = _P
    L.dmpm_launch_count.argtypes = [_P]
    L.dmpm_launch_count.restype = ctypes.c_int64
    L.dmpm_set_profiling.argtypes = [_P, ctypes.c_int]
    L.dmpm_kernel_stats.argtypes = [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)]
    L.dmpm_cell_sort.argtypes = [_P, ctypes.c_int, _P, _P, _P, ctypes.POINTER(ctypes.c_int)]
    L.dmpm_compute_volumes_noalloc.argtypes = [ctypes.c_int, _P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_float, _P, _P, _P]
    L.dmpm_kernel_name.argtypes = [ctypes.c_int]
    L.dmpm_kernel_name.restype = ctypes.c_char_p
    L.dmpm_batch_create.argtypes = [ctypes.c_int, ctypes.c_int, _P, ctypes.POINTER(_P)]
    L.dmpm_batch_destroy.argtypes = [_P]
    L.dmpm_batch_last_error.argtypes = [_P]
    L.dmpm_batch_last_error.restype = ctypes.c_char_p
    L.dmpm_batch_set_params.argtypes = [_P, ctypes.POINTER(Params)]
    L.dmpm_batch_set_particles.argtypes = [_P, ctypes.c_int] + [_P] * 9
    L.dmpm_batch_set_target_mass.argtypes = [_P, ctypes.c_int, _P]
    L.dmpm_batch_set_launch.argtypes = [_P, ctypes.POINTER(BatchLaunch)]
    L.dmpm_batch_get_launch.argtypes = [_P, ctypes.POINTER(BatchLaunch)]
    L.dmpm_batch_setup.argtypes = [_P]
    L.dmpm_batch_gradient.argtypes = [_P, _P]
    L.dmpm_batch_autotune.argtypes = [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.dmpm_batch_get_control_grad.argtypes = [_P, ctypes.c_int, _P]
    L.dmpm_batch_get_particles.argtypes = [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P]
    L.dmpm_batch_info.argtypes = [_P, ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
    L.dmpm_batch_stream.argtypes = [_P, ctypes.POINTER(_P)]
    L.dmpm_mesh_lattice_dims.argtypes = [_P, _P, ctypes.c_float, _P]
    L.dmpm_mesh_lattice_points.argtypes = [_P, ctypes.c_int, _P, ctypes.c_int, _P, _P, ctypes.c_float, _P,
                                           ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
    _lib = L
    return L


def _cm(M) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(M, dtype=np.float64).transpose(0, 2, 1).reshape(-1, 9))


def _from_cm(a) -> np.ndarray:
    return a.reshape(-1, 3, 3).transpose(0, 2, 1)


def _ptr(a) -> Optional[int]:
    """numpy array, torch tensor (data_ptr) or raw int -> address."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


class Context:
    """One engine context (one scene, one stream) on one GPU."""

    def __init__(self, precision: str = "fp32", device: int = 0):
        self.lib = load_library()
        self.precision = FP64 if precision in ("fp64", FP64) else FP32_MIXED
        h = _P()
        st = self.lib.dmpm_create(device, self.precision, ctypes.byref(h))
        if st != OK:
            raise DmpmError(st, "dmpm_create(device=%d) failed (no CUDA device?)" % device)
        self.h = h
        self.n = 0
        self.dims = (0, 0, 0)
        self.num_layers = 0
        self._keep = []

    # -------------------------------------------------------------- plumbing
    def _ck(self, st: int, what: str, allow_nonfinite: bool = False) -> int:
        if st == OK or (allow_nonfinite and st == ERR_NONFINITE):
            return st
        msg = self.lib.dmpm_last_error(self.h)
        raise DmpmError(st, "%s: %s" % (what, msg.decode() if msg else ""))

    def close(self):
        if getattr(self, "h", None):
            self.lib.dmpm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def info(self) -> dict:
        buf = (ctypes.c_int64 * 10)()
        self.lib.dmpm_get_info(self.h, buf, 10)
        keys = ["n", "dim_x", "dim_y", "dim_z", "layers", "precision", "checkpoint_every", "device_bytes",
                "launches", "status"]
        return dict(zip(keys, list(buf)))

    @property
    def launch_count(self) -> int:
        return int(self.lib.dmpm_launch_count(self.h))

    @property
    def stream(self) -> int:
        return int(self.lib.dmpm_stream(self.h) or 0)

    def set_profiling(self, on: bool = True):
        """Bracket every hot-path kernel with CUDA events on the context stream."""
        self._ck(self.lib.dmpm_set_profiling(self.h, int(bool(on))), "set_profiling")

    def kernel_stats(self) -> dict:
        """{kernel name: (total device ms, launches)} since profiling was enabled."""
        out = {}
        for k in range(NUM_KERNEL_IDS):
            ms = ctypes.c_double()
            cnt = ctypes.c_int64()
            self._ck(self.lib.dmpm_kernel_stats(self.h, k, ctypes.byref(ms), ctypes.byref(cnt)), "kernel_stats")
            if cnt.value:
                out[self.lib.dmpm_kernel_name(k).decode()] = (float(ms.value), int(cnt.value))
        return out

    def synchronize(self):
        self._ck(self.lib.dmpm_synchronize(self.h), "synchronize")

    # -------------------------------------------------------------- setup
    def set_device_limit(self, max_bytes: int):
        """Cap the device bytes this context may hold (0 = none); over it, calls fail with ERR_OOM."""
        self._ck(self.lib.dmpm_set_device_limit(self.h, int(max_bytes)), "set_device_limit")

    def set_grid(self, dims: Sequence[int], dx: float = 1.0, min_point=(0.0, 0.0, 0.0)):
        mn = np.ascontiguousarray(min_point, dtype=np.float64)
        self._ck(self.lib.dmpm_set_grid(self.h, int(dims[0]), int(dims[1]), int(dims[2]), float(dx), mn.ctypes.data),
                 "set_grid")
        self.dims = tuple(int(d) for d in dims)

    def set_params(self, dt: float, drag: float = 0.0, f_ext=(0.0, 0.0, 0.0), smoothing: float = 0.0,
                   adjoint: str = "refcompat", control: str = "per_layer", loss: str = "ref",
                   checkpoint_every: int = 0, keep_adjoints: bool = False, keep_intermediates: bool = False,
                   block_size: int = 0, tile_cap: int = 0, sort_every: int = 0, warp_general: bool = False,
                   control_stride: int = 0, eager: bool = False, brick_cells: Optional[int] = None,
                   deterministic: bool = False, reorder_particles: bool = False):
        p = Params()
        self.lib.dmpm_default_params(ctypes.byref(p))
        p.dt, p.drag, p.smoothing = float(dt), float(drag), float(smoothing)
        for i in range(3):
            p.f_ext[i] = float(f_ext[i])
        p.adjoint_mode = ADJ_EXACT if adjoint == "exact" else ADJ_REFCOMPAT
        p.control_mode = CTRL_TIED if control == "tied" else CTRL_PER_LAYER
        p.loss_kind = LOSS_L2 if loss == "l2" else LOSS_REF_LOGMASS
        p.checkpoint_every = int(checkpoint_every)
        p.keep_adjoints = int(bool(keep_adjoints))
        p.keep_intermediates = int(bool(keep_intermediates))
        p.block_size = int(block_size)
        p.tile_cap = int(tile_cap)
        p.sort_every = int(sort_every)
        p.warp_general = int(bool(warp_general))
        p.control_stride = int(control_stride)
        p.eager = int(bool(eager))
        if brick_cells is not None:  # else the library default (bricks of 2^3 cells for G2P)
            p.brick_cells = int(brick_cells)
        p.deterministic = int(bool(deterministic))
        p.reorder_particles = int(bool(reorder_particles))
        self._ck(self.lib.dmpm_set_params(self.h, ctypes.byref(p)), "set_params")
        self.params = p

    def set_particles(self, x, m, lam, mu, v=None, F=None, C=None, dFc=None, vol=None):
        n = int(np.asarray(x).shape[0])
        arrs = {
            "x": np.ascontiguousarray(x, dtype=np.float64),
            "v": None if v is None else np.ascontiguousarray(v, dtype=np.float64),
            "F": None if F is None else _cm(F),
            "C": None if C is None else _cm(C),
            "dFc": None if dFc is None else _cm(dFc),
            "m": np.ascontiguousarray(m, dtype=np.float64),
            "vol": None if vol is None else np.ascontiguousarray(vol, dtype=np.float64),
            "lam": np.ascontiguousarray(lam, dtype=np.float64),
            "mu": np.ascontiguousarray(mu, dtype=np.float64),
        }
        self._set_particles_raw(n, **arrs)

    def _set_particles_raw(self, n, x, v, F, C, dFc, m, vol, lam, mu):
        """Upload already laid-out host buffers (numpy, torch or int pointers)."""
        st = self.lib.dmpm_set_particles(self.h, n, _ptr(x), _ptr(v), _ptr(F), _ptr(C), _ptr(dFc), _ptr(m),
                                         _ptr(vol), _ptr(lam), _ptr(mu))
        self._ck(st, "set_particles")
        self.n = n

    def set_points_ref(self, points: np.ndarray):
        """points: float32 array (N, 118) in the reference MaterialPoint layout."""
        pts = np.ascontiguousarray(points, dtype=np.float32)
        self._ck(self.lib.dmpm_set_points_ref(self.h, pts.ctypes.data, pts.shape[0]), "set_points_ref")
        self.n = pts.shape[0]

    def compute_volumes(self):
        self._ck(self.lib.dmpm_compute_volumes(self.h), "compute_volumes")

    def set_target_mass(self, m):
        a = np.ascontiguousarray(m, dtype=np.float64)
        self._ck(self.lib.dmpm_set_target_mass(self.h, a.ctypes.data), "set_target_mass")

    def rasterize_target(self, points, point_mass: float):
        a = np.ascontiguousarray(points, dtype=np.float64)
        self._ck(self.lib.dmpm_rasterize_target(self.h, a.shape[0], a.ctypes.data, float(point_mass)),
                 "rasterize_target")

    def target_mass(self) -> np.ndarray:
        out = np.empty(int(np.prod(self.dims)), dtype=np.float64)
        self._ck(self.lib.dmpm_get_target_mass(self.h, out.ctypes.data), "get_target_mass")
        return out

    def load_scene(self, scene, with_volumes: bool = True, with_target: bool = True):
        """Grid, particles, volumes (CalculatePointCloudVolumes) and target raster of a scenes.Scene."""
        self.set_grid(scene.dims, scene.dx, scene.min_point)
        self.set_particles(scene.x, scene.m, scene.lam, scene.mu, v=scene.v, F=scene.F, C=scene.C, dFc=scene.dFc,
                           vol=scene.vol)
        if with_volumes:
            self.compute_volumes()
        if with_target:
            self.rasterize_target(scene.target_points, scene.target_mp)

    # -------------------------------------------------------------- graph
    def setup(self, num_layers: int):
        self._ck(self.lib.dmpm_setup(self.h, int(num_layers)), "setup")
        self.num_layers = int(num_layers)

    def forward(self, start_layer: int = 0, allow_nonfinite: bool = True) -> int:
        return self._ck(self.lib.dmpm_forward(self.h, int(start_layer)), "forward", allow_nonfinite)

    def loss(self, allow_nonfinite: bool = True) -> float:
        out = ctypes.c_double()
        self._ck(self.lib.dmpm_loss(self.h, ctypes.byref(out)), "loss", allow_nonfinite)
        return float(out.value)

    def backward(self, control_layer: int = 0, allow_nonfinite: bool = True) -> int:
        return self._ck(self.lib.dmpm_backward(self.h, int(control_layer)), "backward", allow_nonfinite)

    # -------------------------------------------------------------- reads / writes
    def get(self, layer: int, field: str) -> np.ndarray:
        w = WIDTH[field]
        out = np.empty(self.n * w, dtype=np.float64)
        self._ck(self.lib.dmpm_get_particles(self.h, int(layer), FIELDS[field], out.ctypes.data), "get " + field)
        if w == 9:
            return _from_cm(out)
        if w == 3:
            return out.reshape(-1, 3)
        return out

    def set_layer(self, layer: int, field: str, value):
        a = _cm(value) if WIDTH[field] == 9 else np.ascontiguousarray(value, dtype=np.float64)
        self._ck(self.lib.dmpm_set_layer_particles(self.h, int(layer), FIELDS[field], a.ctypes.data), "set " + field)

    def get_grid(self, layer: int, field: str) -> np.ndarray:
        G = int(np.prod(self.dims))
        w = GRID_WIDTH[field]
        out = np.empty(G * w, dtype=np.float64)
        self._ck(self.lib.dmpm_get_grid(self.h, int(layer), GRID_FIELDS[field], out.ctypes.data), "grid " + field)
        return out.reshape(-1, 3) if w == 3 else out

    def control_grad(self, layer: int = 0, out=None) -> np.ndarray:
        """dL/d dFc as (N, 3, 3); `out` may be a (pinned) buffer of N*9 doubles (returned column-major)."""
        if out is not None:
            self._ck(self.lib.dmpm_get_control_grad(self.h, int(layer), _ptr(out)), "control_grad")
            return out
        a = np.empty(self.n * 9, dtype=np.float64)
        self._ck(self.lib.dmpm_get_control_grad(self.h, int(layer), a.ctypes.data), "control_grad")
        return _from_cm(a)

    def adam_step(self, t: int, lr: float = 1e-2, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-5,
                  layer: int = 0, normalize: bool = True):
        """Descend_Adam on the controls (device); t is the 1-based step count."""
        self._ck(self.lib.dmpm_adam_step(self.h, int(layer), lr, beta1, beta2, eps, int(t), int(normalize)),
                 "adam_step")

    def descend(self, rule: str, lr: float, t: int = 1, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-5,
                layer: int = 0, normalize: bool = True):
        """One of PointCloud's descent rules on the controls (device): "adam",
        "amsgrad", "lion" (beta1 = its beta), "gd" or "dldf" (Descend_dLdF)."""
        r = DESCEND[rule]
        self._ck(self.lib.dmpm_descend(self.h, int(layer), r, lr, beta1, beta2, eps, int(t), int(normalize)),
                 "descend " + rule)

    def dldf_norm(self, layer: int = 0) -> float:
        out = ctypes.c_double()
        self._ck(self.lib.dmpm_dldf_norm(self.h, int(layer), ctypes.byref(out)), "dldf_norm")
        return float(out.value)

    def cell_sort(self, layer: int):
        """(sorted cell keys, stable order, item starts) of the FP32 path's cell sort on a layer."""
        keys = np.empty(self.n, dtype=np.uint32)
        order = np.empty(self.n, dtype=np.uint32)
        items = np.empty(self.n + 1, dtype=np.uint32)
        ni = ctypes.c_int()
        self._ck(self.lib.dmpm_cell_sort(self.h, int(layer), keys.ctypes.data, order.ctypes.data, items.ctypes.data,
                                         ctypes.byref(ni)), "cell_sort")
        return keys, order, items[: ni.value + 1].copy()

    def get_points_ref(self, layer: int, points: np.ndarray) -> np.ndarray:
        assert points.dtype == np.float32 and points.shape == (self.n, 118) and points.flags.c_contiguous
        self._ck(self.lib.dmpm_get_points_ref(self.h, int(layer), points.ctypes.data), "get_points_ref")
        return points


class Batch:
    """Many independent scenes advanced together (dmpm_batch_*): FP32-mixed,
    every layer kept, tied controls, one launch per stage per time step,
    optionally replayed as a CUDA graph."""

    def __init__(self, specs: Sequence[dict], device: int = 0):
        """specs: per instance {"n", "dims", "dx", "min_point", "steps"}."""
        self.lib = load_library()
        arr = (Instance * len(specs))()
        for i, sp in enumerate(specs):
            arr[i].n = int(sp["n"])
            arr[i].dim_x, arr[i].dim_y, arr[i].dim_z = (int(d) for d in sp["dims"])
            arr[i].dx = float(sp.get("dx", 1.0))
            for c in range(3):
                arr[i].min_point[c] = float(sp.get("min_point", (0.0, 0.0, 0.0))[c])
            arr[i].steps = int(sp["steps"])
        h = _P()
        st = self.lib.dmpm_batch_create(device, len(specs), ctypes.cast(arr, _P), ctypes.byref(h))
        if st != OK:
            raise DmpmError(st, "dmpm_batch_create failed (no CUDA device, or invalid instances)")
        self.h = h
        self.specs = [dict(sp) for sp in specs]
        self.count = len(specs)

    def _ck(self, st: int, what: str, allow_nonfinite: bool = False) -> int:
        if st == OK or (allow_nonfinite and st == ERR_NONFINITE):
            return st
        msg = self.lib.dmpm_batch_last_error(self.h)
        raise DmpmError(st, "%s: %s" % (what, msg.decode() if msg else ""))

    def close(self):
        if getattr(self, "h", None):
            self.lib.dmpm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_params(self, dt: float, drag: float = 0.0, f_ext=(0.0, 0.0, 0.0), smoothing: float = 0.0,
                   adjoint: str = "exact", loss: str = "ref"):
        p = Params()
        self.lib.dmpm_default_params(ctypes.byref(p))
        p.dt, p.drag, p.smoothing = float(dt), float(drag), float(smoothing)
        for i in range(3):
            p.f_ext[i] = float(f_ext[i])
        p.adjoint_mode = ADJ_EXACT if adjoint == "exact" else ADJ_REFCOMPAT
        p.control_mode = CTRL_TIED
        p.loss_kind = LOSS_L2 if loss == "l2" else LOSS_REF_LOGMASS
        self._ck(self.lib.dmpm_batch_set_params(self.h, ctypes.byref(p)), "batch_set_params")

    def set_particles(self, inst: int, x, m, lam, mu, v=None, F=None, C=None, dFc=None, vol=None):
        a = [np.ascontiguousarray(x, dtype=np.float64), None if v is None else np.ascontiguousarray(v, dtype=np.float64),
             None if F is None else _cm(F), None if C is None else _cm(C), None if dFc is None else _cm(dFc),
             np.ascontiguousarray(m, dtype=np.float64), None if vol is None else np.ascontiguousarray(vol, dtype=np.float64),
             np.ascontiguousarray(lam, dtype=np.float64), np.ascontiguousarray(mu, dtype=np.float64)]
        self._ck(self.lib.dmpm_batch_set_particles(self.h, int(inst), *[_ptr(t) for t in a]), "batch_set_particles")

    def set_target_mass(self, inst: int, target):
        t = np.ascontiguousarray(target, dtype=np.float64)
        self._ck(self.lib.dmpm_batch_set_target_mass(self.h, int(inst), t.ctypes.data), "batch_set_target_mass")

    def set_launch(self, sort_every: int = 0, ctas_per_sm: int = 0, particle_block: int = 0, use_graph: bool = True):
        c = BatchLaunch(int(sort_every), int(ctas_per_sm), int(particle_block), int(bool(use_graph)))
        self._ck(self.lib.dmpm_batch_set_launch(self.h, ctypes.byref(c)), "batch_set_launch")

    def launch(self) -> dict:
        c = BatchLaunch()
        self._ck(self.lib.dmpm_batch_get_launch(self.h, ctypes.byref(c)), "batch_get_launch")
        return {"sort_every": c.sort_every, "ctas_per_sm": c.ctas_per_sm, "particle_block": c.particle_block,
                "use_graph": bool(c.use_graph)}

    def setup(self):
        self._ck(self.lib.dmpm_batch_setup(self.h), "batch_setup")

    def gradient(self, allow_nonfinite: bool = False) -> np.ndarray:
        out = np.empty(self.count, dtype=np.float64)
        self._ck(self.lib.dmpm_batch_gradient(self.h, out.ctypes.data), "batch_gradient", allow_nonfinite)
        return out

    def autotune(self, reps: int = 2) -> float:
        ms = ctypes.c_double()
        self._ck(self.lib.dmpm_batch_autotune(self.h, int(reps), ctypes.byref(ms)), "batch_autotune")
        return float(ms.value)

    def control_grad(self, inst: int) -> np.ndarray:
        a = np.empty(int(self.specs[inst]["n"]) * 9, dtype=np.float64)
        self._ck(self.lib.dmpm_batch_get_control_grad(self.h, int(inst), a.ctypes.data), "batch_control_grad")
        return _from_cm(a)

    def get(self, inst: int, layer: int, field: str) -> np.ndarray:
        w = WIDTH[field]
        out = np.empty(int(self.specs[inst]["n"]) * w, dtype=np.float64)
        self._ck(self.lib.dmpm_batch_get_particles(self.h, int(inst), int(layer), FIELDS[field], out.ctypes.data),
                 "batch_get " + field)
        return _from_cm(out) if w == 9 else out.reshape(-1, 3)

    def info(self) -> dict:
        a = (ctypes.c_int64 * 6)()
        self._ck(self.lib.dmpm_batch_info(self.h, a, 6), "batch_info")
        return {"instances": a[0], "particles": a[1], "nodes": a[2], "device_bytes": a[3],
                "launches_per_gradient": a[4], "graph": bool(a[5])}

    @property
    def stream(self) -> int:
        s = _P()
        self._ck(self.lib.dmpm_batch_stream(self.h, ctypes.byref(s)), "batch_stream")
        return s.value or 0


def mesh_lattice_points(V, F, point_dx: float, min_point=None, max_point=None) -> np.ndarray:
    """Point cloud of a watertight, outward-oriented triangle mesh on the GPU
    (dmpm_mesh_lattice_points): the lattice points of spacing point_dx over
    [min_point, max_point] (default: the vertices' float32 bounding box, as
    LoadMPMPointCloudFromObj takes it) whose winding number is >= 1/2, in the
    reference's lattice order.  V: (nv, 3), F: (nf, 3) 0-based; returns
    (n, 3) float32."""
    lib = load_library()
    V = np.ascontiguousarray(V, dtype=np.float32)
    F = np.ascontiguousarray(F, dtype=np.int32)
    mn = np.ascontiguousarray(V.min(axis=0) if min_point is None else min_point, dtype=np.float32)
    mx = np.ascontiguousarray(V.max(axis=0) if max_point is None else max_point, dtype=np.float32)
    dims = np.zeros(3, dtype=np.int32)
    st = lib.dmpm_mesh_lattice_dims(mn.ctypes.data, mx.ctypes.data, float(point_dx), dims.ctypes.data)
    if st != OK:
        raise DmpmError(st, "mesh_lattice_dims: invalid bounds or spacing")
    cap = int(np.prod(dims.astype(np.int64)))
    out = np.empty((cap, 3), dtype=np.float32)
    n = ctypes.c_int64()
    st = lib.dmpm_mesh_lattice_points(V.ctypes.data, len(V), F.ctypes.data, len(F), mn.ctypes.data, mx.ctypes.data,
                                      float(point_dx), out.ctypes.data, cap, ctypes.byref(n))
    if st != OK:
        raise DmpmError(st, "mesh_lattice_points failed")
    return out[: n.value].copy()


def mesh_jittered_points(V, F, cell_dx: float, per_axis: int, seed: int, min_point=None, max_point=None) -> np.ndarray:
    """Jittered stratified points inside a watertight mesh on the GPU
    (dmpm_mesh_jittered_points): one point per sub-cell of spacing
    cell_dx / per_axis, kept where the winding number is >= 1/2."""
    lib = load_library()
    lib.dmpm_mesh_jittered_points.argtypes = [_P, ctypes.c_int, _P, ctypes.c_int, _P, _P, ctypes.c_float, ctypes.c_int,
                                              ctypes.c_uint64, _P, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
    Vf = np.ascontiguousarray(V, dtype=np.float32)
    Fi = np.ascontiguousarray(F, dtype=np.int32)
    mn = np.ascontiguousarray(Vf.min(axis=0) if min_point is None else min_point, dtype=np.float32)
    mx = np.ascontiguousarray(Vf.max(axis=0) if max_point is None else max_point, dtype=np.float32)
    n = ctypes.c_int64()
    args = (Vf.ctypes.data, len(Vf), Fi.ctypes.data, len(Fi), mn.ctypes.data, mx.ctypes.data, float(cell_dx),
            int(per_axis), int(seed) & 0xFFFFFFFFFFFFFFFF)
    st = lib.dmpm_mesh_jittered_points(*args, None, 0, ctypes.byref(n))
    if st not in (OK, ERR_TOO_LARGE):
        raise DmpmError(st, "mesh_jittered_points")
    out = np.empty((n.value, 3), dtype=np.float32)
    st = lib.dmpm_mesh_jittered_points(*args, out.ctypes.data, n.value, ctypes.byref(n))
    if st != OK:
        raise DmpmError(st, "mesh_jittered_points")
    return out


def read_obj(path: str):
    """Vertices (float32) and triangles (0-based) of the 'v' and 'f' lines of an
    OBJ file; 'f' entries may be v, v/vt, v//vn or v/vt/vn, negative indices
    count from the end, polygons are split into a fan of triangles."""
    V, F = [], []
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            if t[0] == "v":
                V.append([float(x) for x in t[1:4]])
            elif t[0] == "f":
                idx = [int(x.split("/")[0]) for x in t[1:]]
                idx = [i - 1 if i > 0 else len(V) + i for i in idx]
                for k in range(1, len(idx) - 1):
                    F.append([idx[0], idx[k], idx[k + 1]])
    return np.asarray(V, dtype=np.float32), np.asarray(F, dtype=np.int32)


def point_cloud_from_obj(path: str, point_dx: float, density: float, lam: float, mu: float) -> dict:
    """LoadMPMPointCloudFromObj (MPMPolyscope.cpp:10-60): the mesh's lattice
    points (mesh_lattice_points over the vertices' bounding box), v = 0, F = I,
    m = point_dx^3 density, the given lam and mu.  Returns the arrays
    Context.set_particles takes."""
    V, F = read_obj(path)
    x = mesh_lattice_points(V, F, point_dx).astype(np.float64)
    n = len(x)
    pdx = np.float32(point_dx)
    m = float(np.float32(pdx * pdx * pdx * np.float32(density)))
    return {"x": x, "v": np.zeros((n, 3)), "F": np.broadcast_to(np.eye(3), (n, 3, 3)).copy(),
            "m": np.full(n, m), "lam": np.full(n, float(np.float32(lam))), "mu": np.full(n, float(np.float32(mu)))}


# ---------------------------------------------------------------- surfaces
def _surf_lib():
    lib = load_library()
    I64 = ctypes.c_int64
    lib.dmpm_surface_grid_dims.argtypes = [_P, _P, ctypes.c_float, _P]
    lib.dmpm_surface_p2g_mass.argtypes = [_P, I64, ctypes.c_float, _P, ctypes.c_float, _P, _P]
    lib.dmpm_surface_g2g_mass.argtypes = [_P, _P, ctypes.c_float, _P, _P, ctypes.c_float, _P, _P]
    lib.dmpm_surface_sphere_field.argtypes = [_P, I64, ctypes.c_float, ctypes.c_int, _P, ctypes.c_float, _P, _P]
    lib.dmpm_surface_extract.argtypes = [_P, _P, ctypes.c_float, _P, ctypes.c_float, _P, I64, _P, I64,
                                         ctypes.POINTER(I64), ctypes.POINTER(I64)]
    return lib


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a if shape is None else a.reshape(shape)


def _dims(d):
    return np.ascontiguousarray([int(v) for v in d], dtype=np.int32)


def _surf_ck(st, what):
    if st != OK:
        raise DmpmError(st, what)


def surface_grid_dims(min_point, max_point, dx: float):
    """ceil((max_x - min_x) / dx) nodes per axis (dmpm_surface_grid_dims)."""
    lib = _surf_lib()
    mn, mx = _f32(min_point), _f32(max_point)  # held here for the duration of the call
    d = np.zeros(3, dtype=np.int32)
    _surf_ck(lib.dmpm_surface_grid_dims(mn.ctypes.data, mx.ctypes.data, float(dx), d.ctypes.data), "surface_grid_dims")
    return tuple(int(v) for v in d)


def p2g_mass(points, mp_m: float, dims, dx: float, min_point) -> np.ndarray:
    """SingleThreadMPM::P2G_Mass on the GPU: node masses, flat in node order."""
    lib = _surf_lib()
    p, d, mn = _f32(points, (-1, 3)), _dims(dims), _f32(min_point)
    out = np.empty(int(np.prod(dims)), dtype=np.float32)
    _surf_ck(lib.dmpm_surface_p2g_mass(p.ctypes.data, len(p), float(mp_m), d.ctypes.data, float(dx), mn.ctypes.data,
                                       out.ctypes.data), "p2g_mass")
    return out


def g2g_mass(mass1, dims1, dx1: float, min1, dims2, dx2: float, min2) -> np.ndarray:
    """SingleThreadMPM::G2G_Mass on the GPU."""
    lib = _surf_lib()
    m1, d1, mn1, d2, mn2 = _f32(mass1), _dims(dims1), _f32(min1), _dims(dims2), _f32(min2)
    out = np.empty(int(np.prod(dims2)), dtype=np.float32)
    _surf_ck(lib.dmpm_surface_g2g_mass(m1.ctypes.data, d1.ctypes.data, float(dx1), mn1.ctypes.data, d2.ctypes.data,
                                       float(dx2), mn2.ctypes.data, out.ctypes.data), "g2g_mass")
    return out


def sphere_field(points, radius: float, blur_iterations: int, dims, dx: float, min_point) -> np.ndarray:
    """The sphere-union field of SphereUnionMarchingCubesSurfaceFromPointCloud on the GPU."""
    lib = _surf_lib()
    p, d, mn = _f32(points, (-1, 3)), _dims(dims), _f32(min_point)
    out = np.empty(int(np.prod(dims)), dtype=np.float32)
    _surf_ck(lib.dmpm_surface_sphere_field(p.ctypes.data, len(p), float(radius), int(blur_iterations), d.ctypes.data,
                                           float(dx), mn.ctypes.data, out.ctypes.data), "sphere_field")
    return out


def extract_surface(field, dims, dx: float, min_point, iso: float):
    """Triangle mesh (V float32 (n, 3), F int32 (m, 3)) of {field = iso} (dmpm_surface_extract)."""
    lib = _surf_lib()
    f = _f32(field)
    d, mn = _dims(dims), _f32(min_point)
    nv, nf = ctypes.c_int64(), ctypes.c_int64()
    st = lib.dmpm_surface_extract(f.ctypes.data, d.ctypes.data, float(dx), mn.ctypes.data, float(iso), None, 0, None,
                                  0, ctypes.byref(nv), ctypes.byref(nf))
    if st not in (OK, ERR_TOO_LARGE):
        raise DmpmError(st, "extract_surface")
    V = np.empty((nv.value, 3), dtype=np.float32)
    F = np.empty((nf.value, 3), dtype=np.int32)
    _surf_ck(lib.dmpm_surface_extract(f.ctypes.data, d.ctypes.data, float(dx), mn.ctypes.data, float(iso),
                                      V.ctypes.data, nv.value, F.ctypes.data, nf.value, ctypes.byref(nv),
                                      ctypes.byref(nf)), "extract_surface")
    return V, F


def marching_cubes_point_cloud(points, iso_mass: float, grid_dx: float, quality: float, min_point, max_point):
    """The reference GUI's MarchingCubesPointCloud (DiffMPMAnimator3D.cpp:488-514) on
    the GPU: P2G_Mass (unit point mass) on the grid of spacing grid_dx, G2G_Mass onto
    a grid refined by `quality`, and the iso_mass level set of the fine masses."""
    dims = surface_grid_dims(min_point, max_point, grid_dx)
    coarse = p2g_mass(points, 1.0, dims, grid_dx, min_point)
    q = np.float32(quality)
    fdims = tuple(int(np.float32(d) * q) for d in dims)
    fdx = float(np.float32(grid_dx) / q)
    fine = g2g_mass(coarse, dims, grid_dx, min_point, fdims, fdx, min_point)
    return extract_surface(fine, fdims, fdx, min_point, iso_mass)


def sphere_union_surface(points, radius: float, grid_dx: float, iso_mass: float, blur_iterations: int, min_point,
                         max_point):
    """SphereUnionMarchingCubesSurfaceFromPointCloud (SphereUnionSurfacing.cpp:7-128)
    on the GPU (grid_dx is the spacing of the field's grid, as there)."""
    dims = surface_grid_dims(min_point, max_point, grid_dx)
    f = sphere_field(points, radius, blur_iterations, dims, grid_dx, min_point)
    return extract_surface(f, dims, grid_dx, min_point, iso_mass)


def write_obj(path: str, V, F) -> None:
    """A mesh as Wavefront OBJ (1-based faces)."""
    with open(path, "w") as f:
        for v in np.asarray(V):
            f.write("v %.9g %.9g %.9g\n" % tuple(v))
        for t in np.asarray(F):
            f.write("f %d %d %d\n" % (t[0] + 1, t[1] + 1, t[2] + 1))
