"""The C ABI library loads and exports every function include/dmpm.h declares
(no GPU calls)."""
import os
import re
import subprocess

import pytest

import dmpm

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(REPO, "include", "dmpm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dmpm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = dmpm.load_library()
    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", dmpm.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (dmpm_\w+)", out))
    assert set(names) <= exported, sorted(set(names) - exported)


def test_params_struct_matches_header():
    p = dmpm.Params()
    dmpm.load_library().dmpm_default_params(p)
    assert p.adjoint_mode == dmpm.ADJ_REFCOMPAT and p.control_mode == dmpm.CTRL_PER_LAYER
    assert abs(p.dt - 1.0 / 120.0) < 1e-15 and p.drag == 0.5 and abs(p.smoothing - 0.1) < 1e-15


def test_params_layout_matches_c(tmp_path):
    """Every field of the ctypes Params sits at the offset the C compiler gives dmpm_params."""
    fields = [f for f, _ in dmpm.Params._fields_]
    prog = tmp_path / "layout.c"
    prog.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "dmpm.h"\nint main(void) {\n'
                    '  printf("%zu\\n", sizeof(dmpm_params));\n'
                    + "".join('  printf("%%zu\\n", offsetof(dmpm_params, %s));\n' % f for f in fields)
                    + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(REPO, "include"), str(prog), "-o", str(exe)])
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    import ctypes
    assert vals[0] == ctypes.sizeof(dmpm.Params)
    assert vals[1:] == [getattr(dmpm.Params, f).offset for f in fields]


def test_null_arguments_are_rejected_without_gpu():
    lib = dmpm.load_library()
    assert lib.dmpm_create(0, 7, None) == dmpm.ERR_ARG
    assert lib.dmpm_destroy(None) == dmpm.ERR_ARG
    assert lib.dmpm_forward(None, 0) == dmpm.ERR_ARG


def test_host_only_size_helpers_without_gpu():
    """The grid-size helpers of the mesh sampler and of the surfacing functions are
    host arithmetic: the reference's ceil((max - min) / dx) (+ 1 for the sampler's
    lattice, GeometryLoading.cpp:21-23; the x extent on every axis for the surfacing
    grids, SphereUnionSurfacing.cpp:13-16), and bad arguments are rejected."""
    import ctypes

    import numpy as np

    lib = dmpm.load_library()
    mn = np.float32([-1.0, -0.5, 0.0])
    mx = np.float32([1.0, 0.5, 0.3])
    d = np.zeros(3, np.int32)
    lib.dmpm_mesh_lattice_dims.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p]
    assert lib.dmpm_mesh_lattice_dims(mn.ctypes.data, mx.ctypes.data, 0.1, d.ctypes.data) == dmpm.OK
    want = [int(np.ceil(np.float32(mx[a] - mn[a]) / np.float32(0.1))) + 1 for a in range(3)]
    assert list(d) == want
    assert lib.dmpm_mesh_lattice_dims(mn.ctypes.data, mx.ctypes.data, -1.0, d.ctypes.data) == dmpm.ERR_ARG
    assert dmpm.surface_grid_dims(mn, mx, 0.05) == (40, 40, 40)
    with pytest.raises(dmpm.DmpmError):
        dmpm.surface_grid_dims(mn, mx, 0.0)


def test_kernel_ids_names_and_bench_tables_agree():
    """dmpm_kernel_name (host only) names every id below DMPM_NUM_KERNEL_IDS and no
    other, the Python mirror has the same count, and every kernel bench.py's
    algorithmic-byte tables describe is one of those names."""
    import ctypes
    import sys

    src = open(os.path.join(REPO, "include", "dmpm.h")).read()
    n = int(re.search(r"#define DMPM_NUM_KERNEL_IDS (\d+)", src).group(1))
    assert n == dmpm.NUM_KERNEL_IDS
    lib = dmpm.load_library()
    lib.dmpm_kernel_name.restype = ctypes.c_char_p
    names = [lib.dmpm_kernel_name(k) for k in range(n)]
    assert all(names) and len(set(names)) == n
    assert lib.dmpm_kernel_name(n) is None and lib.dmpm_kernel_name(-1) is None
    names = {b.decode() for b in names}
    sys.path.insert(0, REPO)
    import bench

    described = set(bench.PER_PARTICLE_BYTES) | set(bench.PER_TOUCHED_NODE_BYTES) | set(bench.PER_GRID_NODE_BYTES)
    assert described <= names, sorted(described - names)
    assert {"adj_finalize", "adj_finalize_transport", "adj_p2g_gather"} <= described


def test_bench_roofline_tables():
    """bench.py's algorithmic bytes: the per-particle figures of one time step's
    kernels sum to 1604 B (what the roofline text quotes), and the compute object
    turns the ncu-counted flop per particle-step into rates and fractions."""
    import sys

    sys.path.insert(0, REPO)
    import bench

    step = ("p_op1", "p2g", "g2p_p_op2", "adj_g2p_scatter", "adj_p2g_gather", "adj_finalize", "adj_finalize_transport")
    assert sum(bench.PER_PARTICLE_BYTES[k] for k in step) == 1604
    assert bench.algorithmic_bytes("adj_p2g_gather", 10, 3, 7) == 10 * bench.PER_PARTICLE_BYTES["adj_p2g_gather"] + 3 * 32
    assert bench.algorithmic_bytes("g_op", 10, 3, 7) == 7 * 32
    r = bench.compute_rates(1e9)
    for p in ("fp32", "fp64"):
        f = bench.FLOP_PER_PARTICLE_STEP[p]
        assert abs(r[p]["tflops"] - f * 1e-3) < 1e-9
        assert abs(r[p]["frac"] - r[p]["tflops"] / r[p]["nominal_tflops"]) < 1e-12
