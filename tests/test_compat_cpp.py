"""The DiffMPMLib3D-compatible C++ API (compat/, libdmpm_compat.so) used from a
C++ program the way the reference's callers use the reference
(tests/cpp/compgraph_check.cpp: scene load with CalculatePointCloudVolumes and
a P2G target raster, CompGraph SetUpCompGraph / ComputeForwardPass /
EndLayerMassLoss / ComputeBackwardPass, standalone ForwardTimeStep and
Back_Timestep, the CheckGradients fixture), compared with the reference's golden
vectors.  The C++ API stores float (the reference's MaterialPoint), so inputs
are float32-rounded and tolerances sit at the float level."""
import os
import subprocess

import numpy as np
import pytest

import dmpm
from tests.golden.make_golden import ROLLOUT_LAYERS, rollout_scene
from tests.helpers import load_golden, normrel, relerr, write_mpmbin

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "a-differentiable-material-point-method-for-shape-morphing_b200")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    import build as pkg_build

    pkg_build.build_compat()
    out = tmp_path_factory.mktemp("cpp") / "compgraph_check"
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(PKG, "compat"), "-I",
                           os.path.join(REPO, "include"), os.path.join(REPO, "tests", "cpp", "compgraph_check.cpp"),
                           "-L", PKG, "-ldmpm_compat", "-ldmpm", "-Wl,-rpath," + PKG, "-o", str(out)])
    return str(out)


def run(exe, tmp_path, precision, deterministic=False, tag="", reorder=False):
    sc = rollout_scene()
    z33 = np.zeros((sc.n, 3, 3))
    write_mpmbin(tmp_path / "cloud.mpmbin", sc.x, sc.v, sc.F, sc.C, z33, sc.m, np.zeros(sc.n), sc.lam, sc.mu, sc.dFc)
    nt = len(sc.target_points)
    zt = np.zeros((nt, 3))
    eye = np.broadcast_to(np.eye(3), (nt, 3, 3))
    write_mpmbin(tmp_path / "target.mpmbin", sc.target_points, zt, eye, np.zeros((nt, 3, 3)), np.zeros((nt, 3, 3)),
                 np.full(nt, sc.target_mp), np.zeros(nt), np.zeros(nt), np.zeros(nt), np.zeros((nt, 3, 3)))
    out = tmp_path / ("out%d%s.bin" % (precision, tag))
    args = [exe, str(tmp_path / "cloud.mpmbin"), str(tmp_path / "target.mpmbin"), str(out), str(precision),
            str(sc.dims[0]), str(ROLLOUT_LAYERS), repr(sc.dt), repr(sc.drag), repr(sc.smoothing),
            *[repr(float(v)) for v in sc.f_ext]] + (["1" if deterministic else "0", "1" if reorder else "0"])
    res = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    a = np.fromfile(out, dtype=np.float64)
    n = int(a[0])
    o = 2
    take = lambda k: (a[o:o + k], o + k)
    r = {"n": n, "loss": a[1]}
    r["vol"], o = take(n)
    r["x_last"], o = take(3 * n)
    r["dLdF0"], o = take(9 * n)
    r["dLdx0"], o = take(3 * n)
    r["x1_standalone"], o = take(3 * n)
    r["dLdF0_back_timestep"], o = take(9 * n)
    r["P0"], o = take(9 * n)
    r["check_gradients_rel"] = a[o]
    r["dldf_norm"] = a[o + 1]
    return r, sc


def cm(a):  # (n*9,) column-major -> (n,3,3)
    return a.reshape(-1, 3, 3).transpose(0, 2, 1)


def test_compgraph_cpp_fp64_matches_reference(gpu_ready, exe, tmp_path):
    g = load_golden("rollout_f64")
    r, sc = run(exe, tmp_path, dmpm.FP64)
    assert r["n"] == sc.n
    assert relerr(r["vol"], g["vol"]) < 1e-5
    assert abs(r["loss"] - float(g["loss"])) / abs(float(g["loss"])) < 1e-5
    assert relerr(r["x_last"].reshape(-1, 3), g["x_%d" % (ROLLOUT_LAYERS - 1)]) < 1e-6
    assert relerr(r["x1_standalone"].reshape(-1, 3), g["x_1"]) < 1e-6
    assert relerr(cm(r["P0"]), g["P_0"]) < 1e-3
    assert normrel(cm(r["dLdF0"]), g["dLdF_0"]) < 1e-3
    assert normrel(r["dLdx0"].reshape(-1, 3), g["dLdx_0"]) < 1e-3
    # Back_Timestep on layers 1 -> 0 reproduces the graph's layer-0 adjoint
    assert normrel(cm(r["dLdF0_back_timestep"]), cm(r["dLdF0"])) < 1e-5
    assert abs(r["dldf_norm"] - np.linalg.norm(g["dLdF_0"])) / np.linalg.norm(g["dLdF_0"]) < 1e-3
    # CheckGradients: FD tensor vs the multiplication trick (FD in float is noisy)
    assert r["check_gradients_rel"] < 0.05


def test_compgraph_cpp_fp32_mixed_close_to_reference(gpu_ready, exe, tmp_path):
    g = load_golden("rollout_f64")
    r, sc = run(exe, tmp_path, dmpm.FP32_MIXED)
    assert relerr(r["vol"], g["vol"]) < 1e-5
    assert abs(r["loss"] - float(g["loss"])) / abs(float(g["loss"])) < 1e-4
    assert relerr(r["x_last"].reshape(-1, 3), g["x_%d" % (ROLLOUT_LAYERS - 1)]) < 1e-5
    assert normrel(cm(r["dLdF0"]), g["dLdF_0"]) < 1e-2


def test_compgraph_cpp_deterministic_repeats_bit_for_bit(gpu_ready, exe, tmp_path):
    """SingleThreadMPM::SetEngineDeterministic and CompGraph::SetDeterministic:
    the FP32-mixed path with integer node sums, in two processes on the same
    inputs -- volumes, loss, states and adjoints the same bits, and at the FP32
    path's distance from the reference."""
    g = load_golden("rollout_f64")
    a, sc = run(exe, tmp_path, dmpm.FP32_MIXED, deterministic=True, tag="a")
    b, _ = run(exe, tmp_path, dmpm.FP32_MIXED, deterministic=True, tag="b")
    for k in ("vol", "x_last", "dLdF0", "dLdx0", "x1_standalone", "dLdF0_back_timestep", "P0"):
        assert np.array_equal(a[k], b[k]), k
    assert a["loss"] == b["loss"]
    assert relerr(a["vol"], g["vol"]) < 1e-5
    assert abs(a["loss"] - float(g["loss"])) / abs(float(g["loss"])) < 1e-4
    assert relerr(a["x_last"].reshape(-1, 3), g["x_%d" % (ROLLOUT_LAYERS - 1)]) < 1e-5
    assert normrel(cm(a["dLdF0"]), g["dLdF_0"]) < 1e-2


def test_compgraph_cpp_reorder_keeps_the_callers_order(gpu_ready, exe, tmp_path):
    """CompGraph::SetReorderParticles: the engine stores the cloud in cell
    order, and every layer's points, states and adjoints come back in the
    caller's order -- the same values as without reordering, to the FP32
    path's summation-order noise."""
    a, _ = run(exe, tmp_path, dmpm.FP32_MIXED, deterministic=True, tag="plain")
    b, _ = run(exe, tmp_path, dmpm.FP32_MIXED, deterministic=True, tag="reorder", reorder=True)
    assert np.array_equal(a["vol"], b["vol"])  # the stage functions' volumes: no reordering there
    assert abs(a["loss"] - b["loss"]) <= 1e-6 * abs(a["loss"])
    assert relerr(b["x_last"], a["x_last"]) < 1e-6
    assert normrel(b["dLdF0"], a["dLdF0"]) < 1e-4
    assert normrel(b["dLdx0"], a["dLdx0"]) < 1e-4


def test_stage_level_api_composes_the_fused_step(gpu_ready, tmp_path):
    """SingleThreadMPM::P_op_1, G_Reset, P2G, G_op, G2P, P_op_2 called one by one
    (tests/cpp/stages_check.cpp) give the step SingleThreadMPM::ForwardTimeStep
    gives; MultiThreadMPM::ForwardTimeStep is the step without smoothing; G_op's
    point-gravity form follows the reference's formula."""
    import build as pkg_build

    pkg_build.build_compat()
    exe = str(tmp_path / "stages_check")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(PKG, "compat"), "-I",
                           os.path.join(REPO, "include"), os.path.join(REPO, "tests", "cpp", "stages_check.cpp"),
                           "-L", PKG, "-ldmpm_compat", "-ldmpm", "-Wl,-rpath," + PKG, "-o", exe])
    res = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
