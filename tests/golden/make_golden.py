"""Generate golden vectors from the reference's own CPU code.

Runs the reference library (DiffMPMLib3D sources compiled by
oracle/build_ref.sh into oracle/_ref/, FP32 as shipped and the FP64 retyped
build) on seeded synthetic inputs and stores the results as small .npz files
next to this script.  Needs the reference sources (run where they exist):

    bash oracle/build_ref.sh && python tests/golden/make_golden.py

Fixtures:
  elementary_{f32,f64}.npz  polar factors, PK stress, dP/dF:dF (reference
                            finite-difference variant), d(J F^-T)/dF by the
                            reference's d_JFit_dF_FD, B-spline values, on the
                            CheckGradients fixture F = 0.8 Rx(45 deg),
                            lam = 58333, mu = 38888.9 (DiffMPMAnimator3D.cpp:212-243)
                            and on seeded random F.
  rollout_{f32,f64}.npz     a seeded sphere scene: volumes
                            (CalculatePointCloudVolumes), target raster,
                            per-layer particle state and grids after
                            ComputeForwardPass, EndLayerMassLoss, and every
                            layer's adjoint after ComputeBackwardPass(0).
  rollout_long_f64.npz      a second seeded sphere (459 particles, 12^3 grid)
                            rolled out for 1, 10, 30 and 100 steps by the FP64
                            build: the last layer's x, v, F, the loss and the
                            layer-0 adjoint (dLdx, dLdv, dLdF, dLdC) of each.  The
                            reference's adjoint grows about twofold per step, to
                            ~1e21 at 100 steps.
  rollout_long_f32.npz      the same rollouts by the shipped FP32 build (same
                            volumes and target), the float reference's own drift
                            from the FP64 build.
  config0_f64.npz           the small benchmark configuration at full size (a
                            jittered sphere of 8,778 particles on 32^3, 100 steps
                            at half the explicit CFL limit) by the FP64 build with
                            its own adjoint: volumes, target raster, the final
                            positions, the loss and the layer-0 dLdF and dLdx.

    python tests/golden/make_golden.py [elementary rollout long mpmbin config0]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "a-differentiable-material-point-method-for-shape-morphing_b200"))

import scenes  # noqa: E402
from oracle.lib import Elementary, RefGraph  # noqa: E402

ROLLOUT_LAYERS = 6


def rollout_scene():
    return scenes.small_scene(seed=1, res=16, steps=ROLLOUT_LAYERS - 1, v_std=0.5, drag=0.3, smoothing=0.1,
                              f_ext=(0.0, -2.0, 0.5), dt=2e-4)


def elementary_inputs():
    th = np.pi / 4
    Rx = np.array([[1, 0, 0], [0, np.cos(th), -np.sin(th)], [0, np.sin(th), np.cos(th)]])
    Fs = [0.8 * Rx]
    rng = np.random.default_rng(42)
    for t in range(24):
        k = t % 4
        if k == 0:
            F = np.eye(3) + 1e-3 * rng.normal(size=(3, 3))
        elif k == 1:
            F = np.eye(3) + 0.2 * rng.normal(size=(3, 3))
        elif k == 2:
            Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
            Q *= np.sign(np.linalg.det(Q))
            F = Q @ np.diag(rng.uniform(0.6, 1.4, 3)) @ Q.T
        else:
            F = np.eye(3) + 0.3 * rng.normal(size=(3, 3))
            F[:, 0] *= -1.0  # inverted
        Fs.append(F)
    dFs = [rng.normal(size=(3, 3)) for _ in Fs]
    return np.array(Fs), np.array(dFs)


def make_elementary(prec):
    e = Elementary("ref", prec)
    Fs, dFs = elementary_inputs()
    lam, mu = 58333.0, 38888.9
    R, S, P, D2, DJ = [], [], [], [], []
    for F, dF in zip(Fs, dFs):
        r, s = e.polar(F)
        R.append(r)
        S.append(s)
        P.append(e.pk(F, lam, mu))
        D2.append(e.d2(F, lam, mu, dF))
        DJ.append(e.djfit_fd(F))
    xs = np.linspace(-2.5, 2.5, 101)
    np.savez_compressed(os.path.join(HERE, "elementary_%s.npz" % prec), F=Fs, dF=dFs, lam=lam, mu=mu,
                        R=np.array(R), S=np.array(S), P=np.array(P), d2=np.array(D2), djfit=np.array(DJ), bx=xs,
                        b=np.array([e.bspline(x) for x in xs]), bs=np.array([e.bspline_slope(x) for x in xs]))


def make_rollout(prec):
    sc = rollout_scene()
    r = RefGraph(sc, prec)
    vol = r.calc_volumes()
    target = r.target_mass()
    sc.vol = vol.astype(np.float64)
    r = RefGraph(sc, prec)
    r.setup(ROLLOUT_LAYERS, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
    r.forward(0)
    out = {"vol": vol, "target": target}
    for lay in range(ROLLOUT_LAYERS):
        for k in ("x", "v", "F", "C"):
            out["%s_%d" % (k, lay)] = r.get(lay, k)
        if lay < ROLLOUT_LAYERS - 1:
            out["P_%d" % lay] = r.get(lay, "P")
            for k in ("grid_m", "grid_v", "grid_p"):
                out["%s_%d" % (k, lay)] = r.get(lay, k)
    out["loss"] = np.array(r.loss())
    L = ROLLOUT_LAYERS - 1
    out["grid_m_%d" % L] = r.get(L, "grid_m")
    out["grid_dLdm_%d" % L] = r.get(L, "grid_dLdm")
    r.backward(0)
    for lay in range(ROLLOUT_LAYERS):
        for k in ("dLdx", "dLdv", "dLdF", "dLdC"):
            out["%s_%d" % (k, lay)] = r.get(lay, k)
        if lay < ROLLOUT_LAYERS - 1:
            for k in ("dLdP", "dLdv_next", "dLdC_next"):
                out["%s_%d" % (k, lay)] = r.get(lay, k)
            for k in ("grid_dLdv", "grid_dLdp", "grid_dLdm"):
                out["%s_%d" % (k, lay)] = r.get(lay, k)
    np.savez_compressed(os.path.join(HERE, "rollout_%s.npz" % prec), **out)


LONG_STEPS = (1, 10, 30, 100)


def long_scene():
    return scenes.small_scene(seed=31, res=12, radius=0.2, steps=max(LONG_STEPS), v_std=0.3, drag=0.1,
                              smoothing=0.05, f_ext=(0.0, -1.0, 0.0))


def make_rollout_long():
    """Both builds on the same inputs: volumes and target from the FP64 build."""
    sc = long_scene()
    r = RefGraph(sc, "f64")
    vol = r.calc_volumes()
    target = r.target_mass()
    sc.vol = vol.astype(np.float64)
    for prec in ("f64", "f32"):
        out = {"vol": vol, "target": target} if prec == "f64" else {}
        for S in LONG_STEPS:
            r = RefGraph(sc, prec, target_m=target)
            r.setup(S + 1, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
            r.forward(0)
            out["loss_%d" % S] = np.array(r.loss())
            for k in ("x", "v", "F"):
                out["%s_%d" % (k, S)] = r.get(S, k)
            r.backward(0)
            for k in ("dLdx", "dLdv", "dLdF", "dLdC"):
                out["%s0_%d" % (k, S)] = r.get(0, k)
        np.savez_compressed(os.path.join(HERE, "rollout_long_%s.npz" % prec), **out)


def mpmbin_scene():
    return scenes.small_scene(seed=77, res=8, radius=0.25, v_std=0.3)


def make_mpmbin():
    """cloud_ref.mpmbin: the reference's own PointCloud::WriteEntirePointCloudToBinaryFile
    (PointCloud.cpp:334-346) of a small seeded cloud, to pin the .mpmbin format."""
    import ctypes

    sc = mpmbin_scene()
    r = RefGraph(sc, "f32")
    r.lib.ref_scene_write_mpmbin.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    r.lib.ref_scene_write_mpmbin(r.h, os.path.join(HERE, "cloud_ref.mpmbin").encode())


def config0_scene():
    """The small benchmark scene (sphere r = 0.2 on 32^3, 8 per cell, 100 steps),
    its configured dt replaced by half the explicit CFL limit when above it."""
    sc = scenes.config_scene(0)
    lim = sc.cfl_dt()
    if sc.dt > lim:
        sc.dt = 0.5 * lim
    return sc


def make_config0():
    sc = config0_scene()
    r = RefGraph(sc, "f64")
    vol = r.calc_volumes()
    target = r.target_mass()
    sc.vol = vol.astype(np.float64)
    L = sc.steps + 1
    r = RefGraph(sc, "f64", target_m=target)
    r.setup(L, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
    r.forward(0)
    loss = r.loss()
    r.backward(0)
    np.savez_compressed(os.path.join(HERE, "config0_f64.npz"), vol=vol, target=target, dt=np.array(sc.dt),
                        x_last=r.get(L - 1, "x"), loss=np.array(loss), dLdF_0=r.get(0, "dLdF"),
                        dLdx_0=r.get(0, "dLdx"))


if __name__ == "__main__":
    parts = sys.argv[1:] or ["elementary", "rollout", "long", "mpmbin", "config0"]
    for prec in ("f64", "f32"):
        if "elementary" in parts:
            make_elementary(prec)
        if "rollout" in parts:
            make_rollout(prec)
    if "long" in parts:
        make_rollout_long()
    if "mpmbin" in parts:
        make_mpmbin()
    if "config0" in parts:
        make_config0()
    print("wrote", " ".join(parts))
