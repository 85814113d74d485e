#!/usr/bin/env python
"""Benchmark: forward + adjoint particle-steps/s of the MLS-MPM morphing path.

Workload (one "step" = one gradient evaluation): the ellipsoid-to-torus
scene -- solid ellipsoid with semi-axes (0.3, 0.2, 0.15) in the unit box,
jittered stratified sampling at 27 particles per cell (~267k particles),
64^3 grid, fixed-corotated E = 1e4, nu = 0.3, 200 time steps, target a solid
torus R = 0.25, r = 0.08 -- run as forward rollout + end-layer mass loss +
full adjoint (exact mode, tied controls, FP64 gradient accumulation), every
layer kept in HBM.  Seeded synthetic inputs stand in for the reference's
OBJ meshes (which are not part of its tree).

Our arm (default) prints one JSON line with
  value      device-resident throughput (particle-steps/s, whole job)
  e2e        the same through the C ABI with host buffers: pinned-host upload of
             every particle input, forward, loss, adjoint and the read-back of
             the control gradient inside the timed region
  roofline   the dominant kernel's algorithmic bytes / its CUDA-event duration
  compute    FP32 and FP64 flop rates: ncu-counted flop per particle-step x value
  fp64       the plain FP64 GPU path on the same workload, speedup and
             gradient relative error of the FP32-mixed path against it
  cpu_baseline the reference's own CPU code (oracle/_ref) on a bounded sample
`--impl reference` times the reference's CPU implementation alone.
Multi-GPU (torchrun): one independent instance per rank (seed = rank), no
data-path collective; timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "a-differentiable-material-point-method-for-shape-morphing_b200")
for _p in (REPO, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import scenes  # noqa: E402

METRIC = "fwd+adjoint particle-steps/s, FP32-mixed vs FP64 GPU @ grad relerr≤1e-4"
UNIT = "particle-steps/s"
HBM_FALLBACK_GBS = 6650.0


# ---------------------------------------------------------------- helpers
def measured_hbm_gbs():
    """HBM copy bandwidth of this pool's B200s: MEASURED_PEAKS.json's hbm_gbs, else
    the pool's earlier measurement (6.65 TB/s), with a label saying which."""
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback (MEASURED_PEAKS.json absent; earlier pool measurement)"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(ngpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(value: float, world: int) -> float:
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_instances(work, world: int, rank: int):
    """Instances of this rank: longest-processing-time-first assignment of the
    per-instance work (particles x steps) to the least-loaded rank; every
    instance goes to exactly one rank and no data crosses ranks."""
    load = [0.0] * world
    owner = {}
    for i in sorted(range(len(work)), key=lambda i: (-work[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        owner[i] = r
        load[r] += work[i]
    return [i for i in range(len(work)) if owner[i] == rank]


def whole_job_value(units_per_rank_step: float, steps: int, world: int, ms_max: float) -> float:
    """Units all ranks processed / the slowest rank's device time (weak scaling)."""
    return units_per_rank_step * steps * world / (ms_max / 1000.0)


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


FLT_EPSILON = 1.1920928955078125e-07  # the reference's node-mass threshold (ForwardSimulation.cpp:55)


# ---------------------------------------------------------------- workload
def build_scene(instance: int, ppc_root: int):
    sc = scenes.config_scene(1, instance=instance, ppc_root=ppc_root)
    if SHUFFLE:  # the same cloud handed over in a seeded random order
        perm = np.random.default_rng(2024 + instance).permutation(sc.n)
        for f in ("x", "v", "F", "C", "dFc", "m", "lam", "mu", "vol"):
            setattr(sc, f, np.ascontiguousarray(getattr(sc, f)[perm]))
    return sc


# G2P kernel of the FP32 path: None = the library default (bricks of 2^3 cells), 0 = warp
# items, 2 or 4 = bricks of that many cells per axis
BRICK_CELLS = None
# cell-sort interval of the FP32 path (None = the library default, 8 steps)
SORT_EVERY = None
# FP32 path with integer node sums (bit-identical repeats), for every FP32 context
DETERMINISTIC = False
# the caller's particle order: False = the scene's lattice order, True = a seeded random permutation
SHUFFLE = False
# FP32 path: the engine stores the cloud in cell order at setup (dmpm_params::reorder_particles)
REORDER = False


def setup_ctx(dmpm, sc, prec, device, vol, target, dt, checkpoint_every, control="tied", control_stride=0,
              same_inputs=True, deterministic=None):
    """An engine context over scene sc.  same_inputs: upload the scene's
    inputs rounded to float32 on both paths -- the FP32-mixed path rounds them
    so anyway, and the FP64 path then computes from the identical values, so a
    gradient comparison measures arithmetic, not the representation of the
    inputs."""
    if same_inputs:
        sc = sc.float32_inputs()
        vol = None if vol is None else np.asarray(vol, dtype=np.float32).astype(np.float64)
        target = np.asarray(target, dtype=np.float32).astype(np.float64)
    c = dmpm.Context(prec, device)
    c.set_grid(sc.dims, sc.dx, sc.min_point)
    c.set_particles(sc.x, sc.m, sc.lam, sc.mu, v=sc.v, F=sc.F, C=sc.C, dFc=sc.dFc, vol=vol)
    c.set_target_mass(target)
    c.set_params(dt=dt, drag=sc.drag, f_ext=sc.f_ext, smoothing=sc.smoothing, adjoint="exact", control=control,
                 loss="ref", checkpoint_every=checkpoint_every, control_stride=control_stride,
                 brick_cells=BRICK_CELLS if prec == "fp32" else None, sort_every=SORT_EVERY or 0,
                 deterministic=DETERMINISTIC if deterministic is None else deterministic,
                 reorder_particles=REORDER and prec == "fp32")
    c.setup(sc.steps + 1)
    return c


def gradient_step(c):
    c.forward(0)
    loss = c.loss()
    c.backward(0)
    return loss


def finite_gradient(dmpm, c) -> bool:
    st_f = c.forward(0)
    loss = c.loss()
    st_b = c.backward(0)
    ok = st_f == dmpm.OK and st_b == dmpm.OK and math.isfinite(loss)
    return ok and bool(np.all(np.isfinite(c.control_grad())))


def timed_steps(torch, c, steps, fn):
    """CUDA events on the context's stream around `steps` calls of fn."""
    s = torch.cuda.ExternalStream(c.stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(steps):
        fn()
    e1.record(s)
    e1.synchronize()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


# Algorithmic bytes per launch of each kernel of the FP32 path: every particle
# plane it must read or write once (4 B per FP32 value, the FP64 tied-control
# accumulator 8 B), the sorted-order index of the warp-item kernels (4 B per
# particle), and its grid records: per touched node for the particle-parallel
# kernels, per grid node for the node-parallel ones.
# (positions are compensated float pairs, hi + lo: 6 floats per particle)
PER_PARTICLE_BYTES = {
    "p_op1": (9 + 9 + 4 + 9) * 4 + 24 * 4,                  # F, dFc, m/vol/lam/mu, C -> G, R, S
    "p2g": (6 + 1 + 3 + 9 + 1) * 4,                         # x, m, v, G, order
    "g2p_p_op2": (6 + 9 + 9 + 1) * 4 + 27 * 4,              # x, F, dFc, order -> x, v, C, F
    "adj_g2p_scatter": (6 + 24 + 9 + 9 + 1) * 4 + 12 * 4,   # x, adjoint', F, dFc, order -> dLdv', dLdC'
    "adj_p2g_gather": (6 + 1 + 3 + 12 + 9 + 1) * 4 + 18 * 4,  # x, m, v, dLdv'/dLdC', G, order -> M, X, u, z
    # the finalize runs as two launches (both read M): the FP64 part and the FP32 transport part
    "adj_finalize": (9 + 9 + 9 + 9 + 6 + 3 + 9 + 9) * 4 + 9 * 4 + 9 * 8 * 2,  # M, F, dFc, R, S, vol/lam/mu,
                                                                                 # C', dLdF' -> dLdF, FP64 acc
    "adj_finalize_transport": (18 + 9 + 9 + 3 + 1) * 4 + 15 * 4,  # M/X/u/z, G, dLdC', dLdx', m -> dLdx, dLdv, dLdC
    "p2g_mass": 7 * 4, "loss_dldx": 7 * 4 + 24 * 4,
}
PER_TOUCHED_NODE_BYTES = {"p2g": 16, "g2p_p_op2": 16, "adj_g2p_scatter": 16, "adj_p2g_gather": 32,
                          "p2g_mass": 4, "loss_dldx": 4}
PER_GRID_NODE_BYTES = {"g_op": 32, "adj_g_op": 64}

# Executed flop per particle-step of the hot kernels (add + mul + 2 fma over the predicated-on
# thread instructions), counted by ncu on the 64^3, 266,868-particle workload
# (profiles/flops_atomics_hot_kernels_64cubed_267k.txt); it includes the warp-item layout's redundant
# weight evaluations.  Nominal vector peaks: 148 SMs x 128 FP32 / 64 FP64 lanes x 2 at 1965 MHz.
FLOP_PER_PARTICLE_STEP = {"fp32": 11375, "fp64": 1192}
NOMINAL_VECTOR_TFLOPS = {"fp32": 148 * 128 * 2 * 1.965e-3, "fp64": 148 * 64 * 2 * 1.965e-3}


def compute_rates(particle_steps_per_s: float) -> dict:
    out = {"source": "ncu-counted flop per particle-step x measured particle-steps/s, per GPU"}
    for p, f in FLOP_PER_PARTICLE_STEP.items():
        tf = particle_steps_per_s * f / 1e12
        out[p] = {"flop_per_particle_step": f, "tflops": tf, "nominal_tflops": NOMINAL_VECTOR_TFLOPS[p],
                  "frac": tf / NOMINAL_VECTOR_TFLOPS[p]}
    return out


def algorithmic_bytes(kernel: str, n: int, touched: int, nodes: int) -> float:
    return (PER_PARTICLE_BYTES.get(kernel, 0) * n + PER_TOUCHED_NODE_BYTES.get(kernel, 0) * touched
            + PER_GRID_NODE_BYTES.get(kernel, 0) * nodes)


def committed_traffic(kernel: str):
    """DRAM bytes per launch recorded from an ncu capture (profiles/roofline_traffic.txt), if any."""
    path = os.path.join(REPO, "profiles", "roofline_traffic.txt")
    try:
        for line in open(path):
            k, _, v = line.partition("=")
            if k.strip() == kernel:
                return float(v.split()[0])
    except Exception:
        pass
    return None


# ---------------------------------------------------------------- CPU baseline
def cpu_baseline(sc, sample_steps=1, threads=None):
    """The reference's own CPU implementation (oracle/_ref) on a bounded sample:
    MultiThreadMPM forward (all host threads) + EndLayerMassLoss +
    ComputeBackwardPass (serial) over `sample_steps` time steps of the workload."""
    from oracle import lib as olib

    threads = threads or os.cpu_count() or 1
    if olib.ref_available("f32"):
        r = olib.RefGraph(sc, "f32", target_from_points=True)
        vol = r.calc_volumes()
        sc2 = scenes.Scene(**{**sc.__dict__})
        sc2.vol = vol.astype(np.float64)
        r = olib.RefGraph(sc2, "f32", target_from_points=True)
        r.setup(sample_steps + 1, sc.dt, sc.drag, sc.f_ext, 0.0)
        t_fwd = r.time_forward_multithread(sample_steps, threads)
        t_bwd, _ = r.time_loss_backward()
        kind = "reference"
        desc = ("DiffMPMLib3D compiled from its sources (serial build): MultiThreadMPM::ForwardTimeStep with %d "
                "threads + EndLayerMassLoss + ComputeBackwardPass (1 thread) over %d time step(s) of the full "
                "%d-particle workload" % (threads, sample_steps, sc.n))
    else:
        g = olib.OracleGraph(sc, "f32")
        sc2 = scenes.Scene(**{**sc.__dict__})
        sc2.vol = g.calc_volumes().astype(np.float64)
        g = olib.OracleGraph(sc2, "f32")
        g.setup(sample_steps + 1, sc.dt, sc.drag, sc.f_ext, 0.0)
        t0 = time.perf_counter()
        g.forward(0)
        t_fwd = time.perf_counter() - t0
        t0 = time.perf_counter()
        g.loss()
        g.backward(0, 1)
        t_bwd = time.perf_counter() - t0
        threads = 1
        kind = "port"
        desc = "serial CPU restatement (oracle), %d time step(s) of the %d-particle workload" % (sample_steps, sc.n)
    total = t_fwd + t_bwd
    return {"value": sc.n * sample_steps / total, "unit": UNIT, "cores": threads, "kind": kind, "sample": desc,
            "forward_s": t_fwd, "loss_backward_s": t_bwd}


# ---------------------------------------------------------------- arms
def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sc = build_scene(0, args.ppc_root)
    if args.rollout_steps:
        sc.steps = args.rollout_steps
    # the configured dt (5e-4) is 3.7x the explicit CFL limit and diverges; both
    # arms run at half the limit (throughput does not depend on dt)
    dt_sub = sc.dt
    sc.dt = args.dt if args.dt else 0.5 * sc.cfl_dt()
    for _ in range(args.warmup):
        cpu_baseline(sc, 1)
    times = []
    cb = None
    for _ in range(args.steps):
        cb = cpu_baseline(sc, 1)
        times.append(cb["forward_s"] + cb["loss_backward_s"])
    total = sum(times)
    value = sc.n * args.steps / total
    cb = dict(cb)
    cb["value"] = value
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(sc, None if args.dt else dt_sub, 1),
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def workload_config(sc, dt_sub, ckpt):
    return {"workload": "ellipsoid(0.3,0.2,0.15)->torus(R=0.25,r=0.08), 64^3 grid, %d particles (%d per cell), "
                        "%d steps, forward + end-layer mass loss + adjoint" % (sc.n, sc.meta["ppc"], sc.steps),
            "particles": sc.n, "grid": list(sc.dims), "layers": sc.steps + 1, "dt": sc.dt,
            "dt_substituted_from": dt_sub, "checkpoint_every": ckpt, "loss": "reference log-mass + min-mass penalty",
            "l2_policy": "inputs larger than L2 (per-rollout layer state > 5 GB, 126 MB L2)",
            "g2p_kernel": "warp items" if BRICK_CELLS == 0 else "bricks of %d^3 cells" % (BRICK_CELLS or 2),
            "particle_order": "seeded random permutation" if SHUFFLE else "lattice",
            "reorder_particles": REORDER,
            "parallelism": "replicas: one independent instance per GPU"}


def measure_variant(torch, dmpm, sc, vol, target, device, ckpt, args, deterministic=None):
    """One gradient evaluation of scene sc per step on both paths under one
    storage policy (checkpoint_every = ckpt): FP32-mixed particle-steps/s, device
    memory held, and the plain FP64 path on the same policy (its throughput and
    the FP32 gradient's relative error against it).  deterministic=True: the
    FP32 path's integer node sums, and a second evaluation in a fresh context
    to show that the gradient repeats bit for bit."""
    if vol is None:
        sc.dt, _ = _cfl_dt(sc)
        vol, target = _scene_inputs(dmpm, sc, device)
    units = sc.n * sc.steps
    torch.cuda.synchronize()
    base = _mem_used_gb(torch, device)
    c = setup_ctx(dmpm, sc, "fp32", device, vol, target, sc.dt, ckpt, deterministic=deterministic)
    for _ in range(args.warmup):
        gradient_step(c)
    hbm = _mem_used_gb(torch, device) - base
    n = max(1, min(args.steps, 5))
    ms = timed_steps(torch, c, n, lambda: gradient_step(c)) / n
    g32 = c.control_grad()
    info = c.info()
    c.close()
    out = {"particles": sc.n, "steps": sc.steps, "checkpoint_every": info["checkpoint_every"],
           "value": units / (ms / 1000.0), "unit": UNIT, "ms_per_gradient": ms, "hbm_gb": hbm,
           "engine_bytes_gb": info["device_bytes"] / 1e9}
    if deterministic:
        c2 = setup_ctx(dmpm, sc, "fp32", device, vol, target, sc.dt, ckpt, deterministic=True)
        gradient_step(c2)
        g2 = c2.control_grad()
        c2.close()
        out["repeat_bit_identical"] = bool(np.array_equal(g32, g2))
        out["repeat_relerr"] = float(np.linalg.norm(g2 - g32) / np.linalg.norm(g32))
    if not args.no_fp64:
        c64 = setup_ctx(dmpm, sc, "fp64", device, vol, target, sc.dt, ckpt)
        gradient_step(c64)
        ms64 = timed_steps(torch, c64, 1, lambda: gradient_step(c64))
        g64 = c64.control_grad()
        c64.close()
        rel = float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64))
        out["fp64"] = {"value": units / (ms64 / 1000.0), "ms_per_gradient": ms64,
                       "speedup_fp32_mixed_over_fp64": ms64 / ms, "grad_relerr_vs_fp64": rel,
                       "meets_bar": rel <= 1e-4}
    return out


def run_ours(args):
    import torch

    import dmpm

    world, rank, local = dist_setup(args.gpus)
    device = local
    torch.cuda.set_device(device)
    sc = build_scene(rank, args.ppc_root)
    if args.rollout_steps:
        sc.steps = args.rollout_steps
    dt_cfg = sc.dt
    # volumes (CalculatePointCloudVolumes) and the target raster (mass-only P2G of the
    # target samples, as LoadCompGraph builds it) on the FP64 path, shared by both paths
    with dmpm.Context("fp64", device) as c64:
        c64.load_scene(sc)
        c64.set_params(dt=sc.dt)
        c64.setup(1)
        vol = c64.get(0, "vol")
        target = c64.target_mass()
    ckpt = args.checkpoint_every
    # run the configured dt; fall back to half the explicit CFL limit if it blows up
    dt_sub = None
    if args.dt:
        sc.dt = args.dt
    c = setup_ctx(dmpm, sc, "fp32", device, vol, target, sc.dt, ckpt)
    if not args.dt and not finite_gradient(dmpm, c):
        # the configured dt is above the explicit limit and the rollout or its
        # adjoint diverges: rerun at half the CFL limit and record the substitution
        dt_sub = dt_cfg
        sc.dt = 0.5 * sc.cfl_dt()
        c.close()
        c = setup_ctx(dmpm, sc, "fp32", device, vol, target, sc.dt, ckpt)
        assert finite_gradient(dmpm, c), "gradient not finite at half the CFL limit"
    units_per_step = sc.n * sc.steps  # particle-steps of one gradient evaluation
    for _ in range(args.warmup):
        gradient_step(c)
    l0 = c.launch_count
    barrier(world)
    sampler = ClockSampler(device)
    sampler.start()
    ms = timed_steps(torch, c, args.steps, lambda: gradient_step(c))
    clocks = sampler.stop()
    launches = c.launch_count - l0
    barrier(world)
    # per-kernel device times: the same K steps again with every launch bracketed
    # by CUDA events on the engine's stream (kept out of the region above because
    # the events add gaps between kernels)
    c.set_profiling(True)
    ms_prof = timed_steps(torch, c, args.steps, lambda: gradient_step(c))
    kstats = c.kernel_stats()
    c.set_profiling(False)
    ms_max = max_over_ranks(ms, world)
    value = whole_job_value(units_per_step, args.steps, world, ms_max)
    grad32 = c.control_grad()

    # e2e through the C ABI with pinned host buffers
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).pin_memory()
    cm = lambda M: np.ascontiguousarray(np.asarray(M).transpose(0, 2, 1).reshape(-1, 9))
    hx, hv, hF, hC, hd = pin(sc.x), pin(sc.v), pin(cm(sc.F)), pin(cm(sc.C)), pin(cm(sc.dFc))
    hm, hvol, hl, hmu = pin(sc.m), pin(vol), pin(sc.lam), pin(sc.mu)
    hgrad = torch.empty(sc.n * 9, dtype=torch.float64).pin_memory()
    h2d = sum(t.numel() * 8 for t in (hx, hv, hF, hC, hd, hm, hvol, hl, hmu))
    d2h = hgrad.numel() * 8 + 8

    def e2e_step():
        c._set_particles_raw(sc.n, hx, hv, hF, hC, hd, hm, hvol, hl, hmu)
        c.setup(sc.steps + 1)
        gradient_step(c)
        c.control_grad(0, out=hgrad)

    e2e_step()
    barrier(world)
    ms_e2e = max_over_ranks(timed_steps(torch, c, args.steps, e2e_step), world)
    e2e_value = whole_job_value(units_per_step, args.steps, world, ms_e2e)
    touched = int(np.count_nonzero(c.get_grid(0, "grid_m")))
    nodes = int(np.prod(sc.dims))
    c.close()

    # plain FP64 GPU path on the same workload
    fp64 = None
    if not args.no_fp64:
        c64 = setup_ctx(dmpm, sc, "fp64", device, vol, target, sc.dt, ckpt)
        gradient_step(c64)
        n64 = max(1, min(args.steps, 2))
        ms64 = timed_steps(torch, c64, n64, lambda: gradient_step(c64))
        grad64 = c64.control_grad()
        c64.close()
        v64 = units_per_step * n64 / (ms64 / 1000.0)
        relerr = float(np.linalg.norm(grad32 - grad64) / np.linalg.norm(grad64))
        # the FP64 path once more on the scene's unrounded (float64) inputs: how far
        # rounding the inputs to float32 alone moves the gradient of this rollout
        c64 = setup_ctx(dmpm, sc, "fp64", device, vol, target, sc.dt, ckpt, same_inputs=False)
        gradient_step(c64)
        grad64u = c64.control_grad()
        c64.close()
        fp64 = {"value": v64 * world, "unit": UNIT, "ms_per_step": ms64 / n64,
                "speedup_fp32_mixed_over_fp64": (value / world) / v64, "grad_relerr_vs_fp64": relerr,
                "grad_relerr_bar": 1e-4, "meets_bar": relerr <= 1e-4,
                "inputs": "both paths from the same float32-rounded inputs",
                "grad_relerr_fp32_vs_fp64_on_float64_inputs":
                    float(np.linalg.norm(grad32 - grad64u) / np.linalg.norm(grad64u)),
                "grad_relerr_fp64_float32_inputs_vs_float64_inputs":
                    float(np.linalg.norm(grad64 - grad64u) / np.linalg.norm(grad64u))}

    # roofline of the dominant kernel (largest total device time)
    peak, peak_kind = measured_hbm_gbs()
    kern = {k: {"total_ms": v[0], "launches": v[1], "avg_us": 1000.0 * v[0] / v[1]} for k, v in kstats.items()}
    top = max(kern, key=lambda k: kern[k]["total_ms"]) if kern else None
    roof = None
    if top:
        alg = algorithmic_bytes(top, sc.n, touched, nodes)
        achieved = alg / (kern[top]["avg_us"] * 1e-6) / 1e9
        roof = {"kernel": top, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": committed_traffic(top), "algorithmic_bytes_per_launch": alg,
                "avg_launch_us": kern[top]["avg_us"]}
        for k in kern:
            b = algorithmic_bytes(k, sc.n, touched, nodes)
            if b:
                kern[k]["hbm_frac"] = b / (kern[k]["avg_us"] * 1e-6) / 1e9 / peak

    # the target's other clauses, measured in the same run on one GPU: the same
    # workload with checkpoints every 15 layers (recompute in between), and the
    # configuration's own 8 particles per cell
    variants = None
    if world == 1 and not args.no_variants:
        variants = {"checkpointed": measure_variant(torch, dmpm, sc, vol, target, device, 15, args),
                    "deterministic": measure_variant(torch, dmpm, sc, vol, target, device, ckpt, args,
                                                     deterministic=True),
                    "as_specified_8ppc": measure_variant(torch, dmpm, build_scene(rank, 2), None, None, device,
                                                         ckpt, args)}
        variants["checkpointed"]["store_all_ms_per_gradient"] = ms_max / args.steps
        variants["checkpointed"]["recompute_overhead"] = (
            variants["checkpointed"]["ms_per_gradient"] / (ms_max / args.steps) - 1.0)

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(sc, 1)
        cb = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 (f64 polar/SVD, stress derivative, loss and gradient sums)", "data": "synthetic",
                "config": workload_config(sc, dt_sub, ckpt),
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "gpu_launches": launches, "roofline": roof, "compute": compute_rates(value / world), "cpu_baseline": cb,
                "clocks": clocks, "fp64": fp64, "kernels": kern, "ms_per_step_profiled": ms_prof / args.steps,
                **(variants or {})}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------- configs 0, 2, 4
def _cfl_dt(sc):
    """Configured dt, or half the explicit CFL limit when the configured dt exceeds it."""
    lim = sc.cfl_dt()
    return (sc.dt, None) if sc.dt <= lim else (0.5 * lim, sc.dt)


def _scene_inputs(dmpm, sc, device):
    with dmpm.Context("fp64", device) as c64:
        c64.load_scene(sc)
        c64.set_params(dt=sc.dt)
        c64.setup(1)
        return c64.get(0, "vol"), c64.target_mass()


def _mem_used_gb(torch, device):
    free, total = torch.cuda.mem_get_info(device)
    return (total - free) / 1e9


def run_fd(args):
    """Config 1 at full size: the adjoint's directional derivatives g.d (plain
    FP64 path and FP32-mixed path, exact adjoint, tied controls) against FP64
    central differences (L(dFc + h d) - L(dFc - h d)) / 2h along 16 seeded
    directions d with N(0, 1) entries, for h = 1e-3 (the configured step) and
    smaller steps, with the reference's log-mass loss and with plain L2.  The
    reference loss takes log(m + 1 + 1e-4) of node masses of a few 1e-6, so in
    FP64 it resolves mass changes only to ~2e-16 absolute and small steps
    measure its rounding; the L2 loss shows the adjoint itself."""
    import dmpm

    sc = build_scene(0, args.ppc_root)
    if args.rollout_steps:
        sc.steps = args.rollout_steps
    sc.dt, dt_sub = _cfl_dt(sc)
    vol, target = _scene_inputs(dmpm, sc, 0)
    hs = [float(x) for x in args.fd_h.split(",")]
    ndir = 16
    rng = np.random.default_rng(12345)
    dirs = [rng.normal(size=(sc.n, 3, 3)) for _ in range(ndir)]
    out = {"mode": "fd", "workload": "ellipsoid -> torus, 64^3, %d particles, %d steps" % (sc.n, sc.steps),
           "dt": sc.dt, "dt_substituted_from": dt_sub, "directions": ndir}
    for loss in ("ref", "l2"):
        grads = {}
        for prec in ("fp64", "fp32"):
            c = setup_ctx(dmpm, sc, prec, 0, vol, target, sc.dt, 1)
            c.set_params(dt=sc.dt, drag=sc.drag, f_ext=sc.f_ext, smoothing=sc.smoothing, adjoint="exact",
                         control="tied", loss=loss, checkpoint_every=1)
            c.setup(sc.steps + 1)
            gradient_step(c)
            grads[prec] = c.control_grad()
            if prec == "fp64":
                c64 = c
            else:
                c.close()
        base = c64.get(0, "dFc")
        a64 = [float(np.sum(grads["fp64"] * d)) for d in dirs]
        a32 = [float(np.sum(grads["fp32"] * d)) for d in dirs]
        per_h = {}
        for h in hs:
            fds, crossings = [], []
            for d in dirs:
                lp = []
                occ = None
                for sgn in (1.0, -1.0):
                    c64.set_layer(0, "dFc", base + sgn * h * d)
                    c64.forward(0)
                    lp.append(c64.loss())
                    # node-mass threshold crossings between the two rollouts: nodes
                    # (over all layers) occupied, |m| > FLT_EPSILON, in one and not the other
                    masks = [np.abs(c64.get_grid(lay, "grid_m")) > FLT_EPSILON for lay in range(sc.steps + 1)]
                    if occ is None:
                        occ = masks
                    else:
                        crossings.append(int(sum(int(np.count_nonzero(a != b)) for a, b in zip(occ, masks))))
                fds.append((lp[0] - lp[1]) / (2 * h))
            e64 = [abs(a - f) / abs(f) for a, f in zip(a64, fds)]
            e32 = [abs(a - f) / abs(f) for a, f in zip(a32, fds)]
            per_h["%g" % h] = {"relerr_fp64_median": float(np.median(e64)), "relerr_fp64_max": float(np.max(e64)),
                               "relerr_fp32_median": float(np.median(e32)), "relerr_fp32_max": float(np.max(e32))}
            if crossings:
                per_h["%g" % h]["per_direction"] = [
                    {"threshold_crossings": cr, "relerr_fp64": e, "relerr_fp32": e3}
                    for cr, e, e3 in zip(crossings, e64, e32)]
                zero = [e for cr, e in zip(crossings, e64) if cr == 0]
                per_h["%g" % h]["directions_without_crossings"] = len(zero)
                if zero:
                    per_h["%g" % h]["relerr_fp64_max_without_crossings"] = float(np.max(zero))
        c64.close()
        out[loss] = {"grad_relerr_fp32_vs_fp64": float(np.linalg.norm(grads["fp32"] - grads["fp64"]) /
                                                       np.linalg.norm(grads["fp64"])), "per_h": per_h}
    print(json.dumps(out), flush=True)
    return 0


def run_config0(args):
    """Config 0 at full size: the plain FP64 GPU path against the reference's own
    FP64 build (oracle/_ref) on the same scene -- forward state, loss and the
    reference-compatible adjoint -- plus both throughputs."""
    import torch

    import dmpm
    from oracle import lib as olib

    sc = scenes.config_scene(0)
    sc.dt, dt_sub = _cfl_dt(sc)
    vol, target = _scene_inputs(dmpm, sc, 0)
    sc.vol = vol
    L = sc.steps + 1
    out = {"mode": "config0", "particles": sc.n, "grid": list(sc.dims), "steps": sc.steps, "dt": sc.dt,
           "dt_substituted_from": dt_sub, "loss": "reference log-mass + penalty", "adjoint": "refcompat"}
    c = setup_ctx(dmpm, sc, "fp64", 0, vol, target, sc.dt, 1, same_inputs=False)
    c.set_params(dt=sc.dt, drag=sc.drag, f_ext=sc.f_ext, smoothing=sc.smoothing, adjoint="refcompat",
                 control="per_layer", keep_adjoints=True)
    c.setup(L)
    gradient_step(c)
    ms = timed_steps(torch, c, 1, lambda: gradient_step(c))
    g_loss = c.loss()
    c.backward(0)
    out["gpu_fp64_particle_steps_per_s"] = sc.n * sc.steps / (ms / 1000.0)
    if olib.ref_available("f64"):
        r = olib.RefGraph(sc, "f64", target_m=target)
        r.setup(L, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
        t0 = time.perf_counter()
        r.forward(0)
        r_loss = r.loss()
        r.backward(0)
        t_ref = time.perf_counter() - t0
        rel = lambda a, b: float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
        nrel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
        rF, rx = r.get(0, "dLdF"), r.get(0, "dLdx")
        gF, gx = c.get(0, "dLdF"), c.get(0, "dLdx")
        out.update({"ref_fp64_particle_steps_per_s": sc.n * sc.steps / t_ref,
                    "relerr_x_last": rel(c.get(L - 1, "x"), r.get(L - 1, "x")),
                    "relerr_loss": abs(g_loss - r_loss) / abs(r_loss),
                    "relerr_dLdF_layer0": rel(gF, rF), "relerr_dLdx_layer0": rel(gx, rx),
                    "normrel_dLdF_layer0": nrel(gF, rF), "normrel_dLdx_layer0": nrel(gx, rx),
                    "parity_bar": 1e-10})
        # the reference against itself, positions perturbed by one ulp: its
        # finite-difference d(J F^-T)/dF (delta 1e-6, Elasticity.cpp:7-72) turns
        # rounding-level input changes into ~1e-10 changes of the adjoint
        sc_ulp = scenes.Scene(**{**sc.__dict__, "x": sc.x * (1.0 + 2.0 ** -52)})
        r2 = olib.RefGraph(sc_ulp, "f64", target_m=target)
        r2.setup(L, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
        r2.forward(0)
        r2.loss()
        r2.backward(0)
        out.update({"ref_vs_ref_ulp_relerr_dLdF_layer0": rel(r2.get(0, "dLdF"), rF),
                    "ref_vs_ref_ulp_relerr_dLdx_layer0": rel(r2.get(0, "dLdx"), rx),
                    "ref_vs_ref_ulp_normrel_dLdF_layer0": nrel(r2.get(0, "dLdF"), rF)})
    else:
        out["ref_fp64"] = "unavailable: oracle/_ref not built"
    c.close()
    print(json.dumps(out), flush=True)
    return 0


def run_config2(args):
    """Config 2: union of 3 spheres, 128^3, 500 steps -- store-all vs checkpoint
    every 25 steps (peak HBM, recompute overhead), FP32-mixed, exact adjoint."""
    import torch

    import dmpm

    sc = scenes.config_scene(2)
    if args.rollout_steps:
        sc.steps = args.rollout_steps
    sc.dt, dt_sub = _cfl_dt(sc)
    vol, target = _scene_inputs(dmpm, sc, 0)
    out = {"mode": "config2", "particles": sc.n, "grid": list(sc.dims), "steps": sc.steps, "dt": sc.dt,
           "dt_substituted_from": dt_sub, "deterministic": DETERMINISTIC}
    grads = {}
    for ckpt in (1, 25):
        torch.cuda.synchronize()
        base = _mem_used_gb(torch, 0)
        c = setup_ctx(dmpm, sc, "fp32", 0, vol, target, sc.dt, ckpt)
        gradient_step(c)
        first = c.control_grad()
        used = _mem_used_gb(torch, 0) - base
        n = max(1, args.steps // 4)
        ms = timed_steps(torch, c, n, lambda: gradient_step(c)) / n
        grads[ckpt] = c.control_grad()
        if ckpt == 1:  # same inputs twice: the FP32 run-to-run spread (float atomic summation order; 0 when deterministic)
            out["grad_relerr_fp32_repeat"] = float(np.linalg.norm(grads[1] - first) / np.linalg.norm(first))
        out["ckpt%d" % ckpt] = {"ms_per_gradient": ms, "particle_steps_per_s": sc.n * sc.steps / (ms / 1000.0),
                                "hbm_gb": used, "engine_bytes_gb": c.info()["device_bytes"] / 1e9,
                                "checkpoint_every": c.info()["checkpoint_every"]}
        c.close()
    out["recompute_overhead"] = out["ckpt25"]["ms_per_gradient"] / out["ckpt1"]["ms_per_gradient"] - 1.0
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    out["grad_relerr_ckpt25_vs_store_all"] = rel(grads[25], grads[1])
    if not args.no_fp64:
        # the FP64 path twice on the same inputs: its spread is FP64 rounding
        # (atomic summation order) amplified by the adjoint of this rollout
        c64 = setup_ctx(dmpm, sc, "fp64", 0, vol, target, sc.dt, 25)
        t0 = time.perf_counter()
        gradient_step(c64)
        g64 = c64.control_grad()
        out["fp64_ckpt25_s"] = time.perf_counter() - t0
        gradient_step(c64)
        out["grad_relerr_fp64_repeat"] = rel(c64.control_grad(), g64)
        c64.close()
        out["grad_relerr_fp32_store_all_vs_fp64"] = rel(grads[1], g64)
        out["grad_relerr_fp32_ckpt25_vs_fp64"] = rel(grads[25], g64)
        # the FP64 path on the scene's unrounded inputs: the floor that rounding the
        # inputs to float32 sets for any path that stores them in float32
        c64 = setup_ctx(dmpm, sc, "fp64", 0, vol, target, sc.dt, 25, same_inputs=False)
        gradient_step(c64)
        g64u = c64.control_grad()
        c64.close()
        out["inputs"] = "both paths from the same float32-rounded inputs"
        out["grad_relerr_fp64_float32_inputs_vs_float64_inputs"] = rel(g64, g64u)
        out["grad_relerr_fp32_vs_fp64_on_float64_inputs"] = rel(grads[1], g64u)
    print(json.dumps(out), flush=True)
    return 0


def run_config3(args):
    """Config 3: 48 seeded instances (sphere / ellipsoid / box, 5k-150k
    particles, 32^3 or 64^3, 100-300 steps) in one batch: one launch per stage
    per time step, the gradient evaluation replayed as a CUDA graph, launch
    settings autotuned; against the same batch without the graph and against
    one engine context per instance run one after another."""
    import torch

    import dmpm

    world, rank, local = dist_setup(args.gpus)
    all_scs = scenes.batch_scenes(args.instances)
    lim = min(sc.cfl_dt() for sc in all_scs)  # one dt for every instance: the smallest limit
    dt0 = all_scs[0].dt
    dt = dt0 if dt0 <= lim else 0.5 * lim
    units_all = float(sum(sc.n * sc.steps for sc in all_scs))
    mine = shard_instances([sc.n * sc.steps for sc in all_scs], world, rank)
    scs = [all_scs[i] for i in mine]
    units = float(sum(sc.n * sc.steps for sc in scs))  # particle-steps of one gradient evaluation
    inputs = [_scene_inputs(dmpm, sc, local) for sc in scs]
    out = {"mode": "config3", "n_gpus": world, "scaling": "strong", "instances": len(all_scs),
           "instances_on_rank0": len(scs), "particles": int(sum(sc.n for sc in all_scs)),
           "particle_range": [int(min(sc.n for sc in scs)), int(max(sc.n for sc in scs))],
           "steps_range": [int(min(sc.steps for sc in scs)), int(max(sc.steps for sc in scs))],
           "grids": sorted({int(sc.dims[0]) for sc in scs}), "particle_steps_per_gradient": units, "dt": dt,
           "dt_substituted_from": dt0 if dt != dt0 else None}
    torch.cuda.synchronize()
    base = _mem_used_gb(torch, local)
    b = dmpm.Batch([{"n": sc.n, "dims": sc.dims, "dx": sc.dx, "min_point": sc.min_point, "steps": sc.steps}
                    for sc in scs], device=local)
    b.set_params(dt=dt, drag=scs[0].drag, f_ext=scs[0].f_ext, smoothing=scs[0].smoothing, adjoint="exact")
    for i, sc in enumerate(scs):
        vol, target = inputs[i]
        b.set_particles(i, sc.x, sc.m, sc.lam, sc.mu, v=sc.v, F=sc.F, C=sc.C, dFc=sc.dFc, vol=vol)
        b.set_target_mass(i, target)
    b.set_launch(use_graph=True)
    b.setup()
    out["hbm_gb"] = _mem_used_gb(torch, local) - base
    t0 = time.perf_counter()
    out["autotune_best_ms"] = b.autotune(reps=1)
    out["autotune_s"] = time.perf_counter() - t0
    out["launch"] = b.launch()
    stream = torch.cuda.ExternalStream(b.stream)
    reps = max(2, args.steps // 4)

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        fn()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    losses = b.gradient()
    barrier(world)
    ms_graph = max_over_ranks(timed(lambda: b.gradient()), world)
    info = b.info()
    grads = {i: b.control_grad(i) for i in sorted({0, min(1, len(scs) - 1), len(scs) - 1})}
    cfg = b.launch()
    b.set_launch(sort_every=cfg["sort_every"], ctas_per_sm=cfg["ctas_per_sm"],
                 particle_block=cfg["particle_block"], use_graph=False)
    barrier(world)
    ms_eager = max_over_ranks(timed(lambda: b.gradient()), world)
    b.close()
    # whole job: every rank's particle-steps over the slowest rank's device time
    out["batched_graph"] = {"ms_per_gradient": ms_graph, "particle_steps_per_s": units_all / (ms_graph / 1e3),
                            "launches_per_gradient": info["launches_per_gradient"]}
    out["batched_eager"] = {"ms_per_gradient": ms_eager, "particle_steps_per_s": units_all / (ms_eager / 1e3)}
    # one engine context per instance, one after another (each with its own launches and syncs)
    tot_ms, relerr_loss, relerr_grad = 0.0, 0.0, 0.0
    for i, sc in enumerate(scs):
        vol, target = inputs[i]
        c = setup_ctx(dmpm, sc, "fp32", local, vol, target, dt, 1)
        s_i = torch.cuda.ExternalStream(c.stream)
        gradient_step(c)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s_i)
        for _ in range(reps):
            lo = gradient_step(c)
        e1.record(s_i)
        e1.synchronize()
        tot_ms += e0.elapsed_time(e1) / reps
        relerr_loss = max(relerr_loss, abs(lo - losses[i]) / abs(lo))
        if i in grads:
            g = c.control_grad()
            relerr_grad = max(relerr_grad, float(np.linalg.norm(grads[i] - g) / np.linalg.norm(g)))
        c.close()
    tot_ms = max_over_ranks(tot_ms, world)
    out["one_context_per_instance"] = {"ms_per_gradient": tot_ms, "particle_steps_per_s": units_all / (tot_ms / 1e3)}
    out["speedup_graph_over_per_instance"] = tot_ms / ms_graph
    out["speedup_graph_over_eager"] = ms_eager / ms_graph
    out["max_loss_relerr_batch_vs_per_instance"] = relerr_loss
    out["max_grad_relerr_batch_vs_per_instance"] = relerr_grad
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def run_config4(args):
    """Config 4: sphere -> torus at 256^3 (~8M particles), 400 steps, checkpoint
    every 20, 30 device Adam iterations (lr 1e-2) on the per-particle controls of
    the first control frame (layer 0; the reference's optimiser descends one
    frame's dFc at a time, CompGraph.cpp:352-420, with the gradient divided by
    its norm, PointCloud.cpp:83-99); loss curve, per-iteration time, FP32
    gradient error vs the FP64 GPU path at iterations 1 and the last."""
    import torch

    import dmpm

    sc = scenes.config_scene(4)
    if args.rollout_steps:
        sc.steps = args.rollout_steps
    sc.dt, dt_sub = _cfl_dt(sc)
    vol, target = _scene_inputs(dmpm, sc, 0)
    iters = args.iters
    out = {"mode": "config4", "particles": sc.n, "grid": list(sc.dims), "steps": sc.steps, "dt": sc.dt,
           "dt_substituted_from": dt_sub, "checkpoint_every": 20, "iterations": iters, "lr": args.lr,
           "deterministic": DETERMINISTIC}
    torch.cuda.synchronize()
    base = _mem_used_gb(torch, 0)
    if args.controls == "tied":  # one dFc per particle, applied at every step; gradient summed over the layers
        frame = dict(control="tied")
    else:  # layer 0 is the only control frame
        frame = dict(control="per_layer", control_stride=sc.steps)
    c = setup_ctx(dmpm, sc, "fp32", 0, vol, target, sc.dt, 20, **frame)
    out["hbm_gb_fp32"] = _mem_used_gb(torch, 0) - base
    out["controls"] = ("per-particle dFc tied over all layers, exact adjoint" if args.controls == "tied" else
                       "per-particle dFc of layer 0 (one control frame), exact adjoint")
    losses, times, relerrs = [], [], {}

    def fp64_relerr(grad32, dfc):
        c64 = setup_ctx(dmpm, sc, "fp64", 0, vol, target, sc.dt, 20, **frame)
        c64.set_layer(0, "dFc", dfc)
        gradient_step(c64)
        g64 = c64.control_grad(0)
        c64.close()
        return float(np.linalg.norm(grad32 - g64) / np.linalg.norm(g64))

    # Plain Adam (the configuration: 30 iterations at lr 1e-2; --lr changes it), or with --line-search the
    # reference optimiser's line search (CompGraph.cpp:388-420): step, re-run the forward pass,
    # keep the step if the loss fell, else step back (Descend_Adam with -alpha, which updates the
    # moments again, as the reference does) and halve alpha; a frame whose line search finds no
    # decrease ends its descent.
    out["optimizer"] = "adam with the reference line search" if args.line_search else "adam, fixed lr"
    max_ls = 6 if args.line_search else 1
    ls_trials, grad_ms, stopped, last, nonfinite = [], [], None, None, None

    def statused_gradient(holder):
        st_f = c.forward(0)
        holder["loss"] = c.loss()
        st_b = c.backward(0)
        holder["finite"] = st_f == dmpm.OK and st_b == dmpm.OK and math.isfinite(holder["loss"])

    for it in range(1, iters + 1):
        holder = {}
        ms = timed_steps(torch, c, 1, lambda: statused_gradient(holder))
        loss = holder["loss"]
        losses.append(loss)
        grad_ms.append(ms)
        if not holder["finite"]:  # the rollout or its adjoint went non-finite at these controls
            nonfinite = it
            break
        if not args.no_fp64:  # the controls and FP32 gradient of this iteration (host copies)
            last = (it, c.control_grad(0), c.get(0, "dFc"))
            if it == 1:
                relerrs[1] = fp64_relerr(last[1], last[2])
        t0 = time.perf_counter()
        if not args.line_search:
            c.adam_step(t=it, lr=args.lr, layer=0)
            c.synchronize()
            times.append(ms + 1000.0 * (time.perf_counter() - t0))
            continue
        alpha, found = args.lr, False
        for ls in range(max_ls):
            c.adam_step(t=it, lr=alpha, layer=0)
            st = c.forward(0)
            trial = c.loss()
            if st == dmpm.OK and math.isfinite(trial) and trial < loss:
                found = True
                break
            c.adam_step(t=it, lr=-alpha, layer=0)
            alpha *= 0.5
        c.synchronize()
        ls_trials.append(ls + 1)
        times.append(ms + 1000.0 * (time.perf_counter() - t0))
        if not found:
            stopped = it
            break
    if last is not None and last[0] not in relerrs:
        relerrs[last[0]] = fp64_relerr(last[1], last[2])
    out.update({"loss_curve": losses, "ms_per_iteration": times, "ms_per_gradient": grad_ms,
                "line_search_trials": ls_trials, "max_line_search_trials": max_ls,
                "stopped_at_iteration_without_decrease": stopped,
                "stopped_at_iteration_nonfinite": nonfinite,
                "particle_steps_per_s": sc.n * sc.steps / (float(np.median(grad_ms)) / 1000.0),
                "grad_relerr_vs_fp64": relerrs})
    c.close()
    print(json.dumps(out), flush=True)
    return 0


# ---------------------------------------------------------------- mesh sampling and surfacing
def run_next_rows(args):
    """The point-cloud sampler and the two surfacing functions on a 1.08M-point
    workload: the torus fixture (tests/golden/mesh_torus.obj) sampled at a 0.005
    lattice spacing, then surfaced over [-1, 1]^3 with the fixture's parameters.
    GPU: the Python API with host arrays, median of 5 after one warm-up, copies
    included.  CPU baseline: the reference's own sampler and surfacing compiled
    here (oracle/_ref/ref_mesh, ref_surface: readOBJ or the point file, the
    computation and the output file), best of 2, on the same host."""
    import resource

    import torch

    import dmpm

    dmpm.load_library()
    ref_dir = os.path.join(REPO, "oracle", "_ref")
    obj = os.path.join(REPO, "tests", "golden", "mesh_torus.obj")
    dx = 0.005
    box_min, box_max = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)

    def gpu(fn, n=5):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(n):
            t0 = time.perf_counter()
            out = fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts)), out

    def ref(cmd, n=2):
        best, threads = 1e9, 0.0
        for _ in range(n):
            r0 = resource.getrusage(resource.RUSAGE_CHILDREN)
            t0 = time.perf_counter()
            subprocess.check_call(cmd, stdout=subprocess.DEVNULL)
            w = time.perf_counter() - t0
            r1 = resource.getrusage(resource.RUSAGE_CHILDREN)
            if w < best:
                best = w
                threads = ((r1.ru_utime - r0.ru_utime) + (r1.ru_stime - r0.ru_stime)) / w
        return best, threads

    import tempfile

    V, F = dmpm.read_obj(obj)
    t_s, pts = gpu(lambda: dmpm.mesh_lattice_points(V, F, dx))
    pts = pts.astype(np.float32)
    out = {"mode": "mesh sampling and surfacing", "points": int(len(pts)), "host_cores": os.cpu_count()}
    with tempfile.TemporaryDirectory() as tmp:
        pf = os.path.join(tmp, "pts.f32")
        r_s, th_s = ref([os.path.join(ref_dir, "ref_mesh"), obj, repr(dx), pf])
        rp = np.fromfile(pf, dtype=np.float32).reshape(-1, 3)
        out["points_identical_to_reference"] = bool(rp.shape == pts.shape and np.array_equal(rp, pts))
        box = ["-1.0", "-1.0", "-1.0", "1.0", "1.0", "1.0"]
        t_su, (_, Fs) = gpu(lambda: dmpm.sphere_union_surface(pts, 0.025, 0.025, 0.025, 2, box_min, box_max))
        r_su, th_su = ref([os.path.join(ref_dir, "ref_surface"), "spheres", pf, "0.025", repr(float(np.float32(0.025))),
                           "0.025", "2", *box, os.path.join(tmp, "sph.bin")])
        t_mc, (_, Fm) = gpu(lambda: dmpm.marching_cubes_point_cloud(pts, 0.5, 0.05, 2.0, box_min, box_max))
        r_mc, th_mc = ref([os.path.join(ref_dir, "ref_surface"), "mass", pf, "1.0", "0.05", "2.0", "0.5", *box,
                           os.path.join(tmp, "mass.bin")])
    for key, tg, tr, th, tris in (("mesh_sampler", t_s, r_s, th_s, None),
                                  ("sphere_union_surface", t_su, r_su, th_su, len(Fs)),
                                  ("marching_cubes_point_cloud", t_mc, r_mc, th_mc, len(Fm))):
        out[key] = {"gpu_s": tg, "reference_s": tr, "reference_threads": round(th, 1), "speedup": tr / tg}
        if tris is not None:
            out[key]["triangles"] = int(tris)
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--ppc-root", type=int, default=3, help="particles per cell = ppc_root^3 (3 -> ~267k)")
    ap.add_argument("--dt", type=float, default=0.0, help="override dt (default: configured, CFL fallback)")
    ap.add_argument("--checkpoint-every", type=int, default=1)
    ap.add_argument("--brick", type=int, default=None, choices=[0, 2, 4],
                    help="FP32 G2P kernel: 0 warp items, 2 or 4 cells per brick axis (default 2)")
    ap.add_argument("--sort-every", type=int, default=None, help="FP32 cell-sort interval in steps (default 8)")
    ap.add_argument("--deterministic", action="store_true",
                    help="FP32 path with integer node sums: gradients repeat bit for bit")
    ap.add_argument("--shuffle", action="store_true", help="hand the cloud over in a seeded random order")
    ap.add_argument("--reorder", action="store_true",
                    help="FP32 path: store the cloud in cell order at setup (reorder_particles)")
    ap.add_argument("--rollout-steps", type=int, default=0, help="override the 200 time steps (profiling runs)")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the checkpointed and 8-per-cell measurements of the headline line")
    ap.add_argument("--config", type=int, default=1, help="1 = headline workload; 0, 2, 3, 4 = extra measurements")
    ap.add_argument("--iters", type=int, default=30, help="config 4: Adam iterations")
    ap.add_argument("--lr", type=float, default=1e-2, help="config 4: Adam learning rate (configured: 1e-2)")
    ap.add_argument("--controls", choices=["frame", "tied"], default="frame",
                    help="config 4: descend layer 0's controls (one control frame) or controls tied over all layers")
    ap.add_argument("--line-search", action="store_true",
                    help="config 4: wrap each Adam step in the reference optimiser's line search")
    ap.add_argument("--fd", action="store_true", help="config 1: adjoint vs central differences, 16 directions")
    ap.add_argument("--instances", type=int, default=48, help="config 3: number of batched instances")
    ap.add_argument("--fd-h", default="1e-3,1e-4,1e-5,1e-6,1e-7", help="--fd: central-difference steps")
    ap.add_argument("--next-rows", action="store_true",
                    help="time the mesh sampler and the surfacing against the reference's own code")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    global BRICK_CELLS, SORT_EVERY, DETERMINISTIC, SHUFFLE, REORDER
    if args.brick is not None:
        BRICK_CELLS = args.brick
    SORT_EVERY = args.sort_every
    DETERMINISTIC = args.deterministic
    SHUFFLE = args.shuffle
    REORDER = args.reorder
    if args.impl == "reference":
        return run_reference(args)
    if args.fd:
        return run_fd(args)
    if args.next_rows:
        return run_next_rows(args)
    if args.config == 0:
        return run_config0(args)
    if args.config == 2:
        return run_config2(args)
    if args.config == 3:
        return run_config3(args)
    if args.config == 4:
        return run_config4(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
