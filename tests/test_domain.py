"""Spatial domain decomposition (domain.py) on gloo CPU ranks: a scene drifting
across the slab boundaries is stepped forward by 2 and 3 ranks, each holding
only its x slab of the grid (plus ghost planes) and its own particles, with the
halo reduce after P2G, the halo broadcast before G2P and particle migration
every step.  The gathered particles must equal the single-domain FP64 oracle
(the CPU restatement of the reference's ForwardTimeStep) to rounding.

The per-rank stages below are a small numpy restatement of the same
ForwardTimeStep (ForwardSimulation.cpp:126-157) that works on a slab of the
grid; they are test infrastructure, as the oracle is."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

FLT_EPS = 1.1920928955078125e-07
OFFS = np.array([(i, j, k) for i in range(4) for j in range(4) for k in range(4)])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _bsp(q):
    a = np.abs(q)
    return np.where(a < 1, 0.5 * a ** 3 - a * a + 2.0 / 3.0, np.where(a < 2, (2 - a) ** 3 / 6.0, 0.0))


def _pk(F, lam, mu):
    U, _, Vt = np.linalg.svd(F)
    R = U @ Vt
    J = np.maximum(np.linalg.det(F), 1e-6)
    return 2 * mu[:, None, None] * (F - R) + (lam * (J - 1) * J)[:, None, None] * np.linalg.inv(F).transpose(0, 2, 1)


def _stencil(x, sc, p0, p1):
    """Local flat node index (planes [p0, p1)), offsets d = x_g - x and weights
    of the 64 stencil nodes of each particle; nodes outside the grid masked."""
    dims = np.asarray(sc.dims)
    base = np.floor((x - sc.min_point) / sc.dx).astype(np.int64) - 1
    ii = base[:, None, :] + OFFS[None]
    valid = np.all((ii >= 0) & (ii < dims), axis=2)
    assert np.all((ii[..., 0][valid] >= p0) & (ii[..., 0][valid] < p1)), "stencil outside the local planes"
    d = sc.min_point + ii * sc.dx - x[:, None, :]
    w = np.prod(_bsp(d / sc.dx), axis=2) * valid
    flat = ((ii[..., 0] - p0) * dims[1] + ii[..., 1]) * dims[2] + ii[..., 2]
    return np.where(valid, flat, 0), d, w


def _p2g(P, sc, p0, p1):
    """Particle-to-grid on planes [p0, p1): returns (planes, ny, nz, 4) of (p, m)."""
    nloc = (p1 - p0) * sc.dims[1] * sc.dims[2]
    flat, d, w = _stencil(P["x"], sc, p0, p1)
    Fe = P["F"] + P["dFc"]
    G = (-3.0 / sc.dx ** 2 * sc.dt * P["vol"])[:, None, None] * (_pk(Fe, P["lam"], P["mu"]) @ Fe.transpose(0, 2, 1)) \
        + P["m"][:, None, None] * P["C"]
    mvd = P["m"][:, None] * P["v"] * (1 - sc.dt * sc.drag)
    mom = w[..., None] * (mvd[:, None, :] + np.einsum("pab,pnb->pna", G, d))
    grid = np.zeros((nloc, 4))
    np.add.at(grid[:, 3], flat.ravel(), (w * P["m"][:, None]).ravel())
    for a in range(3):
        np.add.at(grid[:, a], flat.ravel(), mom[..., a].ravel())
    return grid.reshape(p1 - p0, sc.dims[1], sc.dims[2], 4)


def _g_op(grid, sc):
    m = grid[..., 3]
    occ = np.abs(m) > FLT_EPS
    v = np.zeros(grid.shape[:-1] + (3,))
    for a in range(3):
        v[..., a] = np.where(occ, grid[..., a] / np.where(occ, m, 1.0) + sc.dt * sc.f_ext[a], 0.0)
    return v


def _g2p(P, v, sc, p0, p1):
    flat, d, w = _stencil(P["x"], sc, p0, p1)
    vg = v.reshape(-1, 3)[flat]
    vn = np.sum(w[..., None] * vg, axis=1)
    Cn = 3.0 / sc.dx ** 2 * np.einsum("pn,pna,pnb->pab", w, vg, d)
    Fe = P["F"] + P["dFc"]
    Fn = (np.eye(3)[None] + sc.dt * Cn) @ Fe
    out = dict(P)
    out["F"] = (1 - sc.smoothing) * Fn + sc.smoothing * P["F"]
    out["x"] = P["x"] + sc.dt * vn
    out["v"] = vn
    out["C"] = Cn
    return out


def _scene():
    import scenes

    sc = scenes.small_scene(seed=41, res=24, radius=0.25, steps=12, v_std=30.0, drag=0.1, smoothing=0.05,
                            f_ext=(0.0, -2.0, 0.0), dt=2e-4)
    sc.v[:, 0] += 400.0  # about one cell of drift along x over the rollout, across the slab faces
    from oracle.lib import OracleGraph

    sc.vol = OracleGraph(sc, "f64").calc_volumes()
    return sc


def _worker(rank, world, port, out):
    import sys

    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (here, os.path.join(here, "a-differentiable-material-point-method-for-shape-morphing_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    from domain import SlabDecomposition

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc = _scene()
        dec = SlabDecomposition(sc.dims[0], world, rank)
        cell = lambda x: torch.from_numpy(np.floor((x[:, 0] - sc.min_point[0]) / sc.dx).astype(np.int64))
        allp = {"id": np.arange(sc.n), "x": sc.x, "v": sc.v, "F": sc.F, "C": sc.C, "dFc": sc.dFc, "m": sc.m,
                "vol": sc.vol, "lam": sc.lam, "mu": sc.mu}
        mine = (dec.owner_of_cell(cell(sc.x)) == rank).numpy()
        P = {k: np.ascontiguousarray(a[mine]) for k, a in allp.items()}
        moved = 0
        for _ in range(sc.steps):
            grid = torch.from_numpy(_p2g(P, sc, dec.p0, dec.p1))
            dec.halo_reduce(grid)
            v = torch.from_numpy(_g_op(grid.numpy(), sc))
            dec.halo_broadcast(v)
            P = _g2p(P, v.numpy(), sc, dec.p0, dec.p1)
            n_before = len(P["id"])
            T = dec.migrate(cell(P["x"]), {k: torch.from_numpy(np.ascontiguousarray(a)) for k, a in P.items()})
            P = {k: t.numpy() for k, t in T.items()}
            moved += int(np.sum(~np.isin(P["id"], P["id"][:n_before]))) if n_before else 0
        gathered = [None] * world
        dist.all_gather_object(gathered, ({k: P[k] for k in ("id", "x", "v", "F", "C")}, moved))
        if rank == 0:
            out["parts"] = gathered
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_decomposition_matches_single_domain(world):
    from oracle.lib import OracleGraph

    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        parts = out["parts"]
    sc = _scene()
    ids = np.concatenate([p[0]["id"] for p in parts])
    assert np.array_equal(np.sort(ids), np.arange(sc.n)), "every particle on exactly one rank"
    assert sum(p[1] for p in parts) > 0, "no particle migrated"
    order = np.argsort(ids)
    o = OracleGraph(sc, "f64")
    L = sc.steps + 1
    o.setup(L, sc.dt, sc.drag, sc.f_ext, sc.smoothing)
    o.forward(0)
    for k in ("x", "v", "F", "C"):
        got = np.concatenate([p[0][k] for p in parts])[order]
        want = o.get(L - 1, k)
        assert np.max(np.abs(got - want)) <= 1e-10 * np.max(np.abs(want)), k
