"""Config 3's multi-GPU layout -- instance sharding, no data-path collective --
run as two ranks.  Each rank takes its shard of the instances
(bench.shard_instances: longest processing time first), evaluates them as one
batch (dmpm_batch_*), and the ranks exchange their per-instance losses and
control gradients and the max-over-ranks reduction bench.py times with, over
gloo on the host.  Every instance must match the same instances evaluated as
one batch in this process, to the summation-order noise of float atomics.

The two ranks are processes on the same GPU: nothing on the device waits on
another rank (the only exchange is on the host, after each rank's kernels have
finished), so this runs the sharded path end to end on one GPU."""
import multiprocessing as mp
import os
import pickle
import socket

import numpy as np
import pytest

from tests.helpers import relerr
from tests.test_gpu_batch import _batch, _scenes

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "a-differentiable-material-point-method-for-shape-morphing_b200")
WORLD = 2


def _rank(rank, world, port, scs, out_path):
    """One rank (a spawned process): its shard as one batch, then the exchange."""
    import sys

    for p in (REPO, PKG):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        import bench
        from tests.test_gpu_batch import _batch as make_batch

        mine = bench.shard_instances([sc.n * sc.steps for sc in scs], world, rank)
        with make_batch([scs[i] for i in mine]) as b:
            b.setup()
            losses = b.gradient()
            grads = [b.control_grad(k) for k in range(len(mine))]
        reduced = bench.max_over_ranks(float(rank + 1), world)
        got = [None] * world
        dist.all_gather_object(got, {"mine": list(mine), "losses": [float(v) for v in losses], "grads": grads,
                                     "max": reduced})
        if rank == 0:
            with open(out_path, "wb") as f:
                pickle.dump(got, f)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_batch_matches_one_batch(gpu_ready, tmp_path):
    scs = _scenes()
    with _batch(scs) as b:
        b.setup()
        losses = b.gradient()
        grads = [b.control_grad(i) for i in range(len(scs))]
    out = str(tmp_path / "ranks.pkl")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, WORLD, port, scs, out)) for r in range(WORLD)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert [p.exitcode for p in procs] == [0] * WORLD
    with open(out, "rb") as f:
        got = pickle.load(f)
    assert sorted(i for r in got for i in r["mine"]) == list(range(len(scs)))
    assert all(len(r["mine"]) >= 1 for r in got)
    for r in got:
        assert r["max"] == float(WORLD)
        for k, i in enumerate(r["mine"]):
            assert abs(r["losses"][k] - losses[i]) <= 1e-6 * abs(losses[i]), i
            assert relerr(r["grads"][k], grads[i]) < 1e-4, i
