"""The benchmark's multi-rank host logic on CPU: two gloo ranks, each with its
own instance, reduce their timings with max-over-ranks and report the
whole-job value; the reference arm does no work on ranks other than 0."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [12.0, 30.0][rank]  # rank 1 is the slow one
        ms_max = bench.max_over_ranks(ms, world)
        bench.barrier(world)
        out[rank] = (ms_max, bench.whole_job_value(1000.0, 5, world, ms_max))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_weak_scaling_value():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(world):
        ms_max, value = res[r]
        assert ms_max == 30.0
        assert value == pytest.approx(1000.0 * 5 * 2 / 0.030)


def test_reference_arm_skips_nonzero_ranks(monkeypatch):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        steps, warmup, ppc_root, dt, rollout_steps = 1, 3, 2, 0.0, 0

    assert bench.run_reference(A()) == 0


def test_instance_sharding_covers_every_instance_once():
    import scenes

    work = [sc.n * sc.steps for sc in scenes.batch_scenes(48)]
    for world in (1, 2, 3, 8):
        shards = [bench.shard_instances(work, world, r) for r in range(world)]
        flat = sorted(i for sh in shards for i in sh)
        assert flat == list(range(len(work)))
        loads = [sum(work[i] for i in sh) for sh in shards]
        # longest-processing-time-first: no rank exceeds the mean by more than one instance
        assert max(loads) - sum(work) / world <= max(work)
