"""Multi-GPU replicas, host side: two gloo ranks on CPU exercise the
barrier, the max over ranks and the deterministic work partition that the
bench uses under torchrun (one process per GPU, no data-path collective)."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

import sfntt
from sfntt import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, q) -> None:
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    r = replicas.Replicas(backend="gloo", timeout_s=60)
    try:
        assert r.active and r.rank == rank and r.world == world
        r.barrier()
        step_ms = 10.0 + 5.0 * rank  # the slowest rank sets the job time
        mx = r.max(step_ms)
        items = sfntt.uneven_workload(64, seed=2024)
        mine = replicas.partition(items, world, rank, replicas.lde_work)
        r.barrier()
        q.put((rank, mx, replicas.job_time_per_unit(mx, world), mine))
    finally:
        r.close()


def test_two_gloo_ranks_barrier_max_and_partition():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, mx, per_unit, _ in got:
        assert mx == 15.0 and per_unit == 7.5
    parts = [set(m) for *_, m in got]
    assert parts[0].isdisjoint(parts[1]) and parts[0] | parts[1] == set(range(64))
    # the same assignment computed locally (no communication needed)
    items = sfntt.uneven_workload(64, seed=2024)
    assert [replicas.partition(items, world, r, replicas.lde_work) for r in range(world)] == [sorted(p) for p in parts]
    loads = [sum(replicas.lde_work(items[i]) for i in p) for p in parts]
    assert max(loads) / min(loads) < 1.2  # balanced by estimated work


def test_single_process_is_a_no_op():
    r = replicas.Replicas(backend="gloo")
    assert not r.active and r.world == 1
    r.barrier()
    assert r.max(3.5) == 3.5
    assert replicas.partition(list(range(5)), 1, 0) == [0, 1, 2, 3, 4]
    with pytest.raises(ValueError):
        replicas.partition([1], 2, 2)
