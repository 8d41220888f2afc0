"""Multi-GPU runs of bench.py are replicas only: every rank runs its own
product on its own GPU, the step time is the maximum over the ranks and the
value counts the work of all of them (weak scaling); no data crosses between
ranks. These tests run that plumbing as two gloo ranks on the CPU, and check
that the reference arm runs on rank 0 alone."""
from __future__ import annotations

import os
import socket
from types import SimpleNamespace

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    from datetime import timedelta
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        r, local, w = bench.dist_env()
        # rank r "took" 10 + 5 r ms: the job's step time is the slowest rank's
        t_ms = bench.replica_max(dist, 10.0 + 5.0 * rank, "cpu")
        dist.barrier()
        q.put((rank, r, local, w, t_ms, bench.replica_tflops(w, 2e12, t_ms * 1e-3)))
    finally:
        dist.destroy_process_group()


def test_replica_time_is_the_slowest_rank_and_value_counts_all():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    for p in procs:
        if p.is_alive():
            p.kill()
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in procs)
    for rank, (r, env_rank, local, w, t_ms, value) in enumerate(got):
        assert (r, env_rank, local, w) == (rank, rank, rank, 2)
        assert t_ms == 15.0
        assert value == pytest.approx(2 * 2e12 / 15e-3 / 1e12)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.replica_max(None, 3.25, "cpu") == 3.25
    assert bench.replica_tflops(1, 1e12, 0.5) == pytest.approx(2.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    """Under torchrun every rank but 0 exits at once without work."""
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    def must_not_run(*a, **k):
        raise AssertionError("the reference ran on rank 1")

    monkeypatch.setattr(bench, "cpu_reference_run", must_not_run)
    assert bench.run_reference(SimpleNamespace(steps=2, warmup=1, gpus=2)) is None


def _rank_leaving(rank: int, world: int, port: int, q) -> None:
    """Rank 1 leaves after joining the group, before the collective; rank 0
    must get an error from its next collective within the group's timeout."""
    from datetime import timedelta
    import time
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=5))
    if rank == 1:
        os._exit(0)  # gone without a word, between steps
    t0 = time.monotonic()
    try:
        bench.replica_max(dist, 1.0, "cpu")
        q.put(("no error", time.monotonic() - t0))
    except Exception as e:  # the peer's departure surfaces as an error, not a hang
        q.put(("error", time.monotonic() - t0, type(e).__name__))
    q.close()
    q.join_thread()  # the result is in the pipe before the process ends
    os._exit(0)


def test_departed_rank_ends_the_next_collective_with_an_error():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_leaving, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(30)
        if p.is_alive():
            p.kill()
    assert got[0] == "error", got
    assert got[1] < 60.0, got
