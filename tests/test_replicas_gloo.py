"""Host logic of `bench.py --gpus N` (replicas only: every rank runs the same workload on
its own GPU, with no collective in the step) on two CPU ranks over gloo: the timed region
is the slowest rank's (a max-reduction every rank takes part in), the whole-job value is
N x one rank's leaf updates over that time, and the reference arm runs on rank 0 alone
(the other ranks return without work)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank            # rank 1 is the slow one
        m = bench.max_over_ranks(ms, dist, "cpu")
        out.put((rank, m, bench.replica_throughput(world, 3_000_000, m)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_throughput_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [m for _, m, _ in res] == [15.0, 15.0]
    assert all(v == pytest.approx(2 * 3_000_000 / 0.015) for _, _, v in res)


def test_max_over_ranks_without_process_group():
    assert bench.max_over_ranks(12.5, None, "cpu") == 12.5
    assert bench.replica_throughput(1, 1000, 1.0) == pytest.approx(1e6)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")
    a = type("A", (), {})()   # no attributes: a rank other than 0 must not look at them
    assert bench.run_reference(a) is None
    assert capsys.readouterr().out == ""
