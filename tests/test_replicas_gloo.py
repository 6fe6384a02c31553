"""The replica plumbing of bench.py with two gloo ranks on the CPU.

bench.py --gpus N runs N independent replicas (one process per GPU); the only
communication is the barrier and the maximum of the timed milliseconds over
the ranks, from which the whole-job throughput counts every rank's cells.
"""

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms_local = [120.0, 150.0][rank]  # rank 1 is the slow one
        value, ms = bench.replica_throughput(3 * 1000 * 10, ms_local, dist, world)
        dist.barrier()
        out.put((rank, value, ms))
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(out.get(timeout=10) for _ in range(2))
    for rank, value, ms in res:
        assert ms == 150.0
        assert value == pytest.approx(2 * 3 * 1000 * 10 / 0.150 / 1e6)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = type("A", (), dict(steps=1, warmup=0, p=5, gpus=2))()
    bench.run_reference(args)  # returns at once, without work or output
    assert capsys.readouterr().out == ""
