"""The multi-process path of bench.py on the CPU (gloo, world size 2): independent replicas
whose times are reduced to the slowest rank's, and a whole-job rate over all replicas; the
reference arm runs on rank 0 only."""
import os
import socket
import sys
from datetime import timedelta

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    try:
        local = [10.0 + 5.0 * rank, 3.0 - rank]  # rank 1 is slower on the first, faster on the second
        out = bench.slowest_rank_ms(local, "cpu")
        rate = bench.replica_rate(1000, world, 4, out[0])
        q.put((rank, bench.dist_env(), out, rate))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, env, out, rate in got:
        assert env == (rank, 2, rank)
        assert out == [15.0, 3.0]
        assert rate == pytest.approx(1000 * 2 * 4 / 15e-3 / 1e9)


def test_single_process_is_unchanged():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.slowest_rank_ms([2.5, 7.0], "cpu") == [2.5, 7.0]
    assert bench.replica_rate(135005697, 1, 200, 1000.0) == pytest.approx(27.0011394)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        gpus, steps, warmup = 2, 1, 1

    assert bench.reference_arm(Args()) is None
    assert capsys.readouterr().out == ""
