"""The multi-rank plumbing of bench.py on the CPU: two gloo ranks on
127.0.0.1 take the max and the sum over ranks and meet at the barrier, as
the replicas of `bench.py --gpus N` do over NCCL (the timed value is all
ranks' rows over the slowest rank's time); the reference arm runs on rank 0
alone and the other ranks leave without output."""
import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    mx = bench.reduce_max(10.0 * (rank + 1), world)
    sm = bench.reduce_sum(float(rank + 1), world)
    bench.barrier(world)
    out.put((rank, mx, sm))
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_and_meet():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, 20.0, 3.0), (1, 20.0, 3.0)]


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    args = type("A", (), {"workload": "select", "steps": 1, "warmup": 0})()
    assert bench.run_reference(args) is None
    assert capsys.readouterr().out == ""
