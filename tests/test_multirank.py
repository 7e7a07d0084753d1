"""The N > 1 path of bench.py on the CPU: two ranks over gloo (127.0.0.1)
meet at the timed region's barriers and combine their numbers as the bench
does with NCCL on GPUs — the slowest rank's time, the sum of the ranks' work
(replicas, no collective on the data path) — and the reference arm runs on
rank 0 only."""
import argparse
import datetime
import os
import socket

import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, port: int, queue) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=60))
    import bench
    world, r, _ = bench._dist()
    bench._barrier(world)
    mx, sm = bench._over_ranks([10.0 + r, 5.0 * r], [100.0 + r, 1.0], world)
    bench._barrier(world)
    queue.put((r, mx, sm))
    dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_add_their_work():
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(queue.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, [11.0, 5.0], [201.0, 2.0]), (1, [11.0, 5.0], [201.0, 2.0])]


def test_one_rank_is_the_identity():
    import bench
    assert bench._over_ranks([3.5], [7], 1) == ([3.5], [7.0])


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = argparse.Namespace(workload="multi_sector", cpu_seconds=1.0, warmup=1, steps=1)
    assert bench.run_reference(args) is None
    assert capsys.readouterr().out == ""
