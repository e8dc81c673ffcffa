"""CPU tests of the multi-GPU (replica) host logic of bench.py with the gloo backend:
every rank takes the same collective steps, the timing is the max over ranks and the
whole-job rate counts every rank's work."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 10.0 + 5.0 * rank
        mx = bench.reduce_max(local_ms, dist, "cpu")
        rate = bench.whole_job_rate(16, mx, world)
        dist.barrier()
        q.put((rank, mx, rate))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_replica_timing_is_max_over_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + world * 7 + os.getpid() % 100
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    want_ms = 10.0 + 5.0 * (world - 1)
    for rank, mx, rate in got:
        assert mx == want_ms
        assert abs(rate - world * 16 / (want_ms / 1e3)) < 1e-6


def test_reference_arm_runs_on_rank0_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")

    class A:
        level, steps, warmup, gpus = 30, 1, 0, 2

    assert bench.run_reference(A()) is None
    assert capsys.readouterr().out == ""
