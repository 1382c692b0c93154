"""The replica plumbing of bench.py on two CPU ranks (gloo, 127.0.0.1).

On N GPUs every rank renders the same workload (replicas, weak scaling);
ranks meet at a barrier before and after the timed steps, the step time is
the maximum over ranks, and only rank 0 prints.  These tests run that logic
with a gloo process group on the host, with no GPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    assert bench._dist_setup() == (world, rank, rank)
    bench._barrier(world)
    out[rank] = bench._max_over_ranks(10.0 * (rank + 1), world)
    bench._barrier(world)
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_max_over_ranks_and_barrier_on_gloo(world):
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    assert dict(out) == {r: 10.0 * world for r in range(world)}


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import sys
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        steps, warmup = 3, 3
    bench.run_reference(Args())  # rank 1: no work, no line
    assert capsys.readouterr().out == ""
