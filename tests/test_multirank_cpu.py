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


def test_clock_sampler_keeps_the_timed_window_and_reads_throttle_reasons():
    """bench.ClockSampler keeps the nvidia-smi samples that arrived during the
    timed region (or, for a region shorter than the sampling interval, the
    first one after it began) and reports the throttle reasons active there."""
    import bench

    class FakeProc:
        def terminate(self):
            pass

        def wait(self, timeout=None):
            pass

    def row(mhz, power, cap, thermal="Not Active"):
        return f"0, {mhz}, 1965, {power}, 0x0, Not Active, Not Active, {thermal}, {cap}"

    c = bench.ClockSampler(0)
    c.proc = FakeProc()
    c.lines = [(0.5, row(345, 90.0, "Not Active")),            # idle, before the region
               (1.05, row(1965, 600.0, "Active")),             # inside
               (1.15, row(1950, 640.0, "Not Active")),         # inside
               (2.5, row(1965, 100.0, "Not Active", "Active"))]  # long after
    c.window = [1.0, 1.2]
    ck = c.stop()
    assert ck["samples"] == 2 and ck["sm_mhz"] == (1965 + 1950) / 2
    assert ck["reasons"] == ["sw_power_cap"] and ck["power_w_max"] == 640.0
    c.window = [2.0, 2.05]  # shorter than the interval: the first sample after it began
    ck = c.stop()
    assert ck["samples"] == 1 and ck["reasons"] == ["sw_thermal_slowdown"]
    c.lines = []
    assert c.stop() is None
