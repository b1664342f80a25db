"""bench.py's multi-rank logic on the host: world-size-2 gloo process groups
(127.0.0.1), no GPU.  Every rank advances its own replica; the timing rule is
the maximum over ranks and the whole-job rate counts every rank's zones;
only rank 0 runs and prints the reference arm."""
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

import bench

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        ms, e2e = 10.0 + 5.0 * rank, 3.0 - rank   # rank 1 is slower on the device, rank 0 end to end
        mx = bench.max_over_ranks([ms, e2e], world)
        dist.barrier()
        q.put((rank, mx, bench.whole_job_rates(world, 1000, 20, mx[0], mx[1])))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, rates in res:
        assert mx == [15.0, 3.0]                      # the slowest rank's times, on every rank
        assert rates == (2 * 1000 * 20 / 15e-3, 2 * 1000 * 20 / 3.0)
    assert sorted(r for r, _, _ in res) == [0, 1]


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks([1.5, 2.5], 1) == [1.5, 2.5]
    assert bench.whole_job_rates(1, 100, 10, 2.0, 0.5) == (100 * 10 / 2e-3, 100 * 10 / 0.5)


def test_reference_arm_runs_on_rank_0_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_reference_arm_splits_the_grid_like_an_mpi_run():
    """The reference arm times the workload's own grid split into one block
    per core, with the least block surface (least ghost work per zone)."""
    assert bench.decompose((192, 192, 128), 16) == ((2, 4, 2), (96, 48, 64))
    assert bench.decompose((192, 192, 128), 8) == ((2, 2, 2), (96, 96, 64))
    assert bench.decompose((192, 192, 128), 64) == ((4, 4, 4), (48, 48, 32))
    counts, block = bench.decompose((192, 192, 128), 12)
    assert counts[0] * counts[1] * counts[2] == 12 and all(n % c == 0 for n, c in zip((192, 192, 128), counts))
