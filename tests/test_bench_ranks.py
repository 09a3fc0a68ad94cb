"""The multi-rank plumbing of bench.py on CPU: world_size-2 `gloo` ranks.

Multi-GPU runs of the bench are independent replicas (one engine per rank,
no data-path collective); the ranks only meet at barriers and for the max of
their device times. These tests run that reduction with two gloo ranks and
check that the reference arm's non-zero ranks exit without work."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 * (rank + 1), "cpu")
        e2e = bench.max_over_ranks(3.0 if rank == 0 else 7.5, "cpu")
        q.put((rank, ms, e2e, bench.job_rate(1000.0, world, ms)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, e2e, rate in got:
        assert ms == 20.0 and e2e == 7.5  # every rank sees the slowest rank's time
        assert rate == pytest.approx(1000.0 * 2 / 0.020)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(4.25, "cpu") == 4.25
    assert bench.job_rate(500.0, 1, 4.0) == pytest.approx(500.0 / 0.004)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip() == ""
