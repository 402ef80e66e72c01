"""The N > 1 bench path on the CPU: every rank is an independent replica, the
job is timed as the slowest rank (max over ranks through the process group),
and throughput counts every rank's voxels.  Two gloo ranks stand in for two
GPUs; the reference arm's extra ranks leave without work."""
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


def _rank(rank, world, port, times, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(times[rank], dist, device="cpu")
        out.put((rank, t, bench.job_gvox_per_s(world, 1024 ** 3, t * 1e-3)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    times = [11.5, 13.25]   # ms per step on each rank
    procs = [ctx.Process(target=_rank, args=(r, 2, port, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, t, value in got:
        assert t == 13.25
        assert value == pytest.approx(2 * 1024 ** 3 / 13.25e-3 / 1e9)


def test_one_rank_is_a_no_op():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(7.0, None) == 7.0
    assert bench.job_gvox_per_s(1, 10 ** 9, 1.0) == 1.0


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
