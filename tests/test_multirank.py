"""The N > 1 path of bench.py on CPU: two gloo ranks.

bench.py runs one replica of the workload per GPU (transposes are
independent: no collective on the data path) and reports the whole job: the
bytes of all ranks over the slowest rank's time.  These tests run that host
logic -- the max-over-ranks all-reduce and the aggregate -- on two processes
with the gloo backend, and check that the reference arm's other ranks exit
without work.
"""
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, times, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        m = bench.max_over_ranks(times[rank], dist, world, device="cpu")
        v = bench.aggregate_gbs(10**9, world, m)
        dist.barrier()
    finally:
        dist.destroy_process_group()
    q.put((rank, m, v))


@pytest.mark.parametrize("times", [(12.5, 20.0), (30.0, 7.25)])
def test_two_ranks_take_the_max_and_aggregate(times):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    slowest = max(times)
    for rank, m, v in out:
        assert m == slowest
        assert abs(v - 2 * 10**9 / (slowest / 1e3) / 1e9) < 1e-9


def test_one_rank_is_the_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, 1) == 3.5
    assert bench.aggregate_gbs(2 * 10**9, 1, 1000.0) == 2.0


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "3"],
                       capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
