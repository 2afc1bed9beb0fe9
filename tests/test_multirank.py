"""The N > 1 path of bench.py on CPU: one replica per rank, the timed region taken as the
slowest rank's (max over ranks), the whole-job rate over all ranks, and the reference arm
run by rank 0 alone.  gloo, world size 2, rendezvous on 127.0.0.1; no GPU."""
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


def _rank_main(rank, world, port, times, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        total = bench.max_over_ranks(times[rank], dist, "cpu")
        out.put((rank, total, bench.whole_job_rate(world, 10, total)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    import torch.multiprocessing as tmp
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    times = [1234.5, 987.25]
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [1234.5, 1234.5]          # every rank sees the slowest rank
    assert res[0][2] == pytest.approx(2 * 10 / 1.2345)     # all ranks' solves over that time


def test_one_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(42.0, None) == 42.0
    assert bench.whole_job_rate(1, 5, 500.0) == pytest.approx(10.0)


def test_reference_arm_other_ranks_exit_quietly():
    """Under torchrun the reference arm runs on rank 0 only; rank 1 exits 0 printing nothing."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
