"""The N > 1 path of bench.py on CPU: two gloo ranks (replicas, no data
collective).  Checks the max-over-ranks timing, the whole-job rate and that
the reference arm runs on rank 0 only."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    r, w, local = bench.dist_setup("gloo", timeout_s=60)
    ms_local = 100.0 + 50.0 * r            # the slower rank defines the step time
    ms = bench.max_over_ranks(ms_local, w, device="cpu")
    bench.barrier(w, sync_cuda=False)
    rate = bench.whole_job_rate(6.98e11, w, ms)
    q.put((r, w, ms, rate))
    import torch
    torch.distributed.destroy_process_group()


def test_two_gloo_ranks_take_max_time():
    import socket
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    for r, w, ms, rate in res:
        assert w == 2 and ms == 150.0
        assert rate == pytest.approx(6.98e11 * 2 / 0.150 / 1e9)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
