"""Multi-GPU row: `bench.py --gpus N` runs N independent replicas (the path
has no exchange step, so no collective on the data path).  The host logic
around them -- max-over-ranks timing, the whole-job value, rank 0 alone
printing and running the reference arm -- runs here as world-size-2 gloo
ranks on the CPU."""
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, ws, port, local_ms, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import bench
        t_max, value = bench.whole_job_value(local_ms[rank], ws, 1000, torch.device("cpu"))
        out.put((rank, t_max, value))
    finally:
        dist.destroy_process_group()


def test_whole_job_value_takes_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 2000
    local_ms = [40.0, 50.0]
    ps = [ctx.Process(target=_rank, args=(r, 2, port, local_ms, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    # both ranks see the slower time; the value counts both ranks' pairs
    assert [g[1] for g in got] == [50.0, 50.0]
    assert all(abs(g[2] - 2 * 1000 / 0.05) < 1e-6 for g in got)


def test_single_rank_value():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    t_max, value = bench.whole_job_value(20.0, 1, 500, torch.device("cpu"))
    assert t_max == 20.0 and abs(value - 500 / 0.02) < 1e-6


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=120, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
