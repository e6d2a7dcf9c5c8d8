"""The N > 1 plumbing of bench.py, on CPU with two gloo ranks: the timing
aggregation takes the slowest rank's time, the whole-job rate counts every
rank's units, and under torchrun the reference arm prints exactly one line
(rank 0) while the other rank exits 0 without work."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
        rate = bench.whole_job_rate(1000, world, t)
        out.put((rank, t, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, rate in res:
        assert t == 15.0                      # the slowest rank's time on every rank
        assert rate == pytest.approx(2 * 1000 / 0.015)


def test_single_rank_helpers():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.whole_job_rate(500, 1, 2.0) == pytest.approx(250000.0)


def test_reference_arm_under_torchrun_prints_one_line():
    from oracle import pyoracle as po
    if po.ref_host() is None:
        pytest.skip("oracle/_ref not built")
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py",
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
           "--points", "3000", "--queries", "2000"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["n_gpus"] == 2
    assert out["value"] > 0 and out["e2e"]["h2d_bytes_per_step"] == 0
    assert out["cpu_baseline"]["kind"] == "reference"
    # the arm describes its workload with exactly the product arm's config
    import bench
    assert out["config"] == bench.bench_config(3000, 2000, 2)
    # every step answers all the queries; the build is reported once
    assert out["build_ms"] > 0 and "all 2000 queries" in out["reference_step"]
