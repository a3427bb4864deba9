"""Multi-process plumbing on CPU (gloo, world size 2): the N > 1 path of bench.py.

* fractura_b200.dist: every rank sees the slowest rank's time and the summed
  work; the whole-job rate counts every rank's frames over the slowest time.
* bench.py --impl reference under torch.distributed.run: rank 0 alone runs the
  CPU reference arm and prints one JSON line; the other rank exits 0 without work.
"""
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


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from fractura_b200 import dist as fd
        fd.barrier()
        slowest = fd.max_over_ranks(100.0 + 25.0 * rank)   # per-rank timed milliseconds
        total = fd.sum_over_ranks(1 + rank)
        rate = fd.whole_job_rate(1e9, 4, world, slowest)
        out.put((rank, slowest, total, rate, fd.active()))
        fd.barrier()
    finally:
        dist.destroy_process_group()


def test_gloo_world2_reductions():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(_worker, args=(2, port, q), nprocs=2, join=True, start_method="spawn")
    got = sorted(q.get() for _ in range(2))
    for rank, slowest, total, rate, active in got:
        assert active
        assert slowest == 125.0          # both ranks see the slower rank
        assert total == 3.0
        assert rate == pytest.approx(1e9 * 4 * 2 / 0.125)


def test_whole_job_rate_single_process():
    from fractura_b200 import dist as fd
    assert not fd.active()
    assert fd.max_over_ranks(7.0) == 7.0
    assert fd.whole_job_rate(2.0, 3, 1, 1000.0) == pytest.approx(6.0)
    with pytest.raises(ValueError):
        fd.whole_job_rate(1.0, 1, 1, 0.0)


def test_reference_arm_under_torchrun_world2():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--workload", "cfg1", "--gpus", "2", "--steps", "1", "--warmup", "3"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["value"] > 0
