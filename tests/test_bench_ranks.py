"""The bench's multi-rank path on CPU (gloo, world size 2): the job time is the
slowest rank's, the value counts every rank's particles, and under torchrun
the reference arm prints one line from rank 0 while the other rank exits 0."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t = bench.max_over_ranks(10.0 + rank * 5.0)
    v = bench.job_rate(world, 1000, 4, t)
    out.put((rank, t, v))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, v in got:
        assert t == 15.0                      # the slowest rank's time on every rank
        assert v == 2 * 1000 * 4 / 15.0       # both ranks' particles


def test_single_process_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.5) == 3.5


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_prints_once():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--workload", "c1", "--steps", "2", "--warmup", "3", "--budget-s", "5"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=540)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 2
    assert d["e2e"]["h2d_bytes_per_step"] == 0
