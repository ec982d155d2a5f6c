"""The N > 1 path of bench.py on CPU: replicas time their steps on their own
device and the job reports the slowest rank (all_reduce MAX, here over a
world-size-2 gloo group); the reference arm under torchrun runs on rank 0
alone and the other ranks exit without work."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t = bench.max_over_ranks_of(dist, 1.0 + rank)          # rank 1 is the slow one
    v = bench.replica_throughput(1000, 10, world, t)
    q.put((rank, t, v))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [t for _, t, _ in out] == [2.0, 2.0]
    # 2 replicas x 1000 cells x 10 steps in the slowest rank's 2 s
    assert all(abs(v - 1e-2) < 1e-12 for _, _, v in out)


def test_max_over_ranks_single_process():
    assert bench.max_over_ranks_of(None, 3.5) == 3.5


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3",
           "--cells", "32", "32", "16"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("ABL 32x32x16 cells") and d["cpu_baseline"]["cpu_model"]
