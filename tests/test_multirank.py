"""The multi-rank plumbing of bench.py on the CPU: two gloo ranks agree on the
max over ranks (the timing rule for N GPUs) and pass the barrier, and the
reference arm launched by torchrun prints one line from rank 0 while rank 1
exits 0 without work.  The replicas themselves exchange nothing (the path does
not shard), so this is the whole of the N > 1 logic."""
import json
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


def _rank(rank, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench

    class Args:
        impl = "reference"

    world, r, local = bench.dist_init(Args)
    m = bench.reduce_max(1.5 + rank, world, Args)
    bench.barrier(world)
    q.put((world, r, local, m))
    dist.destroy_process_group()


def test_max_over_ranks_and_barrier():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in ps)
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(2, 0, 0, 2.5), (2, 1, 1, 2.5)]


def test_reference_arm_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--nx", "6", "--nz", "4", "--cpu-seconds", "0.2"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["e2e"]["value"] == d["value"]
