"""The N > 1 path of bench.py on the CPU (gloo, world size 2): replicas time their own
batches and the job reports the slowest rank (max over ranks) with weak scaling; the
reference arm under torchrun runs on rank 0 alone and prints one JSON line, the other rank
exits 0 without work."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle as O
from conftest import ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, queue):
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}")
    slow = bench.max_over_ranks(1.5 * (rank + 1), world, torch.device("cpu"))
    queue.put((rank, slow, bench.weak_value(world, 8, 3, slow)))
    dist.destroy_process_group()


def test_max_over_ranks_with_gloo():
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(queue.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [3.0, 3.0]
    assert got[0][2] == pytest.approx(2 * 8 * 3 / 3.0)


@pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built")
def test_reference_arm_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--mesh", "30"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
