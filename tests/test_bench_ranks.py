"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2): the
job's time is the maximum over ranks, and under torchrun the reference arm
runs on rank 0 alone, prints one JSON line, and the other rank exits 0
without output. Replicas only: no collective touches the data path."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    out[rank] = (bench.max_over_ranks(1.0 + rank, world, "cpu"), bench.max_over_ranks(5.0 - rank, world, "cpu"))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, free_port(), out), nprocs=2, start_method="spawn", join=True)
    assert out[0] == out[1] == (2.0, 5.0)


def test_reference_arm_under_torchrun():
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("reference build not present")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(free_port()), "bench.py", "--impl", "reference", "--steps", "1",
           "--warmup", "0"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1  # rank 0 only
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["e2e"]["value"] == d["value"]
