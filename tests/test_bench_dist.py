"""The benchmark's multi-rank plumbing on CPU (world size 2, gloo).

With N GPUs `bench.py` runs N replicas (one rank per GPU, each decomposing
its own tensor, no collective on the data path) and reports the maximum of
the per-rank device times.  These tests run that host logic with two gloo
ranks: the max-over-ranks reduction, and the reference arm under torchrun,
where rank 0 alone times the reference CPU MTTKRP and the other rank exits
0 without work.
"""
import json
import os
import socket
import subprocess
import sys

import torch.distributed as tdist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import bench
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = bench.max_over_ranks(10.0 * (rank + 1), tdist, device="cpu")
        tdist.barrier()
    finally:
        tdist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(2, port, out), nprocs=2, start_method="spawn")
        assert dict(out) == {0: 20.0, 1: 20.0}


def test_max_over_ranks_without_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5


def test_reference_arm_under_torchrun_two_ranks(tmp_path):
    """rank 0 prints one JSON line with impl=reference; rank 1 prints none."""
    port = _free_port()
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = "2"
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--ref-sample", "20000"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line.get("unavailable") or (line["value"] > 0 and line["cpu_baseline"]["kind"] == "reference")
