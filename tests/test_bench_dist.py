"""The benchmark's multi-rank plumbing on CPU (world size 2, gloo).

With N GPUs `bench.py` shards one tensor over N ranks (one rank per GPU,
each owning a contiguous 1/N of the nonzeros; each mode's MTTKRP summed over
the ranks by an all-reduce) and reports the maximum of the per-rank device
times.  These tests run that host logic with two gloo ranks: the sharding
and the exchange (each rank's MTTKRP of its share, from the oracle, summed
over the ranks, equals the whole tensor's), the max-over-ranks and per-rank
reductions, and the reference arm under torchrun, where rank 0 alone times
the reference CPU path and the other rank exits 0 without work.
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


def _shard_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import torch
    import bench
    import pyoracle as po
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(3)
        dims = [40, 30, 20]
        n = 1001
        cidx = np.stack([rng.integers(0, d, n) for d in dims])
        vals = rng.random(n)
        X = dict(dims=dims, cidx=[torch.from_numpy(c) for c in cidx], vals=torch.from_numpy(vals))
        sh = bench.shard_slice(X, world, rank)
        fs = [np.random.default_rng(4 + m).random((d, 5)) for m, d in enumerate(dims)]
        mine = np.stack([c.numpy() for c in sh["cidx"]]).astype(np.uint64)
        got = []
        for m in range(3):
            part = torch.from_numpy(po.mttkrp_coo(mine, sh["vals"].numpy(), fs, m))
            tdist.all_reduce(part)
            got.append(part.numpy())
        want = [po.mttkrp_coo(cidx.astype(np.uint64), vals, fs, m) for m in range(3)]
        per = bench.all_ranks(float(sh["hi"] - sh["lo"]), tdist, device="cpu")
        out[rank] = dict(ok=all(np.allclose(a, b, rtol=1e-12, atol=0) for a, b in zip(got, want)),
                         norm=abs(sh["norm_sq"] - float((vals ** 2).sum())) <= 1e-12 * float((vals ** 2).sum()),
                         range=(sh["lo"], sh["hi"]), per=per)
        tdist.barrier()
    finally:
        tdist.destroy_process_group()


def test_sharded_path_two_gloo_ranks():
    """The bench's sharding (contiguous ranges that partition the nonzeros,
    the whole tensor's norm on every rank) and exchange: the sum over the
    ranks of each rank's MTTKRP equals the whole tensor's MTTKRP."""
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.start_processes(_shard_worker, args=(2, port, out), nprocs=2, start_method="spawn")
        r = dict(out)
    assert r[0]["ok"] and r[1]["ok"] and r[0]["norm"] and r[1]["norm"]
    assert r[0]["range"] == (0, 500) and r[1]["range"] == (500, 1001)
    assert r[0]["per"] == [500.0, 501.0] == r[1]["per"]


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
