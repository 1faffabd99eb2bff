"""Sharded CP-ALS: ranks hold shares of one tensor's nonzeros and sum every
mode's MTTKRP over the ranks (blco_cpals_plan_set_reduce).

CPU (gloo, 2 ranks): the torch.distributed reduce hook sums a buffer over
the ranks.  GPU (gloo, 2 processes on one GPU, the exchange through host
copies, so no kernel waits on another process): the sharded CP-ALS follows
the single-process one on the whole tensor (FP64 fits 1e-10, factors
1e-9; mixed form 1e-6).
"""
import ctypes
import os
import socket
import sys

import numpy as np
import pytest
import torch.distributed as tdist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _cpu_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch
    from conftest import load_package
    blco = load_package()
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        buf = np.arange(10, dtype=np.float64) * (rank + 1)
        keep = torch.from_numpy(buf)

        def view(ptr, count, dtype):
            assert ptr == buf.ctypes.data and count == 10 and dtype == blco.DTYPE_F64
            return keep

        fn = blco.dist_reduce(tdist, view=view)
        fn(buf.ctypes.data, 10, blco.DTYPE_F64, None)
        out[rank] = buf.tolist()
    finally:
        tdist.destroy_process_group()


def test_dist_reduce_sums_over_two_gloo_ranks():
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.start_processes(_cpu_worker, args=(2, port, out), nprocs=2, start_method="spawn")
        want = (np.arange(10) * 3.0).tolist()
        assert out[0] == want and out[1] == want


DIMS = [2000, 1500, 80]


def _tensor():
    from conftest import unique_coords
    rng = np.random.default_rng(8)
    cidx = unique_coords(rng, DIMS, 60_000, zipf=0.9)
    vals = rng.random(cidx.shape[1])
    R = 8
    fs = [rng.random((d, R)) for d in DIMS]
    return cidx, vals, fs


def _gpu_worker(rank, world, port, precision, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch
    from conftest import load_package
    blco = load_package()
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cidx, vals, fs = _tensor()
        mine = np.arange(cidx.shape[1]) % world == rank  # any partition of the nonzeros
        t = blco.Tensor.encode(DIMS, np.ascontiguousarray(cidx[:, mine]), vals[mine])
        d_f = [torch.from_numpy(f).cuda() for f in fs]
        lam = torch.ones(fs[0].shape[1], dtype=torch.float64, device="cuda")
        plan = blco.CpalsPlan(t, d_f, lam, blco.make_opts(precision=precision))
        nsq = torch.tensor([float(np.sum(vals[mine] ** 2))], dtype=torch.float64)
        tdist.all_reduce(nsq)
        plan.set_norm_sq(nsq.item())
        plan.set_reduce(blco.dist_reduce(tdist, via_host=True))
        fits = plan.iterate(6, tol=-1.0)
        torch.cuda.synchronize()
        out[rank] = dict(fits=fits, f=[x.cpu().numpy() for x in d_f], lam=lam.cpu().numpy())
        plan.destroy()
        t.free()
    finally:
        tdist.destroy_process_group()


def _single(blco, precision):
    import torch
    cidx, vals, fs = _tensor()
    t = blco.Tensor.encode(DIMS, cidx, vals)
    d_f = [torch.from_numpy(f).cuda() for f in fs]
    lam = torch.ones(fs[0].shape[1], dtype=torch.float64, device="cuda")
    plan = blco.CpalsPlan(t, d_f, lam, blco.make_opts(precision=precision))
    fits = plan.iterate(6, tol=-1.0)
    torch.cuda.synchronize()
    res = dict(fits=fits, f=[x.cpu().numpy() for x in d_f], lam=lam.cpu().numpy())
    plan.destroy()
    t.free()
    return res


@pytest.mark.gpu
@pytest.mark.parametrize("mixed", [False, True])
def test_sharded_cpals_matches_single_process(blco, mixed):
    precision = blco.PRECISION_MIXED if mixed else blco.PRECISION_FP64
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.start_processes(_gpu_worker, args=(2, port, precision, out), nprocs=2, start_method="spawn")
        r0, r1 = dict(out[0]), dict(out[1])
    # every rank takes the same steps
    assert r0["fits"] == r1["fits"]
    for a, b in zip(r0["f"], r1["f"]):
        assert np.array_equal(a, b)
    ref = _single(blco, precision)
    tol = 1e-6 if mixed else 1e-10
    assert np.allclose(r0["fits"], ref["fits"], rtol=0, atol=tol)
    if not mixed:
        for a, b in zip(r0["f"], ref["f"]):
            assert np.linalg.norm(a - b) <= 1e-9 * np.linalg.norm(b)
