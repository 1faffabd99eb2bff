"""Batched CP-ALS (blco_batch_*) through the C ABI.

Every tensor of a batch must follow the same iterations as a CP-ALS of that
tensor alone (blco_cpals, itself checked against the oracle's restatement
of cpals_blco_dev, src/cpd_gpu.cu:21-242): per-iteration fits within 1e-10
absolute, the same iteration count under a tolerance, factors within 1e-9
relative (Frobenius).  Both sides sum the MTTKRP with FP64 atomics in
different orders, so they agree to rounding, not bitwise.  Two tensors are
also checked against the oracle directly.
"""
import numpy as np
import pytest
import torch

import pyoracle as po
from conftest import unique_coords

pytestmark = pytest.mark.gpu

# (dims, nnz, rank, zipf)
CASES = [
    ([300, 200, 100], 5_000, 8, 0.0),
    ([2000, 1500, 40], 30_000, 16, 0.8),
    ([60, 50, 40, 30], 8_000, 5, 0.0),
    ([100, 90, 80, 7, 3], 6_000, 4, 0.0),
    ([5000, 30], 4_000, 12, 1.0),
    ([800, 700, 600], 20_000, 32, 0.0),
    ([400, 30, 20], 3_000, 33, 0.5),
    ([1200, 900, 500], 25_000, 64, 0.0),
    ([50, 40, 30], 500, 1, 0.0),
    ([20000, 3000, 100], 40_000, 16, 1.1),
    ([7, 6, 5], 120, 3, 0.0),
    ([64, 64, 64, 64], 10_000, 24, 0.0),
]


def _make(seed=0, cases=CASES):
    rng = np.random.default_rng(seed)
    out = []
    for dims, nnz, R, z in cases:
        cidx = unique_coords(rng, dims, nnz, zipf=z)
        vals = rng.random(nnz)
        fs = [rng.random((d, R)) for d in dims]
        out.append((dims, cidx, vals, R, fs))
    return out


def _alone(blco, items, iters, tol):
    res = []
    for dims, cidx, vals, R, fs in items:
        t = blco.Tensor.encode(dims, cidx, vals)
        f = [x.copy() for x in fs]
        lam = np.ones(R)
        _, fits = blco.cpals(t, f, lam, iters, tol)
        res.append((fits, f, lam))
        t.free()
    return res


def _batched(blco, items, iters, tol, opts=None, split=None, time_mttkrp=False):
    ts, fs, ls = [], [], []
    for dims, cidx, vals, R, f0 in items:
        ts.append(blco.Tensor.encode(dims, cidx, vals))
        fs.append([torch.from_numpy(x.copy()).cuda() for x in f0])
        ls.append(torch.ones(R, dtype=torch.float64, device="cuda"))
    b = blco.Batch(ts, fs, ls, tol=tol, opts=opts)
    parts = split or [iters]
    fits, done = [], None
    for k in parts:
        fk, done = b.iterate(k)
        fits.append(fk)
        if time_mttkrp:
            assert b.mttkrp_ms() > 0.0
    b.destroy()
    for t in ts:
        t.free()
    return np.concatenate(fits), done, [[x.cpu().numpy() for x in f] for f in fs], [l.cpu().numpy() for l in ls]


def _compare(alone, fits, done, fs, ls):
    for t, (afits, af, al) in enumerate(alone):
        n = len(afits)
        assert done[t] == n, (t, done[t], n)
        assert np.allclose(fits[:n, t], afits, rtol=0, atol=1e-10), (t, np.max(np.abs(fits[:n, t] - afits)))
        # a converged tensor repeats its last fit
        assert np.all(fits[n:, t] == fits[n - 1, t])
        for a, b in zip(fs[t], af):
            assert np.linalg.norm(a - b) <= 1e-9 * np.linalg.norm(b), t
        assert np.allclose(ls[t], al, rtol=1e-9), t


def test_batch_matches_single_tensor_cpals(blco):
    items = _make(0)
    alone = _alone(blco, items, 12, 0.0)
    fits, done, fs, ls = _batched(blco, items, 12, 0.0)
    assert fits.shape == (12, len(items))
    _compare(alone, fits, done, fs, ls)


def test_batch_convergence_per_tensor(blco):
    """With a tolerance, tensors stop at different iterations; each stops
    where blco_cpals stops."""
    items = _make(1)
    alone = _alone(blco, items, 40, 1e-4)
    lens = {len(a[0]) for a in alone}
    assert len(lens) > 1  # the batch really is uneven
    fits, done, fs, ls = _batched(blco, items, 40, 1e-4)
    _compare(alone, fits, done, fs, ls)


def test_batch_graph_and_split_calls(blco):
    """The same run without the CUDA graph and split over three calls."""
    items = _make(2, CASES[:6])
    alone = _alone(blco, items, 10, 0.0)
    fits, done, fs, ls = _batched(blco, items, 10, 0.0, opts=blco.make_opts(verbose=-1), split=[3, 0, 7])
    _compare(alone, fits, done, fs, ls)
    fits, done, fs, ls = _batched(blco, items, 10, 0.0, split=[1, 4, 5])
    _compare(alone, fits, done, fs, ls)


def test_batch_mttkrp_timing_leaves_the_state(blco):
    """Timing one sweep's MTTKRP launches between calls (blco_batch_mttkrp_ms)
    leaves the run as it was: the same fits and factors as blco_cpals."""
    items = _make(4, CASES[:6])
    alone = _alone(blco, items, 9, 0.0)
    fits, done, fs, ls = _batched(blco, items, 9, 0.0, split=[2, 3, 4], time_mttkrp=True)
    _compare(alone, fits, done, fs, ls)


def test_batch_matches_oracle(blco):
    items = _make(3, [CASES[0], CASES[2]])
    fits, done, fs, ls = _batched(blco, items, 8, 0.0)
    for t, (dims, cidx, vals, R, f0) in enumerate(items):
        enc = po.blco_encode(dims, cidx, vals)
        fo = [x.copy() for x in f0]
        lo = np.ones(R)
        fits_o = po.cpals(dims, enc, fo, lo, 8, 0.0)
        assert np.allclose(fits[:, t], fits_o, rtol=0, atol=1e-10)
        for a, b in zip(fs[t], fo):
            assert np.linalg.norm(a - b) <= 1e-9 * np.linalg.norm(b)


def test_batch_many_tensors_one_launch(blco):
    """256 small tensors: the sweep's MTTKRP for a mode slot is one launch
    whatever the batch size (launch count per sweep independent of T)."""
    rng = np.random.default_rng(9)
    cases = []
    for _ in range(256):
        dims = [int(x) for x in rng.integers(20, 400, size=3)]
        nnz = int(min(np.prod(dims) // 2, rng.integers(50, 3000)))
        cases.append((dims, nnz, int(rng.choice([8, 16, 32])), 0.0))
    items = _make(4, cases)
    counts = []
    for sub in (items[:8], items):
        ts, fs, ls = [], [], []
        for dims, cidx, vals, R, f0 in sub:
            ts.append(blco.Tensor.encode(dims, cidx, vals))
            fs.append([torch.from_numpy(x.copy()).cuda() for x in f0])
            ls.append(torch.ones(R, dtype=torch.float64, device="cuda"))
        b = blco.Batch(ts, fs, ls, tol=0.0)
        blco.lib().blco_launch_count(1)
        b.iterate(2)
        counts.append(blco.lib().blco_launch_count(1))
        b.destroy()
        for t in ts:
            t.free()
    assert counts[0] == counts[1]
    alone = _alone(blco, items[:16], 5, 0.0)
    fits, done, fs, ls = _batched(blco, items[:16], 5, 0.0)
    _compare(alone, fits, done, fs, ls)


def test_batch_errors(blco):
    rng = np.random.default_rng(5)
    dims = [30, 20, 10]
    cidx = unique_coords(rng, dims, 200)
    t = blco.Tensor.encode(dims, cidx, rng.random(200))
    f = [torch.rand(d, 65, dtype=torch.float64, device="cuda") for d in dims]
    lam = torch.ones(65, dtype=torch.float64, device="cuda")
    with pytest.raises(blco.BlcoError) as e:
        blco.Batch([t], [f], [lam])
    assert e.value.status == blco.ERR_UNSUPPORTED
    with pytest.raises(blco.BlcoError) as e:
        blco.Batch([], [], [])
    assert e.value.status == blco.ERR_INVALID
    ts = blco.Tensor.encode(dims, cidx, rng.random(200), max_block_size=64, opts=blco.make_opts(stream_data=1))
    f = [torch.rand(d, 8, dtype=torch.float64, device="cuda") for d in dims]
    lam = torch.ones(8, dtype=torch.float64, device="cuda")
    with pytest.raises(blco.BlcoError) as e:
        blco.Batch([ts], [f], [lam])
    assert e.value.status == blco.ERR_UNSUPPORTED
    b = blco.Batch([t], [f], [lam])
    with pytest.raises(blco.BlcoError):
        b.iterate(5000)
    b.destroy()
    t.free()
    ts.free()
