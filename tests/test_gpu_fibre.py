"""GPU parity of the compressed-fibre MTTKRP schedule (kernel id 4).

FP64: against the reference's sequential COO MTTKRP (golden fixtures made by
the reference build) and the oracle, normwise and elementwise relative error
<= 1e-12 (the only difference is the order of FP64 sums).  Mixed forms:
against the oracle in FP64 on the same rounded inputs, normwise <= 1e-5.

The cases cover what the copy's layout has to get right: fibres that span
many walker ranges (one heavy fibre), only single-nonzero fibres (no fibred
stream), only repeated fibres (no loose stream), stream lengths that are not
a multiple of the 4-nonzero step or of the 256-position chunk, 3 to 5 modes,
ranks on every lane count, and the fallback for ranks with no fibre kernel.
"""
import numpy as np
import pytest

import pyoracle as po
from conftest import formula_factors, golden_case, golden_index, unique_coords

pytestmark = pytest.mark.gpu

FIB = 4
TOL = 1e-12
CASES = [c["name"] for c in golden_index()["cases"]]


def _close(out, ref, tol=TOL):
    den = np.linalg.norm(ref)
    err = np.linalg.norm(out - ref) / (den if den > 0 else 1.0)
    assert err <= tol, err
    mask = np.abs(ref) > 0
    if mask.any():
        rel = np.abs(out[mask] - ref[mask]) / np.abs(ref[mask])
        assert rel.max() <= 10 * tol, rel.max()
    assert np.all(out[~mask] == 0.0)
    return err


def _round_bf16(a):
    a32 = np.ascontiguousarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def _dev(fs, dtype=None):
    import torch
    out = [torch.from_numpy(np.ascontiguousarray(f)).cuda() for f in fs]
    return [o.to(dtype) for o in out] if dtype is not None else out


def _run(blco, t, m, fs, dim, R, opts, dtype=None, code=None):
    import torch
    if dtype is None:
        out = torch.zeros(dim, R, dtype=torch.float64, device="cuda")
        blco.mttkrp(t, m, fs, out, opts)
    else:
        out = torch.zeros(dim, R, dtype=torch.float32, device="cuda")
        blco.mttkrp_ex(t, m, fs, out, code, opts)
    torch.cuda.synchronize()
    return out.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("name", CASES)
def test_fibre_matches_reference_golden(blco, name):
    g = golden_case(name)
    dims = [int(d) for d in g["dims"]]
    R = int(g["rank"])
    t = blco.Tensor.encode(g["dims"], g["cidx"], g["vals"], int(g["max_block_size"]))
    fs = _dev(formula_factors(dims, R))
    for m in range(len(dims)):
        _close(_run(blco, t, m, fs, dims[m], R, blco.make_opts(kernel=FIB)), g[f"mttkrp{m}"])


@pytest.mark.parametrize("rank", [1, 4, 6, 8, 16, 32, 64, 100])
def test_fibre_ranks_fp64(blco, rank):
    """Ranks 4..64 (2..32 lanes) take the fibre kernel, the others fall back."""
    rng = np.random.default_rng(rank)
    dims = [300, 2000, 40]
    cidx = unique_coords(rng, dims, 30_000, zipf=1.0)
    vals = rng.random(30_000)
    t = blco.Tensor.encode(dims, cidx, vals)
    fs_h = [rng.random((d, rank)) for d in dims]
    fs = _dev(fs_h)
    for m in range(3):
        _close(_run(blco, t, m, fs, dims[m], rank, blco.make_opts(kernel=FIB)), po.mttkrp_coo(cidx, vals, fs_h, m))


@pytest.mark.parametrize("nmodes,dims", [(3, [5000, 70, 300]), (4, [400, 30, 2000, 9]), (5, [64, 33, 17, 300, 5])])
@pytest.mark.parametrize("zipf", [None, 1.1])
def test_fibre_orders(blco, nmodes, dims, zipf):
    rng = np.random.default_rng(nmodes)
    nnz = 40_003  # not a multiple of the 4-nonzero step or of a 256-position chunk
    cidx = unique_coords(rng, dims, nnz, zipf=zipf)
    vals = rng.random(nnz)
    t = blco.Tensor.encode(dims, cidx, vals, 4096)
    R = 16
    fs_h = [rng.random((d, R)) for d in dims]
    fs = _dev(fs_h)
    for m in range(nmodes):
        _close(_run(blco, t, m, fs, dims[m], R, blco.make_opts(kernel=FIB)), po.mttkrp_coo(cidx, vals, fs_h, m))


def test_fibre_one_heavy_fibre(blco):
    """Most nonzeros in one (row, fibre-mode index) fibre, long enough to be
    split over many walker ranges, plus a sprinkle elsewhere."""
    rng = np.random.default_rng(7)
    dims = [50, 300_000, 20]
    heavy = 250_000
    j = rng.choice(dims[1], size=heavy, replace=False)
    c_heavy = np.stack([np.full(heavy, 3), j, np.full(heavy, 5)]).astype(np.uint64)
    rest = unique_coords(rng, dims, 5_000)
    keep = ~((rest[0] == 3) & (rest[2] == 5))
    cidx = np.concatenate([c_heavy, rest[:, keep]], axis=1)
    vals = rng.random(cidx.shape[1]) - 0.5  # mixed signs
    t = blco.Tensor.encode(dims, cidx, vals)
    R = 32
    fs_h = [rng.random((d, R)) - 0.5 for d in dims]
    fs = _dev(fs_h)
    for m in range(3):
        ref = po.mttkrp_coo(cidx, vals, fs_h, m)
        out = _run(blco, t, m, fs, dims[m], R, blco.make_opts(kernel=FIB))
        err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
        assert err <= TOL, (m, err)


def test_fibre_only_singletons_and_only_repeats(blco):
    R = 8
    rng = np.random.default_rng(11)
    # every nonzero has its own mode-0 index, so every fibre of every mode
    # holds one nonzero: only the loose stream is used
    dims = [1000, 1000, 1000]
    nnz = 999
    perm = rng.permutation(1000)[:nnz]
    cidx = np.stack([np.arange(nnz), rng.integers(0, 1000, nnz), perm]).astype(np.uint64)
    vals = rng.random(nnz)
    t = blco.Tensor.encode(dims, cidx, vals)
    fs_h = [rng.random((d, R)) for d in dims]
    fs = _dev(fs_h)
    for m in range(3):
        _close(_run(blco, t, m, fs, dims[m], R, blco.make_opts(kernel=FIB)), po.mttkrp_coo(cidx, vals, fs_h, m))
    # dense 2 x 3 x 2 block repeated: every fibre has two or more nonzeros
    dims2 = [2, 3, 2]
    cidx2 = np.array(np.unravel_index(np.arange(12), dims2), dtype=np.uint64)
    vals2 = rng.random(12)
    t2 = blco.Tensor.encode(dims2, cidx2, vals2)
    fs2_h = [rng.random((d, R)) for d in dims2]
    fs2 = _dev(fs2_h)
    for m in range(3):
        _close(_run(blco, t2, m, fs2, dims2[m], R, blco.make_opts(kernel=FIB)), po.mttkrp_coo(cidx2, vals2, fs2_h, m))


@pytest.mark.parametrize("nnz", [1, 2, 3, 5, 257])
def test_fibre_tiny(blco, nnz):
    rng = np.random.default_rng(nnz)
    dims = [17, 5, 13]
    cidx = unique_coords(rng, dims, nnz)
    vals = rng.random(nnz)
    t = blco.Tensor.encode(dims, cidx, vals)
    R = 16
    fs_h = [rng.random((d, R)) for d in dims]
    fs = _dev(fs_h)
    for m in range(3):
        _close(_run(blco, t, m, fs, dims[m], R, blco.make_opts(kernel=FIB)), po.mttkrp_coo(cidx, vals, fs_h, m))


@pytest.mark.parametrize("dtype", ["f32", "bf16"])
@pytest.mark.parametrize("rank", [8, 16, 32, 64])
def test_fibre_mixed(blco, dtype, rank):
    import torch
    rng = np.random.default_rng(100 + rank)
    dims = [20_000, 5_000, 300]
    nnz = 200_000
    cidx = unique_coords(rng, dims, nnz, zipf=1.1)
    vals = rng.lognormal(0.0, 1.0, nnz)
    t = blco.Tensor.encode(dims, cidx, vals)
    fs = [rng.random((d, rank)) for d in dims]
    if dtype == "f32":
        fr = [f.astype(np.float32) for f in fs]
        dev = _dev(fr)
        code = blco.DTYPE_F32
    else:
        fr = [_round_bf16(f) for f in fs]
        dev = _dev(fr, torch.bfloat16)
        code = blco.DTYPE_BF16
    v32 = vals.astype(np.float32).astype(np.float64)
    for m in range(3):
        ref = po.mttkrp_coo(cidx, v32, [f.astype(np.float64) for f in fr], m)
        o = _run(blco, t, m, dev, dims[m], rank, blco.make_opts(kernel=FIB), dtype=True, code=code)
        err = np.linalg.norm(o - ref) / np.linalg.norm(ref)
        assert err <= 1e-5, (m, err)


def test_fibre_matches_auto_on_skewed(blco):
    """Zipf(1.1) with heavy rows: kernel 4 and the automatic rule agree."""
    rng = np.random.default_rng(42)
    dims = [200_000, 200_000, 25_000]
    nnz = 400_000
    cidx = unique_coords(rng, dims, nnz, zipf=1.1)
    vals = rng.lognormal(0.0, 1.0, nnz)
    t = blco.Tensor.encode(dims, cidx, vals)
    R = 32
    fs_h = [rng.random((d, R)) for d in dims]
    fs = _dev(fs_h)
    for m in range(3):
        ref = po.mttkrp_coo(cidx, vals, fs_h, m)
        _close(_run(blco, t, m, fs, dims[m], R, blco.make_opts(kernel=FIB)), ref)
        _close(_run(blco, t, m, fs, dims[m], R, blco.make_opts(kernel=10)), ref)
