"""The chunked encoder of streamed tensors, through the C ABI.

A streamed tensor (opts.stream_data) larger than one chunk of its residency
budget is encoded chunk by chunk: keys and a stable sort per chunk on the
GPU, a merge of the sorted runs on the host.  The result must be the
resident encoder's bit for bit (coordinates, values, blocks), with
duplicate coordinates in input order; the streamed MTTKRP and CP-ALS on it
must match the resident ones (1e-12 / 1e-10).
"""
import numpy as np
import pytest

from conftest import unique_coords

pytestmark = pytest.mark.gpu

DIMS = [3000, 2000, 90]


def _tensor(seed, nnz=300_000, dup=20_000):
    rng = np.random.default_rng(seed)
    cidx = unique_coords(rng, DIMS, nnz - dup, zipf=0.9)
    pick = rng.integers(0, nnz - dup, size=dup)
    cidx = np.concatenate([cidx, cidx[:, pick]], axis=1)
    perm = rng.permutation(cidx.shape[1])
    return np.ascontiguousarray(cidx[:, perm]), rng.random(cidx.shape[1])


def _opts(blco, residency):
    return blco.make_opts(stream_data=True, residency_bytes=residency)


@pytest.mark.parametrize("residency", [2 << 20, 5 << 20])
def test_chunked_streamed_encode_is_bit_identical(blco, residency):
    cidx, vals = _tensor(1)
    ref = blco.Tensor.encode(DIMS, cidx, vals, 40_000)
    t = blco.Tensor.encode(DIMS, cidx, vals, 40_000, opts=_opts(blco, residency))
    a, b = t.copy_out(), ref.copy_out()
    assert not a["resident"]
    assert np.array_equal(a["coords"], b["coords"])
    assert np.array_equal(a["vals"].view(np.uint64), b["vals"].view(np.uint64))
    assert np.array_equal(a["block_offsets"], b["block_offsets"])
    t.free()
    ref.free()


def test_chunked_streamed_encode_from_device_coo(blco):
    import torch
    cidx, vals = _tensor(2)
    ref = blco.Tensor.encode(DIMS, cidx, vals, 0)
    d_c = [torch.from_numpy(cidx[n].astype(np.int64)).cuda() for n in range(3)]
    d_v = torch.from_numpy(vals).cuda()
    t = blco.Tensor.encode_device(DIMS, d_c, d_v, 0, _opts(blco, 2 << 20))
    a, b = t.copy_out(), ref.copy_out()
    assert np.array_equal(a["coords"], b["coords"])
    assert np.array_equal(a["vals"].view(np.uint64), b["vals"].view(np.uint64))
    t.free()
    ref.free()


def test_chunked_streamed_mttkrp_and_cpals_match_resident(blco):
    import torch
    cidx, vals = _tensor(3)
    R = 8
    rng = np.random.default_rng(4)
    fs = [rng.random((d, R)) for d in DIMS]
    ref = blco.Tensor.encode(DIMS, cidx, vals, 50_000)
    t = blco.Tensor.encode(DIMS, cidx, vals, 50_000, opts=_opts(blco, 2 << 20))
    dev = [torch.from_numpy(f).cuda() for f in fs]
    for m in range(3):
        o1 = torch.zeros(DIMS[m], R, dtype=torch.float64, device="cuda")
        o2 = torch.zeros(DIMS[m], R, dtype=torch.float64, device="cuda")
        blco.mttkrp(ref, m, dev, o1)
        blco.mttkrp(t, m, dev, o2, _opts(blco, 2 << 20))
        torch.cuda.synchronize()
        x, y = o1.cpu().numpy(), o2.cpu().numpy()
        assert np.linalg.norm(x - y) <= 1e-12 * np.linalg.norm(x), m
    f1 = [f.copy() for f in fs]
    f2 = [f.copy() for f in fs]
    l1, l2 = np.ones(R), np.ones(R)
    _, fits1 = blco.cpals(ref, f1, l1, 6, 0.0)
    _, fits2 = blco.cpals(t, f2, l2, 6, 0.0, _opts(blco, 2 << 20))
    assert np.allclose(fits1, fits2, rtol=0, atol=1e-10)
    for a, b in zip(f1, f2):
        assert np.linalg.norm(a - b) <= 1e-9 * np.linalg.norm(a)
    t.free()
    ref.free()


def test_chunked_streamed_encode_rejects_bad_coordinate_in_late_chunk(blco):
    cidx, vals = _tensor(5)
    cidx = cidx.copy()
    cidx[1, -3] = DIMS[1]  # out of range, in the last chunk
    with pytest.raises(blco.BlcoError) as e:
        blco.Tensor.encode(DIMS, cidx, vals, 0, opts=_opts(blco, 2 << 20))
    assert e.value.status == blco.ERR_INVALID


def test_streamed_mixed_mttkrp_matches_resident(blco):
    """The mixed form on streamed blocks (4-byte values per block) against
    the resident mixed form: FP32 sums in another order, so 1e-5 normwise."""
    import torch
    cidx, vals = _tensor(6)
    R = 16
    rng = np.random.default_rng(7)
    fs = [torch.from_numpy(rng.random((d, R)).astype(np.float32)).cuda() for d in DIMS]
    ref = blco.Tensor.encode(DIMS, cidx, vals, 50_000)
    t = blco.Tensor.encode(DIMS, cidx, vals, 50_000, opts=_opts(blco, 2 << 20))
    for m in range(3):
        o1 = torch.zeros(DIMS[m], R, dtype=torch.float32, device="cuda")
        o2 = torch.zeros(DIMS[m], R, dtype=torch.float32, device="cuda")
        blco.mttkrp_ex(ref, m, fs, o1, blco.DTYPE_F32)
        blco.mttkrp_ex(t, m, fs, o2, blco.DTYPE_F32, _opts(blco, 2 << 20))
        torch.cuda.synchronize()
        x, y = o1.double().cpu().numpy(), o2.double().cpu().numpy()
        assert np.linalg.norm(x - y) <= 1e-5 * np.linalg.norm(x), m
    t.free()
    ref.free()


@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
def test_streamed_blocks_larger_than_the_budget(blco, dtype):
    """Blocks of 200k nonzeros under a 2 MiB budget: the ring copies
    budget-sized pieces of each block, and the MTTKRP equals the resident
    one (FP64 1e-12; the mixed forms stream 4-byte values into buffers sized
    for 8 and flush their own heavy-row sums per piece: 1e-5)."""
    import torch
    cidx, vals = _tensor(9)
    R = 8
    rng = np.random.default_rng(10)
    fs = [torch.from_numpy(rng.random((d, R))).cuda() for d in DIMS]
    tdt, code, tol = {"f64": (torch.float64, blco.DTYPE_F64, 1e-12), "f32": (torch.float32, blco.DTYPE_F32, 1e-5),
                      "bf16": (torch.bfloat16, blco.DTYPE_BF16, 1e-5)}[dtype]
    fs = [f.to(tdt) for f in fs]
    otype = torch.float64 if dtype == "f64" else torch.float32
    ref = blco.Tensor.encode(DIMS, cidx, vals, 200_000)
    t = blco.Tensor.encode(DIMS, cidx, vals, 200_000, opts=blco.make_opts(stream_data=True))
    for m in range(3):
        o1 = torch.zeros(DIMS[m], R, dtype=otype, device="cuda")
        o2 = torch.zeros(DIMS[m], R, dtype=otype, device="cuda")
        blco.mttkrp_ex(ref, m, fs, o1, code)
        blco.mttkrp_ex(t, m, fs, o2, code, _opts(blco, 2 << 20))
        torch.cuda.synchronize()
        x, y = o1.double().cpu().numpy(), o2.double().cpu().numpy()
        assert np.linalg.norm(x - y) <= tol * np.linalg.norm(x), m
    t.free()
    ref.free()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_streamed_cpals_under_a_budget_smaller_than_two_blocks(blco, precision):
    """A streamed CP-ALS plan whose budget leaves less than two blocks of
    200k nonzeros for the ring: pieces of blocks stream through it, the fits
    follow the resident plan's, and the plan's device bytes stay within the
    budget."""
    import torch
    cidx, vals = _tensor(11)
    R = 8
    rng = np.random.default_rng(12)
    fs0 = [rng.random((d, R)) for d in DIMS]
    prec = blco.PRECISION_FP64 if precision == "fp64" else blco.PRECISION_MIXED
    budget = 3 << 20
    ref = blco.Tensor.encode(DIMS, cidx, vals, 200_000)
    t = blco.Tensor.encode(DIMS, cidx, vals, 200_000, opts=blco.make_opts(stream_data=True))
    fits = []
    for tens, opts in ((ref, blco.make_opts(precision=prec)),
                       (t, blco.make_opts(stream_data=True, precision=prec, residency_bytes=budget))):
        dfs = [torch.from_numpy(f.copy()).cuda() for f in fs0]
        lam = torch.ones(R, dtype=torch.float64, device="cuda")
        plan = blco.CpalsPlan(tens, dfs, lam, opts)
        fits.append(np.array(plan.iterate(6, tol=-1.0)))
        if tens is t:
            used = plan.device_bytes()
            assert 0 < used <= budget, used
        plan.destroy()
    tol = 1e-10 if precision == "fp64" else 1e-6
    assert np.allclose(fits[0], fits[1], rtol=0, atol=tol), np.abs(fits[0] - fits[1]).max()
    t.free()
    ref.free()
