"""GPU test of the allocation-free encoder (blco_encode_device_noalloc).

That entry point is for callers that cannot allocate device memory while
they encode (their device memory belongs to another allocator, or they must
not call cudaMalloc); its sort scratch is a fixed array inside the library.
It must produce exactly the encoding of the allocating entry point
(blco_encode), on consecutive calls that reuse the same scratch.  The
encoding is integer/byte work, so the comparison is bit-exact.

This file is collected last on purpose (tests/test_zz_*), so a run that
stops at the first failure has run every other test before it.
"""
import numpy as np
import pytest

from conftest import unique_coords

pytestmark = pytest.mark.gpu


def _noalloc(blco, dims, cidx, vals):
    import torch
    d_c = [torch.from_numpy(cidx[n].astype(np.int64)).cuda() for n in range(len(dims))]
    d_v = torch.from_numpy(vals).cuda()
    out_c = torch.empty(len(vals), dtype=torch.int64, device="cuda")
    out_v = torch.empty(len(vals), dtype=torch.float64, device="cuda")
    blco.encode_device_noalloc(dims, d_c, d_v, out_c, out_v)
    torch.cuda.synchronize()
    return out_c.cpu().numpy().view(np.uint64), out_v.cpu().numpy()


def test_noalloc_encode_matches_allocating_encode_twice(blco):
    rng = np.random.default_rng(2024)
    cases = [
        ([200_000, 150_000, 3_000], 1_500_000, 1.1),  # first call
        ([3_000, 70, 900, 40], 400_000, None),        # second call, different shape and size
    ]
    for dims, nnz, zipf in cases:
        cidx = unique_coords(rng, dims, nnz, zipf)
        vals = rng.lognormal(0.0, 1.0, nnz)
        c_na, v_na = _noalloc(blco, dims, cidx, vals)
        ref = blco.Tensor.encode(dims, cidx, vals).copy_out()
        assert np.array_equal(c_na, ref["coords"])
        assert np.array_equal(v_na, ref["vals"])


def test_noalloc_at_the_maximum_size_matches_the_oracle(blco):
    """Exactly BLCO_NOALLOC_MAX_NNZ nonzeros (the scratch layout's limit),
    skewed coordinates over four modes, against the oracle's encoder."""
    import pyoracle as po
    rng = np.random.default_rng(77)
    dims = [150_000, 90_000, 4_000, 37]
    nnz = int(blco.NOALLOC_MAX_NNZ)
    cidx = unique_coords(rng, dims, nnz, 1.0)
    vals = rng.standard_normal(nnz)
    c_na, v_na = _noalloc(blco, dims, cidx, vals)
    enc = po.blco_encode(dims, cidx, vals)
    assert np.array_equal(c_na, enc["coords"])
    assert np.array_equal(v_na.view(np.uint64), enc["vals"].view(np.uint64))


def test_noalloc_allocates_no_device_memory(blco):
    """After a first call (the library's set-up on this device), an encode
    leaves the device's free memory unchanged: inputs and outputs are the
    caller's, the scratch is the library's fixed array."""
    import torch
    rng = np.random.default_rng(78)
    dims = [40_000, 30_000, 500]
    nnz = 1_000_000
    cidx = unique_coords(rng, dims, nnz, 0.8)
    vals = rng.random(nnz)
    d_c = [torch.from_numpy(cidx[n].astype(np.int64)).cuda() for n in range(3)]
    d_v = torch.from_numpy(vals).cuda()
    out_c = torch.empty(nnz, dtype=torch.int64, device="cuda")
    out_v = torch.empty(nnz, dtype=torch.float64, device="cuda")
    blco.encode_device_noalloc(dims, d_c, d_v, out_c, out_v)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        blco.encode_device_noalloc(dims, d_c, d_v, out_c, out_v)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    ref = blco.Tensor.encode(dims, cidx, vals).copy_out()
    assert np.array_equal(out_c.cpu().numpy().view(np.uint64), ref["coords"])


def test_noalloc_limits_and_errors(blco):
    import torch
    dims = [10, 10, 10]
    small = [torch.zeros(4, dtype=torch.int64, device="cuda") for _ in range(3)]
    vals = torch.zeros(4, dtype=torch.float64, device="cuda")
    out_c = torch.empty(4, dtype=torch.int64, device="cuda")
    out_v = torch.empty(4, dtype=torch.float64, device="cuda")
    # size above the stated maximum: rejected before any device work
    L = blco.lib()
    import ctypes
    ptrs = (ctypes.c_void_p * 3)(*[int(c.data_ptr()) for c in small])
    d = np.array(dims, dtype=np.uint64)
    st = L.blco_encode_device_noalloc(3, d.ctypes.data, blco.NOALLOC_MAX_NNZ + 1, ptrs, int(vals.data_ptr()),
                                      int(out_c.data_ptr()), int(out_v.data_ptr()), None)
    assert st == blco.ERR_UNSUPPORTED
    assert "BLCO_NOALLOC_MAX_NNZ" in L.blco_last_error().decode()
    # a coordinate outside its mode: reported, and the next call is clean
    bad = [torch.tensor([0, 1, 2, 10], dtype=torch.int64, device="cuda")] + small[1:]
    with pytest.raises(blco.BlcoError) as e:
        blco.encode_device_noalloc(dims, bad, vals, out_c, out_v)
    assert e.value.status == blco.ERR_INVALID
    ok = [torch.tensor([0, 1, 2, 9], dtype=torch.int64, device="cuda")] + small[1:]
    blco.encode_device_noalloc(dims, ok, vals, out_c, out_v)
