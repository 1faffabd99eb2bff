"""GPU parity of the 128-bit-key path (the reference's cpd128 build,
gen_blcotensor_host<unsigned __int128>, include/blco.hpp:196-331) through
the C ABI.

Encoder: bit-exact against the w128_* fixtures made by the reference and
against the oracle's restatement on random tensors (blocks, block
coordinates, fields, values).  MTTKRP: within 1e-12 relative of the
reference's COO MTTKRP (fixtures) and of the oracle's (random, all inputs
positive, so elementwise).  CP-ALS: per-iteration fits within 1e-10 of the
oracle's cpals_blco_dev restatement with the same explicit factors.
"""
import os

import numpy as np
import pytest

import pyoracle as po
from conftest import formula_factors, golden_case, golden_index, unique_coords_wide

pytestmark = pytest.mark.gpu

WIDE = [c["name"] for c in golden_index()["wide_cases"]]


def _torch():
    import torch
    return torch


def _check_encoding(t, enc):
    o = t.copy_out()
    assert np.array_equal(o["coords"], enc["coords"])
    assert np.array_equal(o["vals"].view(np.uint64), np.asarray(enc["vals"]).view(np.uint64))
    assert o["block_count"] == len(enc["block_offsets"]) - 1
    assert np.array_equal(o["block_offsets"], enc["block_offsets"])
    assert np.array_equal(o["block_coords"], np.asarray(enc["block_coords"]).reshape(o["block_count"], -1))
    assert o["mode_masks"] == [int(x) for x in enc["mode_masks"]]
    assert o["mode_pos"] == [int(x) for x in enc["mode_pos"]]
    return o


@pytest.mark.parametrize("name", WIDE)
def test_wide_encoder_matches_reference_golden(blco, name):
    g = golden_case(name)
    dims = [int(d) for d in g["dims"]]
    t = blco.Tensor.encode(dims, g["cidx"], g["vals"], int(g["max_block_size"]))
    enc = dict(coords=g["coords"], vals=g["out_vals"], block_offsets=g["block_offsets"],
               block_coords=g["block_coords"], mode_masks=g["mode_masks"], mode_pos=g["mode_pos"])
    o = _check_encoding(t, enc)
    ref = po.blco_encode128(dims, g["cidx"], g["vals"], int(g["max_block_size"]))
    assert o["alto_masks"] == [int(x) for x in ref["alto_masks_lo"]]
    assert o["alto_masks_hi"] == [int(x) for x in ref["alto_masks_hi"]]
    assert o["alto_bits"] > 64
    t.free()


@pytest.mark.parametrize("dims,nnz,B", [
    ([1 << 20, 1 << 20, 1 << 20, 16387], 200_000, 1000),    # 75 bits
    ([(1 << 32) - 1, 1 << 31, 1 << 30, 3], 100_000, 0),      # 95 bits, above what the reference runs
    ([7, 9, 1 << 30, 1 << 30, 3000], 150_000, 1),            # 79 bits, one nonzero per block
    ([(1 << 32) - 1] * 4, 120_000, 777),                     # 128 bits
    ([1 << 14] * 5, 300_000, 4096),                          # 70 bits
])
def test_wide_encoder_matches_oracle_random(blco, dims, nnz, B):
    rng = np.random.default_rng(nnz + B)
    cidx = unique_coords_wide(rng, dims, nnz)
    vals = rng.random(nnz)
    enc = po.blco_encode128(dims, cidx, vals, B)
    t = blco.Tensor.encode(dims, cidx, vals, B)
    _check_encoding(t, enc)
    t.free()


def test_wide_encoder_duplicates_keep_input_order(blco):
    rng = np.random.default_rng(5)
    dims = [1 << 24, 1 << 24, 1 << 24]
    base = unique_coords_wide(rng, dims, 2000)
    cidx = np.concatenate([base, base[:, :700], base[:, 100:300]], axis=1)
    vals = rng.random(cidx.shape[1])
    enc = po.blco_encode128(dims, cidx, vals, 50)
    t = blco.Tensor.encode(dims, cidx, vals, 50)
    _check_encoding(t, enc)
    t.free()


def test_wide_encoder_edges(blco):
    dims = [1 << 30, 1 << 30, 1 << 12]
    t = blco.Tensor.encode(dims, np.zeros((3, 0), np.uint64), np.zeros(0))
    inf = t.info()
    assert inf["nnz"] == 0 and inf["block_count"] == 0 and inf["alto_bits"] == 72
    t.free()
    one = np.array([[5], [(1 << 30) - 1], [4000]], dtype=np.uint64)
    t = blco.Tensor.encode(dims, one, np.array([2.5]))
    o = t.copy_out()
    enc = po.blco_encode128(dims, one, np.array([2.5]), 0)
    _check_encoding(t, enc)
    assert o["block_coords"].any()
    t.free()
    bad = one.copy()
    bad[2, 0] = 1 << 12
    with pytest.raises(blco.BlcoError) as e:
        blco.Tensor.encode(dims, bad, np.array([1.0]))
    assert e.value.status == blco.ERR_INVALID
    with pytest.raises(blco.BlcoError) as e:
        blco.Tensor.encode([(1 << 32) - 1] * 5, np.zeros((5, 1), np.uint64), np.ones(1))
    assert e.value.status == blco.ERR_UNSUPPORTED
    with pytest.raises(blco.BlcoError) as e:
        blco.Tensor.encode(dims, one, np.ones(1), opts=blco.make_opts(stream_data=True))
    assert e.value.status == blco.ERR_UNSUPPORTED


def test_wide_noalloc_encoder_rejects(blco):
    torch = _torch()
    dims = [1 << 30, 1 << 30, 1 << 12]
    d_cidx = [torch.zeros(4, dtype=torch.int64, device="cuda") for _ in dims]
    d_vals = torch.ones(4, dtype=torch.float64, device="cuda")
    oc = torch.zeros(4, dtype=torch.int64, device="cuda")
    ov = torch.zeros(4, dtype=torch.float64, device="cuda")
    with pytest.raises(blco.BlcoError) as e:
        blco.encode_device_noalloc(dims, d_cidx, d_vals, oc, ov)
    assert e.value.status == blco.ERR_UNSUPPORTED


def _mttkrp_gpu(blco, t, fs, mode, kernel=10, init=None):
    torch = _torch()
    d_f = [torch.from_numpy(f).cuda() for f in fs]
    out = torch.zeros((fs[mode].shape[0], fs[0].shape[1]), dtype=torch.float64, device="cuda")
    if init is not None:
        out.copy_(torch.from_numpy(init))
    blco.mttkrp(t, mode, d_f, out, blco.make_opts(kernel=kernel))
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("name", [n for n in WIDE if int(golden_case(n)["rank"]) > 0])
def test_wide_mttkrp_matches_reference_golden(blco, name):
    g = golden_case(name)
    dims = [int(d) for d in g["dims"]]
    fs = formula_factors(dims, int(g["rank"]))
    t = blco.Tensor.encode(dims, g["cidx"], g["vals"], int(g["max_block_size"]))
    for m in range(len(dims)):
        out = _mttkrp_gpu(blco, t, fs, m)
        assert np.allclose(out, g[f"mttkrp{m}"], rtol=1e-12, atol=0), m
    t.free()


@pytest.mark.parametrize("rank", [1, 3, 8, 13, 16, 31, 32, 40, 64, 100, 130, 256])
def test_wide_mttkrp_ranks(blco, rank):
    rng = np.random.default_rng(rank)
    dims = [9000, 8500, 8200, 8192, 8300]  # 69 bits
    cidx = unique_coords_wide(rng, dims, 40_000)
    vals = rng.random(40_000)
    fs = [rng.random((d, rank)) for d in dims]
    t = blco.Tensor.encode(dims, cidx, vals, 3000)
    for m in range(5):
        ref = po.mttkrp_coo(cidx, vals, fs, m)
        out = _mttkrp_gpu(blco, t, fs, m)
        assert np.allclose(out, ref, rtol=1e-12, atol=0), (rank, m)
    t.free()


def test_wide_mttkrp_every_kernel_id_and_accumulates(blco):
    rng = np.random.default_rng(9)
    dims = [1 << 17] * 4  # 68 bits; mode 0 rows repeat
    cidx = unique_coords_wide(rng, dims, 50_000)
    cidx[0] %= 300
    cidx = np.unique(cidx, axis=1)
    vals = rng.random(cidx.shape[1])
    R = 16
    fs = [rng.random((d, R)) for d in dims]
    t = blco.Tensor.encode(dims, cidx, vals)
    for m in range(4):
        ref = po.mttkrp_coo(cidx, vals, fs, m)
        init = rng.random(ref.shape)
        for k in (1, 2, 3, 10, 11, 12, 13, 20, 21):
            out = _mttkrp_gpu(blco, t, fs, m, kernel=k, init=init)
            assert np.allclose(out, ref + init, rtol=1e-12, atol=0), (m, k)
    t.free()


def test_wide_mttkrp_large_many_blocks(blco):
    """4M nonzeros over 5 modes of 16384 (70 key bits, 64 block-coordinate
    values) against the oracle's COO MTTKRP."""
    rng = np.random.default_rng(12)
    dims = [1 << 14] * 5
    nnz = 4_000_000
    cidx = unique_coords_wide(rng, dims, nnz)
    vals = rng.random(nnz)
    R = 32
    fs = [rng.random((d, R)) for d in dims]
    t = blco.Tensor.encode(dims, cidx, vals, 1 << 16)
    assert t.info()["block_count"] >= 64
    for m in (0, 4):
        ref = po.mttkrp_coo(cidx, vals, fs, m)
        out = _mttkrp_gpu(blco, t, fs, m)
        assert np.allclose(out, ref, rtol=1e-12, atol=0), m
    t.free()


def test_wide_forms_and_tuner(blco):
    """Wide keys take FP64 or FP32 factors; BF16 gathers and the tuner
    (one schedule) answer BLCO_ERR_UNSUPPORTED."""
    torch = _torch()
    dims = [1 << 17] * 4  # 68 bits
    rng = np.random.default_rng(2)
    cidx = unique_coords_wide(rng, dims, 1000)
    t = blco.Tensor.encode(dims, cidx, rng.random(1000))
    b16 = [torch.zeros((d, 8), dtype=torch.bfloat16, device="cuda") for d in dims]
    with pytest.raises(blco.BlcoError) as e:
        blco.mttkrp_ex(t, 3, b16[:3] + [None], torch.zeros((dims[3], 8), dtype=torch.float32, device="cuda"),
                       blco.DTYPE_BF16)
    assert e.value.status == blco.ERR_UNSUPPORTED
    with pytest.raises(blco.BlcoError) as e:
        blco.cpals(t, [np.ones((d, 2)) for d in dims], np.ones(2), 1, 0.0,
                   blco.make_opts(precision=blco.PRECISION_MIXED_BF16))
    assert e.value.status == blco.ERR_UNSUPPORTED
    with pytest.raises(blco.BlcoError) as e:
        blco.autotune(t, 0, 8)
    assert e.value.status == blco.ERR_UNSUPPORTED
    t.free()


@pytest.mark.parametrize("rank", [5, 8, 16, 32, 64, 96, 160])
def test_wide_mixed_mttkrp(blco, rank):
    """FP32 values and factors, FP64 run sums, FP32 output: within 1e-5
    normwise of the COO oracle on the same (rounded) inputs."""
    torch = _torch()
    rng = np.random.default_rng(100 + rank)
    dims = [9000, 8500, 8200, 8192, 8300] if rank % 2 else [1 << 17, 1 << 17, 100_000, 1 << 17]
    cidx = unique_coords_wide(rng, dims, 60_000)
    vals = rng.random(60_000).astype(np.float32).astype(np.float64)
    fs = [rng.random((d, rank)).astype(np.float32) for d in dims]
    t = blco.Tensor.encode(dims, cidx, vals, 7000)
    d_f = [torch.from_numpy(f).cuda() for f in fs]
    for m in range(len(dims)):
        ref = po.mttkrp_coo(cidx, vals, [f.astype(np.float64) for f in fs], m)
        out = torch.zeros((dims[m], rank), dtype=torch.float32, device="cuda")
        blco.mttkrp_ex(t, m, d_f, out, blco.DTYPE_F32)
        torch.cuda.synchronize()
        o = out.double().cpu().numpy()
        assert np.linalg.norm(o - ref) <= 1e-5 * np.linalg.norm(ref), (rank, m)
    t.free()


def test_wide_mixed_cpals_within_bound(blco):
    """The chosen form on a wide-key tensor: fit within 1e-5 of FP64."""
    rng = np.random.default_rng(31)
    dims = [1 << 17, 1 << 17, 100_000, 1 << 17]
    nnz = 80_000
    cidx = unique_coords_wide(rng, dims, nnz)
    vals = rng.random(nnz)
    R = 16
    fs0 = [rng.random((d, R)) for d in dims]
    t = blco.Tensor.encode(dims, cidx, vals)
    _, f64 = blco.cpals(t, [f.copy() for f in fs0], np.ones(R), 8, 0.0)
    _, f32 = blco.cpals(t, [f.copy() for f in fs0], np.ones(R), 8, 0.0,
                        blco.make_opts(precision=blco.PRECISION_MIXED))
    assert len(f32) == 8
    assert np.max(np.abs(np.array(f32) - np.array(f64))) <= 1e-5
    t.free()


@pytest.mark.parametrize("R,iters", [(8, 10), (16, 6)])
def test_wide_cpals_matches_oracle(blco, R, iters):
    rng = np.random.default_rng(R)
    dims = [9000, 8500, 8200, 8192, 8300]
    nnz = 30_000
    cidx = unique_coords_wide(rng, dims, nnz)
    vals = rng.random(nnz)
    fs0 = [rng.random((d, R)) for d in dims]
    fo = [f.copy() for f in fs0]
    lo = np.ones(R)
    fits_o = po.cpals_coo(dims, cidx, vals, fo, lo, iters, 0.0)
    t = blco.Tensor.encode(dims, cidx, vals, 5000)
    fg = [f.copy() for f in fs0]
    lg = np.ones(R)
    fit_g, fits_g = blco.cpals(t, fg, lg, iters, 0.0, blco.make_opts(kernel=21))
    assert len(fits_g) == len(fits_o) == iters
    assert np.allclose(fits_g, fits_o, rtol=0, atol=1e-10)
    for a, b in zip(fg, fo):
        assert np.linalg.norm(a - b) <= 1e-9 * np.linalg.norm(b)
    assert np.allclose(lg, lo, rtol=1e-9)
    t.free()


def test_wide_tns_loader(blco, tmp_path):
    """A .tns file whose indices need 100 key bits goes through the GPU
    loader (dims from the largest index per mode) and encodes as the host
    arrays do."""
    rng = np.random.default_rng(21)
    dims = [1 << 25, 1 << 25, 1 << 25, 1 << 25]
    cidx = unique_coords_wide(rng, dims, 20_000)
    vals = rng.random(20_000)
    p = os.path.join(str(tmp_path), "w.tns")
    with open(p, "w") as f:
        for i in range(cidx.shape[1]):
            f.write(" ".join(str(int(c) + 1) for c in cidx[:, i]) + " %r\n" % float(vals[i]))
    t_gpu, info = blco.Tensor.encode_tns(p)
    real_dims = [int(cidx[n].max()) + 1 for n in range(4)]
    assert info["dims"] == real_dims
    t_ref = blco.Tensor.encode(real_dims, cidx, vals)
    a, b = t_gpu.copy_out(), t_ref.copy_out()
    assert a["alto_bits"] > 64
    for k in ("coords", "block_offsets", "block_coords"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(a["vals"].view(np.uint64), b["vals"].view(np.uint64))
    t_gpu.free()
    t_ref.free()
