"""GPU parity of the BLCO encoder (through the C ABI) against the reference
encoder's golden outputs and the oracle: bit-exact."""
import numpy as np
import pytest

import pyoracle as po
from conftest import golden_case, golden_index, unique_coords

pytestmark = pytest.mark.gpu

CASES = [c["name"] for c in golden_index()["cases"]]


def _check_same(t_out, ref):
    assert np.array_equal(t_out["coords"], ref["coords"])
    assert np.array_equal(t_out["vals"], ref["vals"])
    assert [int(x) for x in t_out["mode_masks"]] == [int(x) for x in ref["mode_masks"]]
    assert [int(x) for x in t_out["mode_pos"]] == [int(x) for x in ref["mode_pos"]]
    assert np.array_equal(t_out["block_offsets"], ref["block_offsets"])


@pytest.mark.parametrize("name", CASES)
def test_encode_matches_reference_golden(blco, name):
    g = golden_case(name)
    t = blco.Tensor.encode(g["dims"], g["cidx"], g["vals"], int(g["max_block_size"]))
    out = t.copy_out()
    _check_same(out, dict(coords=g["coords"], vals=g["out_vals"], mode_masks=g["mode_masks"],
                          mode_pos=g["mode_pos"], block_offsets=g["block_offsets"]))
    assert np.array_equal(out["block_coords"], g["block_coords"])
    assert out["block_count"] == len(g["block_offsets"]) - 1
    t.free()


@pytest.mark.parametrize("dims,nnz,B,zipf", [
    ([2_000_000, 2_000_000, 25_000], 300_000, 0, 1.1),
    ([500_000, 200_000, 50_000, 1_000], 200_000, 65_536, 0.9),
    ([1000, 800, 600], 100_000, 0, None),
    ([3, 1 << 20, 7, 1 << 12, 2], 50_000, 10_000, None),
])
def test_encode_random_matches_oracle(blco, dims, nnz, B, zipf):
    rng = np.random.default_rng(nnz)
    cidx = unique_coords(rng, dims, nnz, zipf)
    vals = rng.lognormal(0.0, 1.0, nnz)
    t = blco.Tensor.encode(dims, cidx, vals, B)
    ref = po.blco_encode(dims, cidx, vals, B)
    _check_same(t.copy_out(), ref)
    info = t.info()
    assert [int(x) for x in info["alto_masks"]] == [int(x) for x in ref["alto_masks"]]


def test_encode_duplicates_stable(blco):
    rng = np.random.default_rng(5)
    dims = [50, 40, 30]
    cidx = rng.integers(0, 30, size=(3, 20000)).astype(np.uint64)  # many duplicates
    vals = rng.random(20000)
    t = blco.Tensor.encode(dims, cidx, vals)
    ref = po.blco_encode(dims, cidx, vals)
    _check_same(t.copy_out(), ref)


def test_encode_device_arrays(blco):
    import torch
    rng = np.random.default_rng(9)
    dims = [100_000, 3_000, 20]
    cidx = unique_coords(rng, dims, 60_000)
    vals = rng.random(60_000)
    d_c = [torch.from_numpy(cidx[n].astype(np.int64)).cuda() for n in range(3)]
    d_v = torch.from_numpy(vals).cuda()
    t = blco.Tensor.encode_device(dims, d_c, d_v, 7_000)
    _check_same(t.copy_out(), po.blco_encode(dims, cidx, vals, 7_000))


def test_encode_empty_and_single(blco):
    t = blco.Tensor.encode([3, 4, 5], np.zeros((3, 0), dtype=np.uint64), np.zeros(0))
    out = t.copy_out()
    assert out["nnz"] == 0 and out["block_count"] == 0 and list(out["block_offsets"]) == [0]
    t = blco.Tensor.encode([3, 4, 5], np.array([[2], [3], [4]], dtype=np.uint64), np.array([7.5]))
    out = t.copy_out()
    assert list(out["coords"]) == [2 | (3 << 2) | (4 << 4)] and list(out["vals"]) == [7.5]


def test_encode_errors(blco):
    with pytest.raises(blco.BlcoError) as e:
        blco.Tensor.encode([4, 4], np.array([[0, 4], [0, 0]], dtype=np.uint64), np.ones(2))
    assert e.value.status == blco.ERR_INVALID
    with pytest.raises(blco.BlcoError) as e:
        # 160 key bits: wider than the reference's widest (128-bit) key
        blco.Tensor.encode([(1 << 32) - 1] * 5, np.zeros((5, 1), dtype=np.uint64), np.ones(1))
    assert e.value.status == blco.ERR_UNSUPPORTED
    with pytest.raises(blco.BlcoError) as e:
        blco.Tensor.encode([4, 0], np.zeros((2, 1), dtype=np.uint64), np.ones(1))
    assert e.value.status == blco.ERR_INVALID
