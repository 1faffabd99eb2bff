"""CPU tests of the oracle: pinned against the reference's own outputs.

The golden fixtures were produced by the reference code compiled from its
sources (tests/golden/make_golden.py via oracle/_ref).  The oracle must
reproduce the reference BLCO encoding bit for bit and its COO MTTKRP to
rounding.
"""
import numpy as np
import pytest

import pyoracle as po
from conftest import formula_factors, golden_case, golden_index, unique_coords

CASES = [c["name"] for c in golden_index()["cases"]]


@pytest.mark.parametrize("name", CASES)
def test_encoder_matches_reference_golden(name):
    g = golden_case(name)
    enc = po.blco_encode(g["dims"], g["cidx"], g["vals"], int(g["max_block_size"]))
    assert np.array_equal(enc["coords"], g["coords"])
    assert np.array_equal(enc["vals"], g["out_vals"])  # bit-exact values, ALTO order
    assert np.array_equal(enc["mode_masks"], g["mode_masks"])
    assert np.array_equal(enc["mode_pos"], g["mode_pos"])
    assert np.array_equal(enc["block_offsets"], g["block_offsets"])
    assert np.all(g["block_coords"] == 0)


def test_kat_values():
    """The known-answer vector written out by hand (reference encoder output)."""
    g = golden_case("kat_5x3x9")
    masks, bits = po.alto_masks([5, 3, 9])
    assert [int(m) for m in masks] == [0x52, 0x9, 0x1A4] and bits == 9
    assert [int(c) for c in g["coords"]] == [0x0, 0xB, 0x71, 0xA2, 0xE8, 0x114]
    assert list(g["out_vals"]) == [2, 4, 3, 5, 6, 1]
    assert [int(m) for m in g["mode_masks"]] == [0x7, 0x3, 0xF]
    assert list(g["mode_pos"]) == [0, 3, 5]
    assert list(g["block_offsets"]) == [0, 4, 6]


def test_alto_masks_tie_order():
    masks, bits = po.alto_masks([16, 16, 16])
    assert [int(m) for m in masks] == [0x249, 0x492, 0x924] and bits == 12


def test_alto_masks_reject_wide_keys():
    with pytest.raises(ValueError):
        po.alto_masks([1 << 30, 1 << 30, 1 << 10])


@pytest.mark.parametrize("name", CASES)
def test_coo_mttkrp_matches_reference_golden(name):
    g = golden_case(name)
    dims = [int(d) for d in g["dims"]]
    R = int(g["rank"])
    fs = formula_factors(dims, R)
    for m in range(len(dims)):
        out = po.mttkrp_coo(g["cidx"], g["vals"], fs, m)
        ref = g[f"mttkrp{m}"]
        # same arithmetic order as the reference loop: identical bits
        assert np.array_equal(out, ref), (name, m)


@pytest.mark.parametrize("name", CASES)
def test_blco_stream_mttkrp_matches_reference(name):
    g = golden_case(name)
    dims = [int(d) for d in g["dims"]]
    R = int(g["rank"])
    fs = formula_factors(dims, R)
    enc = dict(coords=g["coords"], vals=g["out_vals"], mode_masks=g["mode_masks"], mode_pos=g["mode_pos"])
    for m in range(len(dims)):
        out = po.mttkrp_blco(enc, fs, m)
        ref = g[f"mttkrp{m}"]
        err = np.linalg.norm(out - ref) / max(np.linalg.norm(ref), 1e-300)
        assert err <= 1e-13, (name, m, err)


@pytest.mark.parametrize("nthreads", [1, 3, 8])
def test_random_init_matches_reference(nthreads):
    import os
    from conftest import GOLDEN
    g = dict(np.load(os.path.join(GOLDEN, f"init_t{nthreads}.npz")))
    fs, lam = po.kruskal_random_init([7, 13, 5], 6, 12345, nthreads)
    for m in range(3):
        assert np.array_equal(fs[m], g[f"f{m}"])
    assert np.array_equal(lam, g["lam"])


def test_encoder_duplicates_keep_input_order():
    dims = [4, 4, 4]
    cidx = np.array([[1, 1, 0, 1], [2, 2, 0, 2], [3, 3, 0, 3]], dtype=np.uint64)
    vals = np.array([10.0, 20.0, 30.0, 40.0])
    enc = po.blco_encode(dims, cidx, vals)
    assert list(enc["vals"]) == [30.0, 10.0, 20.0, 40.0]


def test_encoder_rejects_out_of_range():
    with pytest.raises(ValueError):
        po.blco_encode([4, 4], np.array([[0, 4], [0, 0]], dtype=np.uint64), np.ones(2))


def test_oracle_matches_ref_build_on_random_inputs():
    """When oracle/_ref is built (here, not on the GPU box), compare on
    random inputs beyond the fixtures."""
    if po.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(7)
    for dims, nnz, B in [([300, 70, 9000], 20000, 3000), ([5, 6, 7, 8], 1500, 0), ([2, 3, 2, 5, 1000], 500, 64)]:
        cidx = unique_coords(rng, dims, nnz)
        vals = rng.random(nnz)
        a = po.blco_encode(dims, cidx, vals, B)
        b = po.ref_blco_encode(dims, cidx, vals, B)
        for k in ("coords", "vals", "mode_masks", "mode_pos", "block_offsets"):
            assert np.array_equal(a[k], b[k]), k


def _pinv_check(a, p):
    # Moore-Penrose conditions
    assert np.allclose(a @ p @ a, a, atol=1e-10 * np.abs(a).max())
    assert np.allclose(p @ a @ p, p, atol=1e-10 * max(np.abs(p).max(), 1))
    assert np.allclose(a @ p, (a @ p).T, atol=1e-10)


def test_pinv_full_rank_and_singular():
    rng = np.random.default_rng(3)
    x = rng.random((50, 8))
    a = x.T @ x
    p = po.pinv_sym(a)
    assert np.allclose(p, np.linalg.inv(a), rtol=1e-9, atol=1e-12)
    _pinv_check(a, p)
    y = np.concatenate([x[:, :4], x[:, :4]], axis=1)  # rank 4 of 8
    b = y.T @ y
    q = po.pinv_sym(b)
    _pinv_check(b, q)
    assert np.allclose(q, np.linalg.pinv(b, rcond=1e-12, hermitian=True), atol=1e-8)


def test_cpals_oracle_recovers_exact_low_rank():
    """Dense exactly rank-2 tensor: the fit of the GPU-semantics CP-ALS
    restatement approaches 1."""
    rng = np.random.default_rng(11)
    dims = [6, 5, 4]
    A = [rng.random((d, 2)) + 0.1 for d in dims]
    T = np.einsum("ir,jr,kr->ijk", *A)
    idx = np.array(np.unravel_index(np.arange(T.size), T.shape), dtype=np.uint64)
    enc = po.blco_encode(dims, idx, T.reshape(-1))
    fs = [rng.random((d, 2)) for d in dims]
    lam = np.ones(2)
    fits = po.cpals(dims, enc, fs, lam, 200, 0.0)
    assert fits[-1] > 0.999, fits[-5:]


def test_cpals_oracle_stops_on_tolerance():
    rng = np.random.default_rng(12)
    dims = [30, 20, 10]
    cidx = unique_coords(rng, dims, 800)
    enc = po.blco_encode(dims, cidx, rng.random(800))
    fs = [rng.random((d, 4)) for d in dims]
    lam = np.ones(4)
    fits = po.cpals(dims, enc, fs, lam, 50, 1e-1)
    assert len(fits) < 50
    assert abs(fits[-1] - (fits[-2] if len(fits) > 1 else 0.0)) < 1e-1
