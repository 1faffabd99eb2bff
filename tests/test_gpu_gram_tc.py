"""The mixed form's Gram on the tensor cores (tcgen05, integer digits)
against a plain PyTorch FP64 reference of the same op, and the mixed CP-ALS
with the tensor-core Grams against the CUDA-core Grams and the FP64 form.

Tolerances: per 64-row tile and column, every FP32 value becomes four 8-bit
integer digits under a power-of-two scale above the column's largest
magnitude, so it is represented to within 2^-33 of that magnitude; digit
products are exact, and their sums over a tile stay below 2^22, exact in the
tensor cores' FP32 accumulator; the rest is FP64.  The Gram is checked
normwise within 1e-7 relative, and exactly where the digits are exact
(small integers).
"""
import numpy as np
import pytest
import torch

from conftest import unique_coords

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("I", [1, 63, 64, 65, 513, 4096, 100_003, 2_000_000])
@pytest.mark.parametrize("R", [1, 5, 16, 32, 33, 64])
def test_gram_tc_matches_fp64(blco, I, R):
    if I == 2_000_000 and R not in (32, 64):
        pytest.skip("large case at the benchmark ranks only")
    g = torch.Generator(device="cuda").manual_seed(I * 100 + R)
    U = torch.rand(I, R, dtype=torch.float32, device="cuda", generator=g) - 0.3
    ref = U.double().T @ U.double()
    G = blco.gram_f32(U, tensor_cores=True)
    err = (torch.linalg.norm(G - ref) / torch.linalg.norm(ref)).item()
    assert err <= 1e-7, err
    if I >= 64:
        # a tile whose magnitudes span decades (Zipf-skewed factor rows):
        # the low digits keep the small values
        U[:64] *= torch.logspace(0, -6, 64, device="cuda", dtype=torch.float32)[:, None]
        ref = U.double().T @ U.double()
        G = blco.gram_f32(U, tensor_cores=True)
        err = (torch.linalg.norm(G - ref) / torch.linalg.norm(ref)).item()
        assert err <= 1e-7, err
    Gc = blco.gram_f32(U, tensor_cores=False)
    assert (torch.linalg.norm(Gc - ref) / torch.linalg.norm(ref)).item() <= 1e-12
    # the digit pairs kept (i + j <= 2) are a symmetric set
    assert torch.allclose(G, G.T, rtol=0, atol=1e-12 * ref.abs().max().item())


@pytest.mark.parametrize("R", [3, 16, 32, 48, 64])
def test_gram_tc_is_exact_on_integer_inputs(blco, R):
    """Integers below 2^15 in magnitude are exact in three digits under any
    tile scale, so every partial sum the tensor cores form is an exact
    integer: the Gram must equal the integer Gram exactly (it would not if
    the FP32 accumulator rounded).  Columns of very different magnitudes,
    and whole tiles of zeros."""
    rng = np.random.default_rng(R)
    I = 300_001
    Ui = rng.integers(-3000, 3001, size=(I, R))
    Ui[:, ::3] //= 1000         # columns of magnitude <= 3
    Ui[64 * 10:64 * 12, :] = 0  # two tiles of zeros
    want = Ui.T.astype(np.int64) @ Ui.astype(np.int64)
    U = torch.from_numpy(Ui.astype(np.float32)).cuda()
    G = blco.gram_f32(U, tensor_cores=True).cpu().numpy()
    assert np.array_equal(G, want.astype(np.float64)), np.abs(G - want).max()


def test_gram_tc_bias_free_on_many_tiles(blco):
    """The mean signed error over 1M rows of positive values stays at the
    digits' rounding level (no drift with the number of tiles)."""
    g = torch.Generator(device="cuda").manual_seed(5)
    U = torch.rand(1_000_000, 32, dtype=torch.float32, device="cuda", generator=g)
    ref = U.double().T @ U.double()
    G = blco.gram_f32(U, tensor_cores=True)
    rel = ((G - ref) / ref).mean().item()
    assert abs(rel) <= 2e-9, rel


def test_gram_tc_timeout_is_reported_and_recovered(blco):
    """A launch whose completion wait is made to run out (no MMA, no commit:
    a barrier nothing arrives on) reports BLCO_ERR_TIMEOUT; an ordinary
    launch right after it runs and is exact, so the first freed its tensor
    memory and the context is usable."""
    first, after = blco.gram_tc_timeout_check(0)
    assert first == blco.ERR_TIMEOUT, first
    assert after == blco.OK, after


def test_gram_tc_rejects_large_rank(blco):
    U = torch.zeros(10, 65, dtype=torch.float32, device="cuda")
    with pytest.raises(blco.BlcoError) as e:
        blco.gram_f32(U)
    assert e.value.status == blco.ERR_UNSUPPORTED


@pytest.mark.parametrize("R", [16, 48])
@pytest.mark.parametrize("prec", ["PRECISION_MIXED", "PRECISION_MIXED_BF16"])
def test_mixed_cpals_tensor_core_grams(blco, prec, R):
    """Rank 16 runs the per-super-tile kernel, rank 48 the two-halves one,
    each with the column scaling (and, in the BF16 form, the BF16 copy)."""
    rng = np.random.default_rng(8)
    dims = [4000, 3000, 90]
    cidx = unique_coords(rng, dims, 80_000, zipf=0.9)
    vals = rng.random(80_000)
    t = blco.Tensor.encode(dims, cidx, vals)
    fs0 = [rng.random((d, R)) for d in dims]
    out = {}
    for name, o in [("fp64", blco.make_opts()),
                    ("tc", blco.make_opts(precision=getattr(blco, prec), gram_tensor_cores=True)),
                    ("cuda", blco.make_opts(precision=getattr(blco, prec), gram_tensor_cores=False)),
                    ("default", blco.make_opts(precision=getattr(blco, prec)))]:
        f = [x.copy() for x in fs0]
        _, fits = blco.cpals(t, f, np.ones(R), 10, 0.0, o)
        out[name] = np.array(fits)
    # the tensor-core Grams differ from the CUDA-core ones by the digits'
    # rounding (~1e-8 relative, unbiased).  The BF16-gather form is itself
    # ~1e-3 away from FP64 and its trajectory follows small changes more.
    bound = 1e-6 if prec == "PRECISION_MIXED" else 1e-4
    assert np.max(np.abs(out["tc"] - out["cuda"])) <= bound
    # the default engine is the tensor cores' (same launches, so the same
    # fits up to the order of FP64 atomics in the MTTKRP)
    assert np.max(np.abs(out["default"] - out["tc"])) <= bound
    if prec == "PRECISION_MIXED":
        assert np.max(np.abs(out["tc"] - out["fp64"])) <= 1e-5
    t.free()
