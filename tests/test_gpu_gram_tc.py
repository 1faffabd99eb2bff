"""The mixed form's Gram on the tensor cores (tcgen05, split-BF16) against a
plain PyTorch FP64 reference of the same op, and the mixed CP-ALS with the
tensor-core Grams against the CUDA-core Grams and the FP64 form.

Tolerances: each FP32 value enters as bf16(u) + bf16(u - bf16(u)), 16
mantissa bits (relative representation error <= 2^-17 per value), products
are exact, sums are FP32 over 64-row tiles then FP64; the Gram is
checked normwise within 1e-5 relative (1e-6 when the inputs are BF16-exact,
leaving only the FP32 partial sums: the tensor cores' FP32 accumulation is
not round-to-nearest and leans low).
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
    assert err <= 1e-5, err
    Gc = blco.gram_f32(U, tensor_cores=False)
    assert (torch.linalg.norm(Gc - ref) / torch.linalg.norm(ref)).item() <= 1e-12
    # symmetric by construction of the four blocks
    assert torch.allclose(G, G.T, rtol=0, atol=1e-12 * ref.abs().max().item())


def test_gram_tc_bf16_exact_inputs(blco):
    """BF16-representable inputs: lo = 0, the products are exact, only the
    FP32 sums over 64-row tiles round."""
    g = torch.Generator(device="cuda").manual_seed(5)
    U = (torch.rand(300_000, 32, dtype=torch.float32, device="cuda", generator=g)).bfloat16().float()
    ref = U.double().T @ U.double()
    G = blco.gram_f32(U, tensor_cores=True)
    assert (torch.linalg.norm(G - ref) / torch.linalg.norm(ref)).item() <= 1e-6


def test_gram_tc_rejects_large_rank(blco):
    U = torch.zeros(10, 65, dtype=torch.float32, device="cuda")
    with pytest.raises(blco.BlcoError) as e:
        blco.gram_f32(U)
    assert e.value.status == blco.ERR_UNSUPPORTED


@pytest.mark.parametrize("prec", ["PRECISION_MIXED", "PRECISION_MIXED_BF16"])
def test_mixed_cpals_tensor_core_grams(blco, prec):
    rng = np.random.default_rng(8)
    dims = [4000, 3000, 90]
    cidx = unique_coords(rng, dims, 80_000, zipf=0.9)
    vals = rng.random(80_000)
    t = blco.Tensor.encode(dims, cidx, vals)
    R = 16
    fs0 = [rng.random((d, R)) for d in dims]
    out = {}
    for name, o in [("fp64", blco.make_opts()),
                    ("tc", blco.make_opts(precision=getattr(blco, prec), gram_tensor_cores=True)),
                    ("cuda", blco.make_opts(precision=getattr(blco, prec)))]:
        f = [x.copy() for x in fs0]
        _, fits = blco.cpals(t, f, np.ones(R), 10, 0.0, o)
        out[name] = np.array(fits)
    # the tensor-core Grams lean low by ~1e-7 relative (biased FP32
    # accumulation over a tile); through the fit's cancellation that is a
    # few 1e-6 absolute for FP32 gathers.  The BF16-gather form is itself
    # ~1e-3 away from FP64 and its trajectory follows small changes more.
    bound = 5e-6 if prec == "PRECISION_MIXED" else 1e-4
    assert np.max(np.abs(out["tc"] - out["cuda"])) <= bound
    if prec == "PRECISION_MIXED":
        assert np.max(np.abs(out["tc"] - out["fp64"])) <= 1e-5
    t.free()
