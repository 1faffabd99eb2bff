"""GPU tests of the mixed-precision (chosen) form.

MTTKRP: FP32 values and accumulation with FP32 or BF16 factor gathers,
compared with the oracle evaluated in FP64 on the same rounded inputs
(values rounded to FP32, factors to FP32 or BF16), so only the FP32
accumulation differs: normwise relative error <= 1e-5.

CP-ALS: the chosen form keeps FP64 for the R x R solve, lambda and the fit;
its fit must stay within 1e-5 (absolute) of the FP64 oracle's.
"""
import numpy as np
import pytest

import pyoracle as po
from conftest import unique_coords

pytestmark = pytest.mark.gpu


def _round_bf16(a):
    a32 = np.ascontiguousarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


@pytest.mark.parametrize("dtype", ["f32", "bf16"])
@pytest.mark.parametrize("rank", [8, 16, 32, 64, 24])
def test_mixed_mttkrp_matches_oracle(blco, dtype, rank):
    import torch
    rng = np.random.default_rng(rank)
    dims = [20_000, 5_000, 300]
    nnz = 200_000
    cidx = unique_coords(rng, dims, nnz, zipf=1.1)
    vals = rng.lognormal(0.0, 1.0, nnz)
    t = blco.Tensor.encode(dims, cidx, vals)
    fs = [rng.random((d, rank)) for d in dims]
    if dtype == "f32":
        fr = [f.astype(np.float32) for f in fs]
        dev = [torch.from_numpy(f).cuda() for f in fr]
        code = blco.DTYPE_F32
    else:
        fr = [_round_bf16(f) for f in fs]
        dev = [torch.from_numpy(f).cuda().to(torch.bfloat16) for f in fr]
        code = blco.DTYPE_BF16
    v32 = vals.astype(np.float32).astype(np.float64)
    for m in range(3):
        ref = po.mttkrp_coo(cidx, v32, [f.astype(np.float64) for f in fr], m)
        for kernel in (1, 2, 10, 13):
            out = torch.zeros(dims[m], rank, dtype=torch.float32, device="cuda")
            blco.mttkrp_ex(t, m, dev, out, code, blco.make_opts(kernel=kernel))
            torch.cuda.synchronize()
            o = out.cpu().numpy().astype(np.float64)
            err = np.linalg.norm(o - ref) / np.linalg.norm(ref)
            assert err <= 1e-5, (m, kernel, err)


def test_mixed_mttkrp_rejects_bad_dtype(blco):
    import torch
    t = blco.Tensor.encode([4, 4, 4], np.array([[1], [2], [3]], dtype=np.uint64), np.ones(1))
    fs = [torch.ones(4, 8, dtype=torch.float32, device="cuda") for _ in range(3)]
    out = torch.zeros(4, 8, dtype=torch.float32, device="cuda")
    with pytest.raises(blco.BlcoError) as e:
        blco.mttkrp_ex(t, 0, fs, out, 7)
    assert e.value.status == blco.ERR_INVALID


@pytest.mark.parametrize("precision", ["mixed", "mixed_bf16"])
def test_mixed_cpals_fit_within_1e5(blco, precision):
    from blco_b200 import synth
    X = synth.uniform_tensor_host(40_000, [1000, 800, 600], seed=2)
    R = 16
    rng = np.random.default_rng(5)
    fs0 = [rng.random((d, R)) for d in X["dims"]]
    enc = po.blco_encode(X["dims"], X["cidx"], X["vals"])
    fo = [f.copy() for f in fs0]
    fits_o = po.cpals(X["dims"], enc, fo, np.ones(R), 20, 0.0)
    t = blco.Tensor.encode(X["dims"], X["cidx"], X["vals"])
    prec = blco.PRECISION_MIXED if precision == "mixed" else blco.PRECISION_MIXED_BF16
    fg = [f.copy() for f in fs0]
    _, fits_g = blco.cpals(t, fg, np.ones(R), 20, 0.0, blco.make_opts(precision=prec))
    d = np.max(np.abs(np.array(fits_g) - np.array(fits_o)))
    assert d <= 1e-5, (d, fits_g[-1], fits_o[-1])


def test_mixed_cpals_skewed_fit_within_1e5(blco):
    rng = np.random.default_rng(9)
    dims = [50_000, 40_000, 2_000]
    nnz = 300_000
    cidx = unique_coords(rng, dims, nnz, zipf=1.1)
    vals = rng.lognormal(0.0, 1.0, nnz)
    R = 32
    fs0 = [rng.random((d, R)) for d in dims]
    enc = po.blco_encode(dims, cidx, vals)
    fo = [f.copy() for f in fs0]
    fits_o = po.cpals(dims, enc, fo, np.ones(R), 10, 0.0)
    t = blco.Tensor.encode(dims, cidx, vals)
    # FP32 gathers meet the 1e-5 bound.  BF16 gathers (8-bit mantissa) do not
    # on this skewed tensor (about 1.3e-4 was measured); they are checked
    # against a looser bound and are only chosen when the 1e-5 bound holds.
    for prec, bound in ((blco.PRECISION_MIXED, 1e-5), (blco.PRECISION_MIXED_BF16, 1e-3)):
        fg = [f.copy() for f in fs0]
        _, fits_g = blco.cpals(t, fg, np.ones(R), 10, 0.0, blco.make_opts(precision=prec))
        d = np.max(np.abs(np.array(fits_g) - np.array(fits_o)))
        assert d <= bound, (prec, d, fits_g[-1], fits_o[-1])


def test_mixed_plan_runs_fp64_when_ill_conditioned(blco):
    """A mixed plan whose R x R systems are ill-conditioned continues in FP64
    (the FP32 working set's rounding grows with the condition number):
    initial factors with two nearly equal columns make the first systems'
    condition estimates huge, so the plan is promoted; with the guard off it
    stays mixed.  (Such a start is chaotic in FP64 as well, through the
    order of FP64 atomics, so fits are compared in the next test.)"""
    import torch
    rng = np.random.default_rng(21)
    dims = [3000, 800, 200]
    cidx = unique_coords(rng, dims, 40_000, zipf=0.9)
    vals = rng.random(40_000)
    t = blco.Tensor.encode(dims, cidx, vals)
    R = 8
    fs0 = [rng.random((d, R)) for d in dims]
    for f in fs0:
        f[:, 1] = f[:, 0] * (1.0 + 1e-7 * rng.random(f.shape[0]))

    def promoted(precision, guard):
        dfs = [torch.from_numpy(f.copy()).cuda() for f in fs0]
        lam = torch.ones(R, dtype=torch.float64, device="cuda")
        plan = blco.CpalsPlan(t, dfs, lam, blco.make_opts(precision=precision, guard_cond=guard))
        plan.iterate(3, tol=-1.0)
        _, pr = plan.condition()
        plan.destroy()
        return pr

    assert not promoted(blco.PRECISION_FP64, 0.0)  # an FP64 plan has nothing to promote
    assert promoted(blco.PRECISION_MIXED, 0.0)
    assert not promoted(blco.PRECISION_MIXED, -1.0)
    t.free()


def test_promoted_plan_follows_fp64(blco):
    """Promotion at creation hands the caller's FP64 factors to the FP64
    path unchanged: with a guard every system exceeds (1.5), the mixed plan
    follows the FP64 plan's fits and factors (a well-conditioned tensor, so
    FP64 runs agree to rounding of the atomics' order)."""
    import torch
    rng = np.random.default_rng(23)
    dims = [3000, 800, 200]
    cidx = unique_coords(rng, dims, 40_000)
    vals = rng.random(40_000)
    t = blco.Tensor.encode(dims, cidx, vals)
    R = 8
    fs0 = [rng.random((d, R)) for d in dims]
    out = []
    for precision, guard in ((blco.PRECISION_FP64, 0.0), (blco.PRECISION_MIXED, 1.5)):
        dfs = [torch.from_numpy(f.copy()).cuda() for f in fs0]
        lam = torch.ones(R, dtype=torch.float64, device="cuda")
        plan = blco.CpalsPlan(t, dfs, lam, blco.make_opts(precision=precision, guard_cond=guard))
        fits = plan.iterate(6, tol=-1.0)
        _, pr = plan.condition()
        plan.destroy()
        out.append((np.array(fits), [d.cpu().numpy() for d in dfs], pr))
    (f64, u64, p64), (fmix, umix, pmix) = out
    assert not p64 and pmix
    assert np.allclose(fmix, f64, rtol=0, atol=1e-10), np.abs(fmix - f64).max()
    for a, b in zip(umix, u64):
        assert np.linalg.norm(a - b) <= 1e-9 * np.linalg.norm(b)
    t.free()


def test_mixed_plan_stays_mixed_when_well_conditioned(blco):
    """Uniform random factors of a uniform tensor: every condition estimate
    stays far below the guard and the plan keeps its FP32 working set."""
    import torch
    rng = np.random.default_rng(22)
    dims = [3000, 800, 200]
    cidx = unique_coords(rng, dims, 40_000)
    vals = rng.random(40_000)
    t = blco.Tensor.encode(dims, cidx, vals)
    R = 8
    dfs = [torch.from_numpy(rng.random((d, R))).cuda() for d in dims]
    lam = torch.ones(R, dtype=torch.float64, device="cuda")
    plan = blco.CpalsPlan(t, dfs, lam, blco.make_opts(precision=blco.PRECISION_MIXED))
    plan.iterate(4, tol=-1.0)
    cond, promoted = plan.condition()
    assert not promoted and 1.0 <= cond.max() < blco.GUARD_COND
    plan.destroy()
    t.free()
