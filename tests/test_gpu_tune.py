"""MTTKRP schedule selection on the GPU: the autotuner sweep, every schedule
of its space against the oracle, the selector network's kernels against the
CPU oracle (oracle/mlp_oracle.py), and what the trained network gains over
the fixed rules on the committed sweep table
(blocked-linearized-coordinate_b200/selector/tune_table.npz, made by
selector/make_tune_table.py on a B200), and the committed trained parameters.
"""
import os
import sys

import numpy as np
import pytest
import torch

import pyoracle as po
from conftest import PKG_DIR, unique_coords

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import mlp_oracle as mo  # noqa: E402

pytestmark = pytest.mark.gpu


def _tensor(blco, dims, nnz, zipf, seed):
    rng = np.random.default_rng(seed)
    cidx = unique_coords(rng, dims, nnz, zipf=zipf)
    vals = rng.random(nnz)
    return cidx, vals, blco.Tensor.encode(dims, cidx, vals)


def test_tune_space_and_sweep(blco):
    space = blco.tune_space()
    assert len(space) == blco.TUNE_CONFIGS == 14
    assert {c["kernel"] for c in space} == {1, 2, 3, 4, 13}
    dims = [40_000, 3_000, 60]
    _, _, t = _tensor(blco, dims, 300_000, 1.0, 0)
    for mode in range(3):
        ms, best = blco.autotune(t, mode, 32, blco.DTYPE_F64, reps=2)
        valid = ms > 0
        # the shared-memory schedules apply to the 60-row mode only
        assert valid[8] == valid[9] == (mode == 2)
        assert valid.sum() == (14 if mode == 2 else 12)
        assert best == int(np.argmin(np.where(valid, ms, np.inf)))
        ms2, best2 = blco.autotune(t, mode, 32, blco.DTYPE_F64)  # cached
        assert np.array_equal(ms, ms2) and best2 == best
    t.free()


def _forcing_net(blco, k):
    """A network whose prediction is 0 for schedule k and 10 elsewhere."""
    net = blco.Mlp(hidden=8, seed=0)
    p = np.zeros(net.nparams, dtype=np.float32)
    b3 = p[-blco.TUNE_CONFIGS:]
    b3[:] = 10.0
    b3[k] = 0.0
    net.set_params(p)
    return net


@pytest.mark.parametrize("k", list(range(14)))
def test_every_schedule_matches_oracle(blco, k):
    """Schedule k forced through the learned kernel id (21) with a network
    that proposes k with a wide margin; FP64 results within 1e-12 of the
    oracle's COO MTTKRP, FP32 gathers within 1e-5."""
    dims = [30_000, 2_000, 60]
    cidx, vals, t = _tensor(blco, dims, 200_000, 1.0, 1)
    R = 32
    rng = np.random.default_rng(2)
    fs = [rng.random((d, R)) for d in dims]
    net = _forcing_net(blco, k)
    blco.selector_set(net, 1.0)
    try:
        for mode in range(3):
            cfg, swept = blco.select(t, mode, R, blco.DTYPE_F64, net, 1.0)
            if k in (8, 9) and mode != 2:
                assert swept  # not valid there: the sweep decides
            else:
                assert cfg == k and not swept
            ref = po.mttkrp_coo(cidx, vals, fs, mode)
            out = torch.zeros(dims[mode], R, dtype=torch.float64, device="cuda")
            blco.mttkrp(t, mode, [torch.from_numpy(f).cuda() for f in fs], out,
                        blco.make_opts(kernel=blco.KERNEL_LEARNED))
            got = out.cpu().numpy()
            assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)
            out32 = torch.zeros(dims[mode], R, dtype=torch.float32, device="cuda")
            blco.mttkrp_ex(t, mode, [torch.from_numpy(f).float().cuda() for f in fs], out32, blco.DTYPE_F32,
                           blco.make_opts(kernel=blco.KERNEL_LEARNED))
            assert np.linalg.norm(out32.cpu().numpy() - ref) <= 1e-5 * np.linalg.norm(ref)
    finally:
        blco.selector_set(None)
        net.destroy()
        t.free()


def test_mlp_kernels_match_oracle(blco):
    rng = np.random.default_rng(3)
    H, n = 64, 200
    net = blco.Mlp(hidden=H, seed=7)
    p = net.params()
    assert p.size == mo.num_params(H)
    X = rng.normal(size=(n, mo.F)).astype(np.float32)
    Y = rng.normal(size=(n, mo.K)).astype(np.float32)
    M = (rng.random((n, mo.K)) > 0.25).astype(np.float32)
    out = net.predict(X)
    ref, _ = mo.forward(p, X, H)
    assert np.allclose(out, ref, rtol=1e-4, atol=1e-5), np.max(np.abs(out - ref))
    g, loss = net.grad(X, Y, M)
    lref, gref = mo.loss_grad(p, X, Y, M, H)
    assert abs(loss - lref) <= 1e-5 * abs(lref)
    assert np.linalg.norm(g - gref) <= 1e-4 * np.linalg.norm(gref), np.linalg.norm(g - gref) / np.linalg.norm(gref)
    # per parameter block as well (no block may hide behind the others)
    o = 0
    for shape in ((H, mo.F), (H,), (H, H), (H,), (mo.K, H), (mo.K,)):
        sz = int(np.prod(shape))
        gb, rb = g[o:o + sz], gref[o:o + sz]
        assert np.linalg.norm(gb - rb) <= 1e-4 * max(np.linalg.norm(rb), 1e-6), shape
        o += sz
    net.destroy()


def test_mlp_training_is_deterministic_and_learns(blco):
    rng = np.random.default_rng(4)
    n = 300
    X = rng.normal(size=(n, mo.F)).astype(np.float32)
    W = rng.normal(size=(mo.F, mo.K))
    Y = np.abs(X @ W).astype(np.float32) * 0.2
    M = np.ones_like(Y)
    params = []
    losses = []
    for _ in range(2):
        net = blco.Mlp(hidden=32, seed=11)
        l0 = mo.loss_grad(net.params(), X, Y, M, 32)[0]
        losses.append((l0, net.train(X, Y, M, epochs=80, batch=32, lr=3e-3, seed=5)))
        params.append(net.params())
        net.destroy()
    assert np.array_equal(params[0], params[1])
    l0, l1 = losses[0]
    assert l1 < 0.2 * l0, (l0, l1)
    # the reported loss is the oracle's loss at the trained parameters
    assert abs(mo.loss_grad(params[0], X, Y, M, 32)[0] - l1) <= 1e-4 * l1


def _table():
    path = os.path.join(PKG_DIR, "selector", "tune_table.npz")
    if not os.path.exists(path):
        pytest.fail("selector/tune_table.npz is missing (make it with selector/make_tune_table.py)")
    return dict(np.load(path))


def test_learned_selector_beats_fixed_rules(blco):
    """Train on the sweep table's tensors that are not held out (GPU, this
    library's kernels), choose schedules for the held-out tensors' modes, and compare
    the mean time / best time with the reference's -k 10 rule, this
    library's kernel-10 rule and the same network untrained."""
    T = _table()
    X, ms = T["X"], T["ms"]
    held = T["heldout"]
    Y, M = mo.targets(ms)
    valid = ms > 0

    def choose(pred, rows):
        return mo.choose(pred, valid[rows])[0]

    net0 = blco.Mlp(hidden=64, seed=1)
    untrained = choose(net0.predict(X[held]), held)
    net0.destroy()
    net = blco.Mlp(hidden=64, seed=1)
    loss = net.train(X[~held], Y[~held], M[~held], epochs=300, batch=64, lr=2e-3, seed=0)
    pred = net.predict(X[held])
    learned = choose(pred, held)
    ref_rule = np.array([mo.reference_rule(d, v) for d, v in zip(T["dim"][held], valid[held])])
    auto = np.array([mo.auto_rule(f, v) for f, v in zip(X[held], valid[held])])
    r = dict(learned=mo.regret(ms[held], learned), reference_rule=mo.regret(ms[held], ref_rule),
             auto_rule=mo.regret(ms[held], auto), untrained=mo.regret(ms[held], untrained))
    # with the sweep as fallback when no other schedule group is predicted
    # to be more than the margin slower
    fb, close = mo.choose(pred, valid[held], 0.1, ms=ms[held])
    r["learned_with_fallback"] = mo.regret(ms[held], fb)
    print("held-out rows", int(held.sum()), "train loss", loss, "regret", r, "fallback share", close.mean())
    assert r["learned"] < r["reference_rule"]
    assert r["learned"] < r["untrained"]
    assert r["learned_with_fallback"] <= r["learned"] + 1e-12
    net.destroy()


def test_tuned_kernel_in_cpals(blco):
    """CP-ALS with kernel 20 (the sweep's schedule per mode) follows the
    same fits as with kernel 10."""
    dims = [5_000, 3_000, 80]
    cidx, vals, t = _tensor(blco, dims, 60_000, 0.9, 6)
    R = 16
    rng = np.random.default_rng(7)
    fs0 = [rng.random((d, R)) for d in dims]
    fits = []
    for k in (10, 20):
        f = [x.copy() for x in fs0]
        _, fk = blco.cpals(t, f, np.ones(R), 8, 0.0, blco.make_opts(kernel=k))
        fits.append(np.array(fk))
    assert np.allclose(fits[0], fits[1], rtol=0, atol=1e-10)
    t.free()


def test_committed_selector_is_reproducible_and_used(blco, tmp_path):
    """selector/selector_params.npz is what selector/train_selector.py makes
    on this GPU (bit for bit: training is deterministic), the binary copy
    holds the same parameters, and the default selector drives kernel id 21
    (MTTKRP within 1e-12 of the oracle)."""
    import subprocess
    import sys as _sys
    from conftest import PKG_DIR
    out = tmp_path / "p.npz"
    r = subprocess.run([_sys.executable, os.path.join(PKG_DIR, "selector", "train_selector.py"), "--out", str(out)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    mine = np.load(out)["params"]
    committed = np.load(os.path.join(PKG_DIR, "selector", "selector_params.npz"))
    assert np.array_equal(mine, committed["params"])
    raw = open(os.path.join(PKG_DIR, "selector", "selector_params.bin"), "rb").read()
    hdr = np.frombuffer(raw[:8], dtype="<i4")
    assert hdr[0] == int(committed["hidden"]) and hdr[1] == mine.size
    assert np.array_equal(np.frombuffer(raw[8:], dtype="<f4"), mine)
    net = blco.default_selector(margin=0.1)
    try:
        dims = [30_000, 2_000, 60]
        cidx, vals, t = _tensor(blco, dims, 200_000, 1.0, 1)
        R = 32
        rng = np.random.default_rng(2)
        fs = [rng.random((d, R)) for d in dims]
        for mode in range(3):
            cfg, _ = blco.select(t, mode, R, blco.DTYPE_F64, net, 0.1)
            assert 0 <= cfg < blco.TUNE_CONFIGS
            ref = po.mttkrp_coo(cidx, vals, fs, mode)
            out_t = torch.zeros(dims[mode], R, dtype=torch.float64, device="cuda")
            blco.mttkrp(t, mode, [torch.from_numpy(f).cuda() for f in fs], out_t,
                        blco.make_opts(kernel=blco.KERNEL_LEARNED))
            assert np.linalg.norm(out_t.cpu().numpy() - ref) <= 1e-12 * np.linalg.norm(ref)
        t.free()
    finally:
        blco.selector_set(None)
