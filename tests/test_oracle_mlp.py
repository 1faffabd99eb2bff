"""CPU tests of the selector network's oracle (oracle/mlp_oracle.py): its
analytic gradient against central finite differences, and the fixed
selection rules on hand-made rows."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import mlp_oracle as mo  # noqa: E402


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    H, n = 7, 9
    p = rng.normal(scale=0.5, size=mo.num_params(H))
    X = rng.normal(size=(n, mo.F))
    Y = rng.normal(size=(n, mo.K))
    M = (rng.random((n, mo.K)) > 0.3).astype(np.float64)
    loss, g = mo.loss_grad(p, X, Y, M, H)
    assert g.shape == p.shape and loss > 0
    eps = 1e-6
    idx = rng.choice(p.size, size=60, replace=False)
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp, _ = mo.loss_grad(q, X, Y, M, H)
        q[i] -= 2 * eps
        lm, _ = mo.loss_grad(q, X, Y, M, H)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_targets_and_rules():
    # schedules 12 and 13 (the compressed-fibre kernel) do not apply in row 0
    ms = np.array([[2.0, 1.0, -1, 4.0, 4, 4, 4, 4, -1, -1, 8, 8, -1, -1],
                   [1.0, 1.0, 1, 1, 1, 1, 1, 1, 0.5, 0.25, 1, 1, 0.75, 0.8]], dtype=np.float32)
    Y, M = mo.targets(ms)
    assert M[0, 2] == 0 and M[0, 8] == 0 and M[0, 12] == 0 and M[1].all()
    assert Y[0, 1] == 0 and abs(Y[0, 0] - 1.0) < 1e-7 and abs(Y[1, 0] - 2.0) < 1e-7
    valid0, valid1 = ms[0] > 0, ms[1] > 0
    assert mo.reference_rule(50, valid0) == 0          # kernel 3 not valid there
    assert mo.reference_rule(50, valid1) == 8
    assert mo.reference_rule(1000, valid1) == 0
    f = np.zeros(mo.F)
    f[23] = 1.0
    assert mo.auto_rule(f, valid1) == 8                # output in shared memory first
    f[23] = 0.0
    assert mo.auto_rule(f, valid1) == 12               # then the fibre kernel where it applies
    f[14] = 0.5
    f[0] = np.log2(4e6) / 32     # 4M nonzeros, half of them heavy
    f[13] = 0.5
    assert mo.auto_rule(f, valid0) == 3
    f[13] = 0.05                 # 200k heavy: below the threshold
    assert mo.auto_rule(f, valid0) == 0
    pred = np.array([[0.0, 0.01, 0.5, 0.5, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1]])
    c, close = mo.choose(pred, np.ones((1, 14), bool))
    assert c[0] == 0 and not close[0]
    # the twin (same group) does not count against the margin
    c, close = mo.choose(pred, np.ones((1, 14), bool), 0.3, ms=np.arange(14.0)[None, ::-1] + 1)
    assert c[0] == 0 and not close[0]
    c, close = mo.choose(pred, np.ones((1, 14), bool), 0.6, ms=np.arange(14.0)[None, ::-1] + 1)
    assert close[0] and c[0] == 13
    assert abs(mo.regret(ms, np.array([1, 9])) - 1.0) < 1e-12
    assert abs(mo.regret(ms, np.array([0, 0])) - (2.0 + 4.0) / 2) < 1e-12
