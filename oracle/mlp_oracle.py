"""CPU oracle of the schedule selector network (TEST INFRASTRUCTURE ONLY).

A plain numpy FP64 restatement of the network that the library trains and
runs on the GPU (csrc/tune.cu): F inputs -> H (ReLU) -> H (ReLU) -> K
outputs, parameters packed as W1[H][F] b1[H] W2[H][H] b2[H] W3[K][H] b3[K],
loss = sum(mask * (out - Y)^2) / sum(mask).  The selector has no
counterpart in the reference (whose -k 10 rule is fixed,
src/alto_dev.cu:1975,1996-2001), so this file is the only statement of the
arithmetic the GPU kernels are checked against; its own gradient is pinned
by central finite differences in tests/test_oracle_mlp.py.

It also states the two fixed selection rules the learned one is compared
with, over the schedule space of csrc/tune.cu (index: kernel, hot chunk,
tile order):
  0 (1, -, contiguous)  1 (1, -, round-robin)
  2 (2, 512, c)  3 (2, 512, rr)  4 (2, 2048, c)  5 (2, 2048, rr)
  6 (2, 128, c)  7 (2, 128, rr)  8 (3, -, c)  9 (3, -, rr)
  10 (13, -, c)  11 (13, -, rr)
  12 (4, -, strided tasks)  13 (4, -, tasks in stream order)
"""
import numpy as np

F, K = 25, 14


def unpack(p, H, F=F, K=K):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    out = []
    for shape in ((H, F), (H,), (H, H), (H,), (K, H), (K,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    assert o == p.size, (o, p.size)
    return out


def num_params(H, F=F, K=K):
    return H * F + H + H * H + H + K * H + K


def forward(p, X, H):
    W1, b1, W2, b2, W3, b3 = unpack(p, H)
    X = np.asarray(X, dtype=np.float64)
    A1 = np.maximum(X @ W1.T + b1, 0.0)
    A2 = np.maximum(A1 @ W2.T + b2, 0.0)
    out = A2 @ W3.T + b3
    return out, (X, A1, A2)


def loss_grad(p, X, Y, M, H):
    """(loss, gradient as a flat FP64 array in the packed order)."""
    W1, b1, W2, b2, W3, b3 = unpack(p, H)
    out, (X, A1, A2) = forward(p, X, H)
    M = np.asarray(M, dtype=np.float64)
    cnt = M.sum()
    inv = 1.0 / cnt if cnt > 0 else 0.0
    d = M * (out - np.asarray(Y, dtype=np.float64))
    loss = float((d * d).sum() * inv)
    dOut = 2.0 * d * inv
    gW3 = dOut.T @ A2
    gb3 = dOut.sum(0)
    dA2 = (dOut @ W3) * (A2 > 0)
    gW2 = dA2.T @ A1
    gb2 = dA2.sum(0)
    dA1 = (dA2 @ W2) * (A1 > 0)
    gW1 = dA1.T @ X
    gb1 = dA1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


def targets(ms):
    """Training targets from sweep timings ms (n x K, -1 = not valid):
    Y = log2(ms / best), mask = valid."""
    ms = np.asarray(ms, dtype=np.float64)
    valid = ms > 0
    best = np.where(valid, ms, np.inf).min(1, keepdims=True)
    Y = np.where(valid, np.log2(np.where(valid, ms, 1.0) / best), 0.0)
    return Y.astype(np.float32), valid.astype(np.float32)


def reference_rule(dim_t, valid):
    """The reference's -k 10: lvl3 when the target mode has at most 100
    rows, else lvl1 (src/alto_dev.cu:1975,1996-2001), contiguous tiles."""
    return 8 if dim_t <= 100 and valid[8] else 0


def auto_rule(features, valid):
    """This library's kernel 10 (csrc/mttkrp.cu mttkrp_select_kernel and
    auto_hot_chunk): 3 when the output fits in shared memory; else 4 (the
    compressed-fibre kernel, strided tasks) where it applies; else 2 with
    round-robin cold tiles when the mode has at least 2^18 heavy nonzeros,
    with chunk 128 below 2^20 heavy nonzeros, 512 below 2^23, else 2048;
    else 1.  The heavy count is recovered from the features (share x nnz)."""
    if features[23] > 0.5 and valid[8]:
        return 8
    if len(valid) > 12 and valid[12]:
        return 12
    hot = float(features[13]) * 2.0 ** (float(features[0]) * 32.0)
    if features[14] <= 0 or hot < 2 ** 18:
        return 0
    return 7 if hot < 2 ** 20 else 3 if hot < 2 ** 23 else 5


def group(k):
    """Schedules that differ only in tile order form one group."""
    return k // 2


def choose(pred, valid, margin=None, ms=None):
    """The selector's choice per row: the valid schedule with the smallest
    prediction; with a margin, rows whose best prediction is not ahead of
    every other group's by the margin take the sweep's best (ms)."""
    p = np.where(valid, pred, np.inf)
    c = np.argmin(p, axis=1)
    if margin is None:
        return c, np.zeros(len(c), dtype=bool)
    other = p.copy()
    for i, k in enumerate(c):
        other[i, 2 * group(k):2 * group(k) + 2] = np.inf
    close = (other.min(1) - p[np.arange(len(c)), c]) < margin
    swept = np.argmin(np.where(valid, ms, np.inf), axis=1)
    return np.where(close, swept, c), close


def regret(ms, choice):
    """Mean of time(choice) / best time over the rows."""
    ms = np.asarray(ms, dtype=np.float64)
    best = np.where(ms > 0, ms, np.inf).min(1)
    return float(np.mean(ms[np.arange(len(choice)), choice] / best))
