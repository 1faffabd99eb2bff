"""Train the MTTKRP schedule selector on the committed sweep table and save
its parameters (runs on a B200: training uses this library's GPU kernels).

  python blocked-linearized-coordinate_b200/selector/train_selector.py [--out PATH]

The network (64 hidden units) is trained on the rows of tune_table.npz that
are not held out (the table's `heldout` flags) for 300 epochs (batch 64,
Adam lr 2e-3, seed 0), the settings whose held-out regret the selector tests
and selector/eval_selector.py measure; the result is deterministic for the
seed.
selector_params.npz holds the flat parameter array, the hidden width and
the final training loss; selector_params.bin holds the same parameters for
C and C++ callers: int32 hidden width, int32 parameter count, then the
parameters as little-endian float32 (cpd64 --selector reads it).
"""
import argparse
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)

HIDDEN, EPOCHS, BATCH, LR, SEED = 64, 300, 64, 2e-3, 0


def load():
    if "blco_b200" in sys.modules:
        return sys.modules["blco_b200"]
    spec = importlib.util.spec_from_file_location("blco_b200", os.path.join(PKG, "__init__.py"),
                                                  submodule_search_locations=[PKG])
    m = importlib.util.module_from_spec(spec)
    sys.modules["blco_b200"] = m
    spec.loader.exec_module(m)
    return m


def targets(ms):
    """Y = log2(ms / best) per row, mask = the schedules that ran (ms > 0)."""
    ms = np.asarray(ms, dtype=np.float64)
    valid = ms > 0
    best = np.where(valid, ms, np.inf).min(1, keepdims=True)
    Y = np.where(valid, np.log2(np.where(valid, ms, 1.0) / best), 0.0)
    return Y.astype(np.float32), valid.astype(np.float32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--table", default=os.path.join(HERE, "tune_table.npz"))
    ap.add_argument("--out", default=os.path.join(HERE, "selector_params.npz"))
    a = ap.parse_args()
    pkg = load()
    T = dict(np.load(a.table))
    train = ~T["heldout"] if "heldout" in T else np.ones(len(T["ms"]), dtype=bool)
    Y, M = targets(T["ms"][train])
    net = pkg.Mlp(hidden=HIDDEN, seed=1)
    loss = net.train(T["X"][train], Y, M, epochs=EPOCHS, batch=BATCH, lr=LR, seed=SEED)
    params = net.params()
    np.savez(a.out, params=params, hidden=np.int32(HIDDEN), loss=np.float32(loss))
    binp = os.path.splitext(a.out)[0] + ".bin"
    with open(binp, "wb") as f:
        f.write(np.array([HIDDEN, params.size], dtype="<i4").tobytes())
        f.write(params.astype("<f4").tobytes())
    print(f"trained on {len(Y)} rows: loss {loss:.5f}; wrote {a.out} and {binp}")
    net.destroy()


if __name__ == "__main__":
    main()
