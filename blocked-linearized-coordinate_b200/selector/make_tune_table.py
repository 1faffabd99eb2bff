"""Generate selector/tune_table.npz: autotuner sweep timings and selector
features for a set of synthetic tensors (runs on a B200).  The table is the
selector's training data (train_selector.py) and the fixed data the
selector tests train on.

The tensors follow the selector workload's recipe at reduced size so the
sweep finishes in minutes: order 3-5; mode lengths log-uniform in
[50, 1e6] (down to 50 so that the shared-memory schedule applies to some
modes) with the total coordinate bits at most 64; nnz log-uniform in
[1e5, 1e7] (the full recipe uses 1e6-5e8), at most 1/20 of the cells
(halved while the skewed draw cannot reach that many distinct cells);
per-tensor Zipf exponent U[0, 1.5] on every mode; rank in {16, 32, 64};
one factor dtype per tensor, uniform over FP64 / FP32 / BF16; seed 5.

Rows: one per (tensor, mode).  Arrays: X (n, 25) features, ms (n, 12)
milliseconds per schedule (-1: not valid), tensor (n,) tensor index,
mode, dim (mode length), rank, dtype.

usage: python blocked-linearized-coordinate_b200/selector/make_tune_table.py [--count 240] [--out PATH]
"""
import argparse
import importlib.util
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)


def load():
    spec = importlib.util.spec_from_file_location("blco_b200", os.path.join(PKG, "__init__.py"),
                                                  submodule_search_locations=[PKG])
    m = importlib.util.module_from_spec(spec)
    sys.modules["blco_b200"] = m
    spec.loader.exec_module(m)
    return m


def draw_shape(rng):
    while True:
        order = int(rng.integers(3, 6))
        dims = [int(round(math.exp(rng.uniform(math.log(50), math.log(1e6))))) for _ in range(order)]
        bits = sum(max(1, (d - 1).bit_length()) for d in dims)
        if bits <= 62:
            return dims


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=240)
    ap.add_argument("--out", default=os.path.join(HERE, "tune_table.npz"))
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    import torch
    pkg = load()
    from blco_b200 import synth
    rng = np.random.default_rng(5)
    X, MS, TI, MO, DI, RK, DT = [], [], [], [], [], [], []
    t0 = time.time()
    for i in range(a.count):
        dims = draw_shape(rng)
        cells = float(np.prod(np.array(dims, dtype=np.float64)))
        nnz = int(math.exp(rng.uniform(math.log(1e5), math.log(1e7))))
        nnz = int(min(nnz, cells // 20))
        s = float(rng.uniform(0.0, 1.5))
        rank = int(rng.choice([16, 32, 64]))
        dtype = int(rng.integers(0, 3))
        while True:
            try:
                T = synth.zipf_tensor_device(nnz, dims, s, seed=5000 + i, value_dist="uniform")
                break
            except RuntimeError:  # too few distinct cells under this skew
                nnz //= 2
        t = pkg.Tensor.encode_device(dims, T["cidx"], T["vals"])
        del T
        for m in range(len(dims)):
            f = pkg.tune_features(t, m, rank, dtype)
            ms, _ = pkg.autotune(t, m, rank, dtype, reps=a.reps)
            X.append(f)
            MS.append(ms)
            TI.append(i)
            MO.append(m)
            DI.append(dims[m])
            RK.append(rank)
            DT.append(dtype)
        t.free()
        torch.cuda.empty_cache()
        if i % 20 == 0:
            print(f"{i} tensors, {len(X)} rows, {time.time() - t0:.0f}s", flush=True)
    np.savez_compressed(a.out, X=np.array(X, dtype=np.float32), ms=np.array(MS, dtype=np.float32),
                        tensor=np.array(TI, dtype=np.int32), mode=np.array(MO, dtype=np.int32),
                        dim=np.array(DI, dtype=np.int64), rank=np.array(RK, dtype=np.int32),
                        dtype=np.array(DT, dtype=np.int32))
    print(f"wrote {a.out}: {len(X)} rows from {a.count} tensors in {time.time() - t0:.0f}s")


if __name__ == "__main__":
    main()
