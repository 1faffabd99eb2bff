"""Generate selector/tune_table.npz: autotuner sweep timings and selector
features for synthetic tensors of the selector workload's recipe (runs on a
B200).  The table is the selector's training data (train_selector.py), the
held-out set its regret is measured on, and the data the selector tests use.

Recipe (seed 5), drawn tensor by tensor until a time budget is spent:
order 3-5; mode lengths log-uniform in [1e3, 1e7], redrawn until the
coordinate bits sum to at most 62 (the generator keeps linear keys below
2^63); nnz log-uniform in [1e6, 5e8], at most 1/20 of the cells and at most
--max-nnz (device memory: the encoder's per-mode copies and the autotuner's
factors of a 5-mode tensor take about 200 bytes per nonzero), halved while the
skewed draw cannot reach that many distinct cells; one Zipf exponent per
tensor, U[0, 1.5], on every mode; rank in {16, 32, 64}; one factor dtype per
tensor, uniform over FP64 / FP32 / BF16.  The last --heldout tensors (at most
a third of them) are held out: the shipped selector is trained on the others
and the tests report its regret on these.

Rows: one per (tensor, mode).  Arrays: X (n, 25) features, ms (n, 14)
milliseconds per schedule (-1: not valid), tensor (n,) tensor index, mode,
dim (mode length), rank, dtype, heldout (n,) bool; per tensor: t_dims
(count, 5, 0-padded), t_nnz, t_zipf, t_rank, t_dtype, t_seed (the synthetic
generator's seed, so that a tensor can be made again).

usage: python blocked-linearized-coordinate_b200/selector/make_tune_table.py
           [--budget SECONDS] [--max-count N] [--heldout 200] [--out PATH]
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


def draw_tensor(rng, max_nnz):
    """One tensor of the recipe: (dims, nnz, zipf exponent, rank, dtype)."""
    while True:
        order = int(rng.integers(3, 6))
        dims = [int(round(math.exp(rng.uniform(math.log(1e3), math.log(1e7))))) for _ in range(order)]
        if sum(math.log2(d) for d in dims) <= 62:
            break
    cells = float(np.prod(np.array(dims, dtype=np.float64)))
    nnz = int(math.exp(rng.uniform(math.log(1e6), math.log(5e8))))
    nnz = int(min(nnz, cells // 20, max_nnz))
    s = float(rng.uniform(0.0, 1.5))
    rank = int(rng.choice([16, 32, 64]))
    dtype = int(rng.integers(0, 3))
    return dims, nnz, s, rank, dtype


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--budget", type=float, default=1200.0, help="seconds of sweeping")
    ap.add_argument("--max-count", type=int, default=2200)
    ap.add_argument("--heldout", type=int, default=200)
    ap.add_argument("--max-nnz", type=float, default=4e8)
    ap.add_argument("--out", default=os.path.join(HERE, "tune_table.npz"))
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    import torch
    pkg = load()
    from blco_b200 import synth
    rng = np.random.default_rng(5)
    X, MS, TI, MO, DI, RK, DT = [], [], [], [], [], [], []
    tdims, tnnz, tz, trk, tdt, tseed = [], [], [], [], [], []
    t0 = time.time()
    i = 0
    while i < a.max_count and time.time() - t0 < a.budget:
        dims, nnz, s, rank, dtype = draw_tensor(rng, int(a.max_nnz))
        seed = 5000 + i
        while True:
            try:
                T = synth.zipf_tensor_device(nnz, dims, s, seed=seed, value_dist="uniform")
                break
            except RuntimeError:  # too few distinct cells under this skew
                nnz //= 2
        t = pkg.Tensor.encode_device(dims, T["cidx"], T["vals"])
        del T
        torch.cuda.empty_cache()
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
        tdims.append(dims + [0] * (5 - len(dims)))
        tnnz.append(nnz)
        tz.append(s)
        trk.append(rank)
        tdt.append(dtype)
        tseed.append(seed)
        i += 1
        if i % 20 == 0:
            print(f"{i} tensors, {len(X)} rows, {time.time() - t0:.0f}s", flush=True)
    count = i
    held_from = count - min(a.heldout, count // 3)
    TI = np.array(TI, dtype=np.int32)
    np.savez_compressed(a.out, X=np.array(X, dtype=np.float32), ms=np.array(MS, dtype=np.float32), tensor=TI,
                        mode=np.array(MO, dtype=np.int32), dim=np.array(DI, dtype=np.int64),
                        rank=np.array(RK, dtype=np.int32), dtype=np.array(DT, dtype=np.int32),
                        heldout=TI >= held_from, t_dims=np.array(tdims, dtype=np.int64),
                        t_nnz=np.array(tnnz, dtype=np.int64), t_zipf=np.array(tz, dtype=np.float64),
                        t_rank=np.array(trk, dtype=np.int32), t_dtype=np.array(tdt, dtype=np.int32),
                        t_seed=np.array(tseed, dtype=np.int64))
    print(f"wrote {a.out}: {len(X)} rows from {count} tensors ({count - held_from} held out) "
          f"in {time.time() - t0:.0f}s")


if __name__ == "__main__":
    main()
