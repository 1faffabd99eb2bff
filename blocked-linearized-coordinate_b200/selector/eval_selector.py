"""Evaluate the shipped schedule selector on the held-out tensors of
selector/tune_table.npz (runs on a B200) and write selector/eval.json.

  python blocked-linearized-coordinate_b200/selector/eval_selector.py [--fit-tensors 20] [--iters 10]

Regret (mean of time(choice) / best time over the held-out modes, from the
table's sweep timings): the shipped network alone, the network with the
sweep as fallback (margin 0.1), this library's kernel-10 rule, the
reference's -k 10 rule (src/alto_dev.cu:1975,1996-2001).  Fit: for the
first --fit-tensors held-out tensors (made again from their recorded
generator parameters), CP-ALS in the mixed form with the learned schedule
(kernel id 21) against the FP64 form with kernel 10, same initial factors,
--iters iterations (40): |fit difference| per tensor at the end and after
10 iterations, and whether the mixed plan's condition guard moved it to
FP64.
"""
import argparse
import importlib.util
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)


def load():
    spec = importlib.util.spec_from_file_location("blco_b200", os.path.join(PKG, "__init__.py"),
                                                  submodule_search_locations=[PKG])
    m = importlib.util.module_from_spec(spec)
    sys.modules["blco_b200"] = m
    spec.loader.exec_module(m)
    return m


def regret(ms, choice):
    ms = np.asarray(ms, dtype=np.float64)
    best = np.where(ms > 0, ms, np.inf).min(1)
    return float(np.mean(ms[np.arange(len(choice)), choice] / best))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--table", default=os.path.join(HERE, "tune_table.npz"))
    ap.add_argument("--out", default=os.path.join(HERE, "eval.json"))
    ap.add_argument("--params", default=None, help="trained selector (default: the committed one)")
    ap.add_argument("--fit-tensors", type=int, default=20)
    ap.add_argument("--iters", type=int, default=40)
    a = ap.parse_args()
    import torch
    pkg = load()
    from blco_b200 import synth
    T = dict(np.load(a.table))
    held = T["heldout"]
    X, ms = T["X"][held], T["ms"][held]
    valid = ms > 0
    net = pkg.default_selector(margin=0.1, path=a.params)
    pred = net.predict(X)
    p = np.where(valid, pred, np.inf)
    learned = np.argmin(p, axis=1)
    # the fallback rule of kernel id 21: the sweep unless another schedule
    # group is predicted slower by the margin (groups: 2k, 2k + 1)
    other = p.copy()
    for i, k in enumerate(learned):
        other[i, 2 * (k // 2):2 * (k // 2) + 2] = np.inf
    close = (other.min(1) - p[np.arange(len(learned)), learned]) < 0.1
    swept = np.argmin(np.where(valid, ms, np.inf), axis=1)
    fallback = np.where(close, swept, learned)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    out = dict(heldout_tensors=int(np.unique(T["tensor"][held]).size), heldout_modes=int(held.sum()),
               train_tensors=int(np.unique(T["tensor"][~held]).size),
               regret=dict(learned=regret(ms, learned), learned_with_fallback=regret(ms, fallback),
                           fallback_share=float(close.mean())))
    # the fixed rules as csrc/mttkrp.cu and the reference state them
    auto = []
    for f, v in zip(X, valid):
        if f[23] > 0.5 and v[8]:
            auto.append(8)
        elif v[12]:
            auto.append(12)
        else:
            hot = float(f[13]) * 2.0 ** (float(f[0]) * 32.0)
            auto.append(0 if (f[14] <= 0 or hot < 2 ** 18) else 7 if hot < 2 ** 20 else 3 if hot < 2 ** 23 else 5)
    ref = [8 if d <= 100 and v[8] else 0 for d, v in zip(T["dim"][held], valid)]
    out["regret"]["auto_rule"] = regret(ms, np.array(auto))
    out["regret"]["reference_rule"] = regret(ms, np.array(ref))
    print(json.dumps(out["regret"]), flush=True)
    # fit of the mixed form with the learned schedule against FP64
    pkg.selector_set(net, 0.1)
    fits = []
    ids = np.unique(T["tensor"][held])[:a.fit_tensors]
    for ti in ids:
        dims = [int(d) for d in T["t_dims"][ti] if d > 0]
        nnz, s, R = int(T["t_nnz"][ti]), float(T["t_zipf"][ti]), int(T["t_rank"][ti])
        Xt = synth.zipf_tensor_device(nnz, dims, s, seed=int(T["t_seed"][ti]), value_dist="uniform")
        t = pkg.Tensor.encode_device(dims, Xt["cidx"], Xt["vals"])
        del Xt
        res = {}
        for name, prec, k in (("fp64", pkg.PRECISION_FP64, 10), ("mixed", pkg.PRECISION_MIXED, 21)):
            g = torch.Generator(device="cuda").manual_seed(int(ti))
            fs = [torch.rand(d, R, dtype=torch.float64, device="cuda", generator=g) for d in dims]
            lam = torch.ones(R, dtype=torch.float64, device="cuda")
            plan = pkg.CpalsPlan(t, fs, lam, pkg.make_opts(kernel=k, precision=prec))
            w0 = time.time()
            f = plan.iterate(a.iters, tol=-1.0)
            torch.cuda.synchronize()
            _, promoted = plan.condition()
            res[name] = (float(f[-1]), time.time() - w0, float(f[min(10, len(f)) - 1]), bool(promoted))
            plan.destroy()
        t.free()
        torch.cuda.empty_cache()
        d = abs(res["mixed"][0] - res["fp64"][0])
        d10 = abs(res["mixed"][2] - res["fp64"][2])
        fits.append(dict(tensor=int(ti), dims=dims, nnz=nnz, zipf=s, rank=R, fit_fp64=res["fp64"][0],
                         fit_mixed=res["mixed"][0], abs_diff=d, abs_diff_at_10=d10,
                         mixed_promoted_to_fp64=res["mixed"][3]))
        print(f"tensor {ti}: dims {dims} nnz {nnz} R {R} fit fp64 {res['fp64'][0]:.9f} mixed "
              f"{res['mixed'][0]:.9f} |diff| {d:.2e} (at 10: {d10:.2e}) promoted {res['mixed'][3]}", flush=True)
    pkg.selector_set(None)
    out["fit"] = dict(iters=a.iters, tensors=fits, max_abs_diff=max([x["abs_diff"] for x in fits] or [0.0]),
                      max_abs_diff_at_10=max([x["abs_diff_at_10"] for x in fits] or [0.0]),
                      promoted=sum(x["mixed_promoted_to_fp64"] for x in fits))
    with open(a.out, "w") as fo:
        json.dump(out, fo, indent=1)
    print("wrote", a.out, "max |fit diff|", out["fit"]["max_abs_diff"])


if __name__ == "__main__":
    main()
