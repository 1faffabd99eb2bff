"""Profiling drivers (run under ncu or alone) for the two benchmark paths.

  python blocked-linearized-coordinate_b200/prof.py mttkrp --nnz N --dtype f32|f64|bf16 [--kernel K] [--reps R]
      One MTTKRP per mode of the Zipf(1.1) 2M x 2M x 25k tensor (rank 32),
      timed with CUDA events; factors in the requested dtype.
  python blocked-linearized-coordinate_b200/prof.py batch --count T [--iters I]
      Batched CP-ALS sweeps over T small tensors of the many-small-tensors
      recipe (FP64); prints device ms per sweep.
  python blocked-linearized-coordinate_b200/prof.py cpals --nnz N --dtype f64|f32|bf16 [--iters I]
      CP-ALS iterations on the Zipf(1.1) 2M x 2M x 25k tensor (rank 32):
      ms per iteration, MTTKRP ms per mode, and the rest of the iteration.
  python blocked-linearized-coordinate_b200/prof.py stream --nnz N [--block B] [--residency BYTES] [--dtype f64|f32] [--no-dedupe]
      The streamed form on the 4-mode 500k x 200k x 50k x 1k Zipf(0.9) shape,
      rank 64, FP64: ms per CP-ALS iteration and host-to-device GB/s against
      a measured pinned copy.
  python blocked-linearized-coordinate_b200/prof.py wide --nnz N [--rank R] [--reps K] [--iters I]
      The wide-key workload: Zipf(1.1) over 2^20 x 2^20 x 2^20 x 4096
      (72 key bits, the reference's 128-bit build), FP64: encode time and
      block count, per-mode MTTKRP times, CP-ALS ms per iteration.
  python blocked-linearized-coordinate_b200/prof.py tns --nnz N --dir D
      Writes the Zipf(1.1) 2M x 2M x 25k tensor with N nonzeros as a .tns
      file (cpd64's writer, values as %g) and times cpd64's file-to-BLCO
      step with the GPU loader and with the host loader (--host-load).
"""
import argparse
import importlib.util
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))


def load():
    if "blco_b200" in sys.modules:
        return sys.modules["blco_b200"]
    spec = importlib.util.spec_from_file_location("blco_b200", os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    m = importlib.util.module_from_spec(spec)
    sys.modules["blco_b200"] = m
    spec.loader.exec_module(m)
    return m


def run_mttkrp(a, pkg, torch):
    from blco_b200 import synth
    dims = [2_000_000, 2_000_000, 25_000]
    X = synth.zipf_tensor_device(a.nnz, dims, 1.1, seed=0)
    t = pkg.Tensor.encode_device(dims, X["cidx"], X["vals"])
    del X
    torch.cuda.empty_cache()
    R = a.rank
    g = torch.Generator(device="cuda").manual_seed(1)
    fs = [torch.rand(d, R, dtype=torch.float64, device="cuda", generator=g) for d in dims]
    if a.dtype != "f64":
        fs = [f.to(torch.float32 if a.dtype == "f32" else torch.bfloat16) for f in fs]
        fd = pkg.DTYPE_F32 if a.dtype == "f32" else pkg.DTYPE_BF16
    o = pkg.make_opts(kernel=a.kernel)
    for m in range(3):
        out = torch.zeros(dims[m], R, dtype=torch.float64 if a.dtype == "f64" else torch.float32, device="cuda")
        ts = []
        for _ in range(a.reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            if a.dtype == "f64":
                pkg.mttkrp(t, m, fs, out, o)
            else:
                pkg.mttkrp_ex(t, m, fs, out, fd, o)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        print(f"mode {m}: ms {['%.3f' % x for x in ts]}", flush=True)
    t.free()


def run_cpals(a, pkg, torch):
    from blco_b200 import synth
    dims = [2_000_000, 2_000_000, 25_000]
    X = synth.zipf_tensor_device(a.nnz, dims, 1.1, seed=0)
    t = pkg.Tensor.encode_device(dims, X["cidx"], X["vals"])
    del X
    torch.cuda.empty_cache()
    R = a.rank
    g = torch.Generator(device="cuda").manual_seed(1234)
    fs = [torch.rand(d, R, dtype=torch.float64, device="cuda", generator=g) for d in dims]
    lam = torch.ones(R, dtype=torch.float64, device="cuda")
    prec = {"f64": pkg.PRECISION_FP64, "f32": pkg.PRECISION_MIXED, "bf16": pkg.PRECISION_MIXED_BF16}[a.dtype]
    plan = pkg.CpalsPlan(t, fs, lam, pkg.make_opts(kernel=a.kernel, precision=prec))
    plan.iterate(3, tol=-1.0)
    ms0, c0 = plan.mttkrp_ms()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    fits = plan.iterate(a.iters, tol=-1.0)
    e1.record()
    torch.cuda.synchronize()
    ms1, c1 = plan.mttkrp_ms()
    per = (ms1 - ms0) / max(1, c1 - c0)
    it = e0.elapsed_time(e1) / a.iters
    print(f"cpals {a.dtype} ms/iter {it:.3f} mttkrp ms/mode {['%.3f' % x for x in per]} "
          f"rest ms/iter {it - sum(per):.3f} fit {fits[-1]:.9f}", flush=True)
    plan.destroy()
    t.free()


def run_stream(a, pkg, torch):
    """The streamed (out-of-memory) form on the 4-mode Zipf(0.9) shape
    500k x 200k x 50k x 1k, rank 64, FP64: blocks of --block nonzeros in
    pinned host memory, copied through a ring of at most --residency bytes;
    host-to-device GB/s per CP-ALS iteration against a pinned copy."""
    from blco_b200 import synth
    dims = [500_000, 200_000, 50_000, 1_000]
    if a.no_dedupe:
        X = synth.zipf_coo_device(a.nnz, dims, 0.9, seed=0)
    else:
        X = synth.zipf_tensor_device(a.nnz, dims, 0.9, seed=0, value_dist="uniform")
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    # pinned host-to-device peak: 2 GiB, best of 3
    hb = torch.empty(1 << 28, dtype=torch.float64).pin_memory()
    db = torch.empty(1 << 28, dtype=torch.float64, device="cuda")
    best = 0.0
    for _ in range(3):
        e0.record()
        db.copy_(hb, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, hb.numel() * 8 / (e0.elapsed_time(e1) * 1e-3) / 1e9)
    del hb, db
    prec = {"f64": pkg.PRECISION_FP64, "f32": pkg.PRECISION_MIXED}[a.dtype]
    o = pkg.make_opts(kernel=10, stream_data=True, residency_bytes=a.residency, precision=prec)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()  # the generator's cached blocks
    t0 = time.perf_counter()
    t = pkg.Tensor.encode_device(dims, X["cidx"], X["vals"], a.block, o)
    encode_s = time.perf_counter() - t0
    del X
    torch.cuda.empty_cache()
    inf = t.info()
    R = a.rank
    g = torch.Generator(device="cuda").manual_seed(1234)
    fs = [torch.rand(d, R, dtype=torch.float64, device="cuda", generator=g) for d in dims]
    lam = torch.ones(R, dtype=torch.float64, device="cuda")
    plan = pkg.CpalsPlan(t, fs, lam, o)
    plan.iterate(1, tol=-1.0)
    torch.cuda.synchronize()
    free_b, total_b = torch.cuda.mem_get_info()
    e0.record()
    fits = plan.iterate(a.iters, tol=-1.0)
    e1.record()
    torch.cuda.synchronize()
    it = e0.elapsed_time(e1) / a.iters
    h2d = len(dims) * a.nnz * (16 if a.dtype == "f64" else 12)
    print(f"streamed {a.dtype} nnz {a.nnz} blocks {inf['block_count']} residency {a.residency} ms/iter {it:.1f} "
          f"h2d GB/iter {h2d / 1e9:.2f} h2d GB/s {h2d / (it * 1e-3) / 1e9:.1f} pinned peak GB/s {best:.1f} "
          f"frac {h2d / (it * 1e-3) / 1e9 / best:.3f} device GB in use {(total_b - free_b) / 1e9:.1f} "
          f"fit {fits[-1]:.6f} encode s {encode_s:.2f}", flush=True)
    plan.destroy()
    t.free()


WIDE_DIMS = [1 << 20, 1 << 20, 1 << 20, 1 << 12]  # 72 key bits


def run_wide(a, pkg, torch):
    from blco_b200 import synth
    dims = WIDE_DIMS
    X = synth.wide_tensor_device(a.nnz, dims, 1.1, seed=0)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    t = pkg.Tensor.encode_device(dims, X["cidx"], X["vals"])
    e1.record()
    torch.cuda.synchronize()
    del X
    torch.cuda.empty_cache()
    inf = t.info()
    print(f"encode ms {e0.elapsed_time(e1):.3f} blocks {inf['block_count']} key bits {inf['alto_bits']}", flush=True)
    R = a.rank
    g = torch.Generator(device="cuda").manual_seed(1)
    fs = [torch.rand(d, R, dtype=torch.float64, device="cuda", generator=g) for d in dims]
    o = pkg.make_opts(kernel=10)
    for m in range(len(dims)):
        out = torch.zeros(dims[m], R, dtype=torch.float64, device="cuda")
        pkg.mttkrp(t, m, fs, out, o)
        ts = []
        for _ in range(a.reps):
            e0.record()
            pkg.mttkrp(t, m, fs, out, o)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        alg = a.nnz * 16 + sum(d * R * 8 for d in dims)
        best = min(ts)
        print(f"mode {m}: ms {['%.3f' % x for x in ts]} alg GB/s {alg / best / 1e6:.0f}", flush=True)
    f32 = [f.float() for f in fs]
    for m in range(len(dims)):
        out = torch.zeros(dims[m], R, dtype=torch.float32, device="cuda")
        pkg.mttkrp_ex(t, m, f32, out, pkg.DTYPE_F32, o)
        ts = []
        for _ in range(a.reps):
            e0.record()
            pkg.mttkrp_ex(t, m, f32, out, pkg.DTYPE_F32, o)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        print(f"mode {m} f32: ms {['%.3f' % x for x in ts]}", flush=True)
    del f32
    if a.iters:
        for name, prec in (("fp64", pkg.PRECISION_FP64), ("mixed_f32", pkg.PRECISION_MIXED)):
            lam = torch.ones(R, dtype=torch.float64, device="cuda")
            plan = pkg.CpalsPlan(t, [f.clone() for f in fs], lam, pkg.make_opts(kernel=10, precision=prec))
            plan.iterate(2, tol=-1.0)
            e0.record()
            fits = plan.iterate(a.iters, tol=-1.0)
            e1.record()
            torch.cuda.synchronize()
            ms, calls = plan.mttkrp_ms()
            print(f"cpals {name} ms/iter {e0.elapsed_time(e1) / a.iters:.3f} fit {fits[-1]:.9f} "
                  f"mttkrp ms/mode (all calls) {['%.3f' % (x / max(1, calls)) for x in ms]}", flush=True)
            plan.destroy()
    t.free()


def run_batch(a, pkg, torch):
    from blco_b200 import synth
    Xs = synth.batch_tensors_device(a.count, seed=0)
    ts = [pkg.Tensor.encode_device(x["dims"], x["cidx"], x["vals"]) for x in Xs]
    g = torch.Generator(device="cuda").manual_seed(1)
    fs = [[torch.rand(d, x["rank"], dtype=torch.float64, device="cuda", generator=g) for d in x["dims"]] for x in Xs]
    ls = [torch.ones(x["rank"], dtype=torch.float64, device="cuda") for x in Xs]
    del Xs
    b = pkg.Batch(ts, fs, ls, tol=0.0)
    b.iterate(2)
    b.iterate(a.iters)
    print("batched ms/sweep %.3f" % (b.last_ms() / a.iters), flush=True)
    b.destroy()
    for t in ts:
        t.free()


def run_tns(a, pkg, torch):
    import re
    import subprocess
    import numpy as np
    from blco_b200 import synth
    dims = [2_000_000, 2_000_000, 25_000]
    X = synth.zipf_tensor_device(a.nnz, dims, 1.1, seed=0)
    os.makedirs(a.dir, exist_ok=True)
    binp = os.path.join(a.dir, "t.bin")
    with open(binp, "wb") as f:
        np.array([3], dtype=np.uint64).tofile(f)
        np.array(dims, dtype=np.uint64).tofile(f)
        np.array([a.nnz], dtype=np.uint64).tofile(f)
        for c in X["cidx"]:
            c.to(torch.int64).cpu().numpy().astype(np.uint64).tofile(f)
        X["vals"].cpu().numpy().tofile(f)
    del X
    cpd = os.path.join(HERE, "bin", "cpd64")
    subprocess.run([cpd, "-b", binp, "-f", "1"], capture_output=True, text=True)
    tns = binp + ".tns"
    size = os.path.getsize(tns)
    for mode, extra in (("gpu", []), ("host", ["--host-load"])):
        r = subprocess.run([cpd, "-i", tns, "-k", "10", "-m", "0", "-r", "8", "-x", "1"] + extra,
                           capture_output=True, text=True)
        if r.returncode != 0:
            print(mode, "failed:", r.stderr[-500:])
            continue
        rd = float(re.search(r"Reading tensor file\]: ([0-9.]+)", r.stdout).group(1))
        enc = float(re.search(r"encode time = ([0-9.]+)", r.stdout).group(1))
        total = rd if mode == "gpu" else rd + enc
        print(f"{mode} loader: {size / 1e9:.2f} GB file, {a.nnz} nonzeros: file to BLCO {total:.3f} s "
              f"(read {rd:.3f} s, encode {enc:.3f} s)", flush=True)


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    m = sub.add_parser("mttkrp")
    m.add_argument("--nnz", type=int, default=20_000_000)
    m.add_argument("--dtype", default="f32", choices=["f64", "f32", "bf16"])
    m.add_argument("--kernel", type=int, default=10)
    m.add_argument("--reps", type=int, default=1)
    m.add_argument("--rank", type=int, default=32)
    b = sub.add_parser("batch")
    b.add_argument("--count", type=int, default=64)
    b.add_argument("--iters", type=int, default=1)
    tn = sub.add_parser("tns")
    tn.add_argument("--nnz", type=int, default=50_000_000)
    tn.add_argument("--dir", default="tns_prof")
    c = sub.add_parser("cpals")
    c.add_argument("--nnz", type=int, default=200_000_000)
    c.add_argument("--dtype", default="f32", choices=["f64", "f32", "bf16"])
    c.add_argument("--kernel", type=int, default=10)
    c.add_argument("--rank", type=int, default=32)
    c.add_argument("--iters", type=int, default=10)
    sm = sub.add_parser("stream")
    sm.add_argument("--nnz", type=int, default=500_000_000)
    sm.add_argument("--rank", type=int, default=64)
    sm.add_argument("--block", type=int, default=64 << 20)
    sm.add_argument("--residency", type=int, default=8 << 30)
    sm.add_argument("--iters", type=int, default=2)
    sm.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    sm.add_argument("--no-dedupe", action="store_true",
                    help="draw the COO chunk by chunk without removing repeated coordinates")
    w = sub.add_parser("wide")
    w.add_argument("--nnz", type=int, default=50_000_000)
    w.add_argument("--rank", type=int, default=32)
    w.add_argument("--reps", type=int, default=3)
    w.add_argument("--iters", type=int, default=3)
    a = ap.parse_args()
    import torch
    pkg = load()
    if os.environ.get("BLCO_LIB"):
        pkg.LIB_PATH = os.environ["BLCO_LIB"]
    {"mttkrp": run_mttkrp, "batch": run_batch, "tns": run_tns, "wide": run_wide,
     "cpals": run_cpals, "stream": run_stream}[a.cmd](a, pkg, torch)


if __name__ == "__main__":
    main()
