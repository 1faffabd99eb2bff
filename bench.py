"""CP-ALS benchmark on the Zipf(1.1) 2M x 2M x 25k, 200M-nonzero, rank-32
workload, one B200 per rank.  The plain FP64 form and the mixed-precision
forms run on the same tensor and initial factors; the headline value is the
fastest mixed form whose final fit is within 1e-5 of the FP64 form's.  The
fits are compared after --fit-iters (40) iterations of the same run (the
timed steps, then untimed ones): while the fit still climbs steeply (about
5e-4 per iteration near iteration 10), the mixed forms' trajectories run a
little ahead of or behind the FP64 one, by up to a few 1e-5, and meet it
again near convergence; the largest gap over the run and the gap at the end
of the timed steps are reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one CP-ALS iteration: MTTKRP of all three modes, the R x R
solves, factor updates, normalisation, Grams and the fit.  Prints one JSON
line (rank 0).  Inputs (3.2 GB stream + 1 GB of factors) are larger than
the 126 MB L2, so no flush is needed between steps.

--impl reference times the reference's own CPU CP-ALS (cpd_alto,
include/cpd.hpp, compiled from the reference sources into oracle/_ref with
scipy's OpenBLAS) on the whole workload with all host threads (about 2.8 s
per iteration), and on the CPU-runnable workload (`c1`); it also runs the
reference's own GPU code on the full workload (`reference_gpu`) with a
full-size fit comparison against this engine's plain form.

Two more legs ride on the same line (skip with --no-batched / --no-wide):
`batched`, batched CP-ALS of 512 small tensors, and `wide`, FP64 CP-ALS of a
100M-nonzero tensor whose keys need 72 bits (the reference's 128-bit build),
with its own roofline and CPU baseline.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

WORKLOAD = dict(workload="cpals_zipf1.1_2Mx2Mx25k_nnz200M_r32", dims=[2_000_000, 2_000_000, 25_000],
                nnz=200_000_000, rank=32, zipf=1.1, values="lognormal(0,1) fp32 summed over duplicates, fp64")
METRIC = "CP-ALS ms/iter"


def gather_ceiling():
    """Random 128-byte factor-row gathers per second on this GPU's load path
    (blocked-linearized-coordinate_b200/bin/gather_ceiling: Zipf(1.1) over 2M
    rows, the workload's per-mode distribution), measured live."""
    exe = os.path.join(ROOT, "blocked-linearized-coordinate_b200", "bin", "gather_ceiling")
    if not os.path.exists(exe):
        return None
    try:
        r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
        return json.loads(r.stdout.strip().splitlines()[-1]) if r.returncode == 0 else None
    except Exception:
        return None


def load_pkg():
    import __graft_entry__ as ge
    return ge._load()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def mttkrp_alg_bytes(dims, nnz, R, mode, s_idx=8, s_val=8, s_fac=8, s_out=8):
    """Algorithmic bytes of one mode-t MTTKRP: the index/value stream once,
    every input factor once and the output once."""
    b = nnz * (s_idx + s_val) + dims[mode] * R * s_out
    for m, d in enumerate(dims):
        if m != mode:
            b += d * R * s_fac
    return b


def traffic_from_profiles(form, nnz, name=None, full_nnz=None):
    """DRAM bytes per MTTKRP (all kernels of one mode, mean over the modes)
    at the full-size workload, from the committed ncu summary of the chosen
    form (or the summary `name`), if there is one."""
    if nnz != (full_nnz or WORKLOAD["nnz"]):
        return None
    p = os.path.join(ROOT, "profiles", name or f"mttkrp_{form}_zipf_2Mx2Mx25k_r32.md")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            if line.startswith("traffic_bytes_per_mttkrp_full_size:"):
                try:
                    return float(line.split(":", 1)[1].strip())
                except ValueError:
                    return None
    return None


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].strip() == "Active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return dict(sm_mhz=statistics.median(sm), sm_max_mhz=mx, reasons=sorted(reasons), samples=len(sm))


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def all_ranks(x, dist, device="cuda"):
    """Every rank's value of a per-rank float, in rank order ([x] without a
    process group)."""
    if not dist:
        return [float(x)]
    import torch
    tt = torch.zeros(dist.get_world_size(), dtype=torch.float64, device=device)
    tt[dist.get_rank()] = float(x)
    dist.all_reduce(tt)
    return [float(v) for v in tt.tolist()]


def max_over_ranks(x, dist, device="cuda"):
    """The maximum of a per-rank float over all ranks (identity without a
    process group); `device` is where the collective's tensor lives (cuda for
    NCCL, cpu for gloo)."""
    if not dist:
        return x
    import torch
    tt = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return tt.item()


def _ref_fits(log):
    import re
    return [float(x) for x in re.findall(r"--> Iter +\d+: f = ([0-9.eE+-]+)", log)]


def reference_gpu_leg(args):
    """The reference's own GPU CP-ALS (cpals_blco_dev, src/cpd_gpu.cu:21-242,
    rebuilt unchanged for sm_100a into oracle/_ref/libblco_refgpu.so) on the
    full workload with the same initial factors as this engine's arm, -k 10,
    warm-up + timed iterations: median of its own per-iteration times (CUDA
    events around each iteration, src/cpd_gpu.cu:148-193) after the warm-up
    iterations.  The reference encodes on the host first (about a minute at
    200M nonzeros).  Then, outside that timing, this engine's plain FP64 form
    runs the same iterations from the same factors: the per-iteration fit
    difference is the full-size parity record."""
    import re
    import tempfile
    import torch
    import pyoracle as po
    if not po.refgpu_available():
        return {"unavailable": "oracle/_ref/libblco_refgpu.so not built"}
    if not torch.cuda.is_available():
        return {"unavailable": "no GPU"}
    from blco_b200 import synth
    dims, nnz, rk = WORKLOAD["dims"], args.nnz, WORKLOAD["rank"]
    X = synth.zipf_tensor_device(nnz, dims, WORKLOAD["zipf"], seed=args.seed)
    cidx = np.ascontiguousarray(np.stack([c.cpu().numpy().astype(np.uint64) for c in X["cidx"]]))
    vals = np.ascontiguousarray(X["vals"].cpu().numpy())
    del X
    g = torch.Generator(device="cuda").manual_seed(1234)
    fs = [np.ascontiguousarray(torch.rand(d, rk, dtype=torch.float64, device="cuda", generator=g).cpu().numpy())
          for d in dims]
    torch.cuda.empty_cache()
    iters = args.warmup + args.steps
    out = {}
    lam = np.ones(rk)
    f = [x.copy() for x in fs]
    with tempfile.NamedTemporaryFile("r", suffix=".log") as lf:
        t0 = time.perf_counter()
        fit = po.refgpu_cpals(dims, cidx, vals, f, lam, iters, -1.0, kernel=10, log_path=lf.name, timeout=2400)
        wall = time.perf_counter() - t0
        log = open(lf.name).read()
    its = [float(x) * 1e3 for x in re.findall(r"--> Iter +\d+: .*time = ([0-9.]+)", log)]
    timed = its[args.warmup:]
    ref_fits = _ref_fits(log)
    out["k10"] = dict(ms_per_step=statistics.median(timed) if timed else None, iterations=len(its),
                      fit_last=fit, wall_s_including_host_encode=wall)
    # parity at full size: this engine's plain FP64 form, same tensor, factors and iterations
    pkg = load_pkg()
    t = pkg.Tensor.encode(dims, cidx, vals)
    dfs = [torch.from_numpy(x.copy()).cuda() for x in fs]
    dl = torch.ones(rk, dtype=torch.float64, device="cuda")
    plan = pkg.CpalsPlan(t, dfs, dl, pkg.make_opts(precision=pkg.PRECISION_FP64))
    ours = plan.iterate(iters, tol=-1.0)
    plan.destroy()
    ours_f = [x.cpu().numpy() for x in dfs]
    t.free()
    n = min(len(ours), len(ref_fits))
    d = [abs(a - b) for a, b in zip(ours[:n], ref_fits[:n])]
    fac = max(float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(ours_f, f))
    out["parity_full_size"] = dict(
        iterations=n, fit_ref_last=ref_fits[n - 1] if n else None, fit_ours_last=ours[n - 1] if n else None,
        max_abs_fit_diff=max(d) if d else None,
        max_rel_fit_diff=max(x / abs(b) for x, b in zip(d, ref_fits[:n])) if d else None,
        factor_rel_diff_last=fac,
        note=("this engine's plain FP64 CP-ALS (kernel 10) against the reference's cpals_blco_dev (-k 10) on the "
              "full workload, same initial factors; fits of every iteration (the reference prints 6 decimals, "
              "so the fit difference is bounded by its print rounding), factors after the last"))
    if args.ref_gpu_wide:
        # the wide-key workload through the reference's 128-bit build (same tensor and factors as the wide leg)
        X = synth.wide_tensor_device(WIDE["nnz"], WIDE["dims"], WIDE["zipf"], seed=WIDE["seed"])
        wc = np.ascontiguousarray(np.stack([c.cpu().numpy().astype(np.uint64) for c in X["cidx"]]))
        wv = np.ascontiguousarray(X["vals"].cpu().numpy())
        del X
        g = torch.Generator(device="cuda").manual_seed(4321)
        wf = [np.ascontiguousarray(torch.rand(d, WIDE["rank"], dtype=torch.float64, device="cuda",
                                              generator=g).cpu().numpy()) for d in WIDE["dims"]]
        torch.cuda.empty_cache()
        lam = np.ones(WIDE["rank"])
        with tempfile.NamedTemporaryFile("r", suffix=".log") as lf:
            t0 = time.perf_counter()
            fit = po.refgpu_cpals(WIDE["dims"], wc, wv, wf, lam, iters, -1.0, kernel=10,
                                  log_path=lf.name, wide=True, timeout=2400)
            wall = time.perf_counter() - t0
            log = open(lf.name).read()
        its = [float(x) * 1e3 for x in re.findall(r"--> Iter +\d+: .*time = ([0-9.]+)", log)]
        timed = its[args.warmup:]
        out["wide_k10"] = dict(workload=WIDE["workload"], ms_per_step=statistics.median(timed) if timed else None,
                               iterations=len(its), fit_last=fit, wall_s_including_host_encode=wall)
    out["note"] = ("reference cpals_blco_dev (oracle/_ref/libblco_refgpu.so, unchanged source for sm_100a), FP64, "
                   "-k 10 (lvl1 for these mode lengths), one block, the full workload and this engine's initial "
                   f"factors; median of the reference's own per-iteration times after {args.warmup} warm-up "
                   "iterations")
    return out


C1 = dict(workload="cpals_uniform_1000x800x600_nnz100k_r16_20iters",
          desc=("1000 x 800 x 600, 100k distinct uniform coordinates, U(0,1) FP64 values, rank 16, 20 iterations "
                "with tolerance 0, factors from the reference's KruskalModelRandomInit (seed 1, one thread)"),
          dims=[1000, 800, 600], nnz=100_000, rank=16, iters=20)


def c1_inputs():
    import pyoracle as po
    from blco_b200 import synth
    X = synth.uniform_tensor_host(C1["nnz"], C1["dims"], seed=0)
    fs, lam = po.kruskal_random_init(C1["dims"], C1["rank"], 1, 1)
    return X, fs, lam


def reference_cpu_c1():
    """The reference's CPU CP-ALS (cpd_alto) on the CPU-runnable workload,
    measured whole (no sample): its own "Per iteration" time with all host
    threads and with one."""
    import pyoracle as po
    X, fs, lam = c1_inputs()
    out = dict(workload=C1["workload"], desc=C1["desc"])
    for nt in sorted({os.cpu_count() or 1, 1}, reverse=True):
        f = [x.copy() for x in fs]
        r = po.ref_cpd_alto(C1["dims"], X["cidx"], X["vals"], f, lam.copy(), C1["iters"], 0.0, nthreads=nt)
        out[f"threads_{nt}"] = r
    best = min((v for k, v in out.items() if k.startswith("threads_")), key=lambda r: r["ms_per_iter"])
    out.update(value=best["ms_per_iter"], unit="ms", cores=best["threads"], fit=best["fit"])
    return out


def run_reference(args, world, rank):
    """The reference's CPU CP-ALS (cpd_alto, include/cpd.hpp:44-187, built
    from the reference sources into oracle/_ref with scipy's OpenBLAS) on the
    workload (the whole tensor unless --ref-sample asks for fewer nonzeros,
    which are then scaled), all host threads, and on the CPU-runnable
    workload whole; then the reference's GPU code on the full workload."""
    if rank != 0:
        return
    import torch
    import pyoracle as po
    if po.ref_lib() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libblco_ref.so not built"}))
        return
    load_pkg()
    from blco_b200 import synth
    sample = min(args.ref_sample, WORKLOAD["nnz"])
    full = sample == WORKLOAD["nnz"]  # --ref-sample 200000000: the whole tensor, measured, not scaled
    dims, rk = WORKLOAD["dims"], WORKLOAD["rank"]
    if torch.cuda.is_available():
        X = synth.zipf_tensor_device(sample, dims, WORKLOAD["zipf"], seed=args.seed if full else 7)
        cidx = np.stack([c.cpu().numpy().astype(np.uint64) for c in X["cidx"]])
        vals = X["vals"].cpu().numpy()
        del X
    else:
        X = synth.uniform_tensor_host(sample, dims, seed=7)
        cidx, vals = X["cidx"], X["vals"]
    nthreads = os.cpu_count() or 1
    rng = np.random.default_rng(0)
    fs = [np.ascontiguousarray(rng.random((d, rk))) for d in dims]
    r = po.ref_cpd_alto(dims, cidx, vals, fs, np.ones(rk), args.warmup + args.steps, 0.0, nthreads=nthreads)
    scale = WORKLOAD["nnz"] / sample
    value = r["ms_per_iter"] + r["mttkrp_ms_per_iter"] * (scale - 1.0)
    if full:
        desc = (f"reference cpd_alto (oracle/_ref, scipy OpenBLAS) on the whole {sample}-nonzero tensor, "
                f"{nthreads} threads, {r['iters']} iterations, its own per-iteration times "
                f"({r['ms_per_iter']:.1f} ms, of which MTTKRP {r['mttkrp_ms_per_iter']:.1f} ms): measured")
    else:
        desc = (f"reference cpd_alto (oracle/_ref, scipy OpenBLAS) on {sample} nonzeros of the same distribution "
                f"with the full mode lengths, {nthreads} threads, {r['iters']} iterations, its own per-iteration "
                f"times ({r['ms_per_iter']:.1f} ms, of which MTTKRP {r['mttkrp_ms_per_iter']:.1f} ms); estimate "
                f"for {WORKLOAD['nnz']} nonzeros = iteration + MTTKRP x ({scale:.0f} - 1): the dense steps already "
                "run at full size, the MTTKRP is scaled by the nonzeros (--ref-sample 200000000 measures the "
                "whole tensor)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "ms", "higher_is_better": False,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": value,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(workload=WORKLOAD["workload"], parallelism="cpu", l2="inputs larger than L2"),
        "cpu_baseline": dict(value=value, unit="ms", cores=nthreads, kind="reference", sample=desc,
                             sample_ms_per_iter=r["ms_per_iter"], sample_mttkrp_ms_per_iter=r["mttkrp_ms_per_iter"],
                             sample_nnz=sample),
        "e2e": dict(value=value, unit="ms", h2d_bytes_per_step=0, d2h_bytes_per_step=0),
        "c1": reference_cpu_c1(),
        "reference_gpu": None if args.no_ref_gpu else reference_gpu_leg(args),
    }
    print(json.dumps(line))


def cpu_baseline_full(args, dims, rk, h_cidx, h_vals):
    """The reference's CPU CP-ALS (cpd_alto, oracle/_ref) on the whole
    benchmark tensor (its host copy), all host threads, 3 iterations: its own
    per-iteration time (rank 0, N=1 only)."""
    import pyoracle as po
    if po.ref_lib() is None:
        return None
    cidx = np.ascontiguousarray(np.stack([c.numpy().view(np.uint64) for c in h_cidx]))
    vals = np.ascontiguousarray(h_vals.numpy())
    nthreads = os.cpu_count() or 1
    rng = np.random.default_rng(0)
    fs = [np.ascontiguousarray(rng.random((d, rk))) for d in dims]
    r = po.ref_cpd_alto(dims, cidx, vals, fs, np.ones(rk), 3, 0.0, nthreads=nthreads)
    return dict(value=r["ms_per_iter"], unit="ms", cores=nthreads, kind="reference",
                mttkrp_ms_per_iter=r["mttkrp_ms_per_iter"],
                sample=(f"reference cpd_alto (oracle/_ref, scipy OpenBLAS) on the whole {cidx.shape[1]}-nonzero "
                        f"tensor, {nthreads} threads, {r['iters']} iterations, its own per-iteration time (MTTKRP "
                        f"{r['mttkrp_ms_per_iter']:.1f} ms of it): measured, not scaled"))


FORMS = {
    # name: (precision code attr, value bytes, factor bytes, output bytes, dtype label)
    "fp64": ("PRECISION_FP64", 8, 8, 8, "f64"),
    "mixed_f32": ("PRECISION_MIXED", 4, 4, 4, "f32 (fp64 solve/lambda/fit)"),
    "mixed_bf16": ("PRECISION_MIXED_BF16", 4, 2, 4, "f32 accumulate, bf16 gathers (fp64 solve/lambda/fit)"),
}


def time_form(pkg, torch, t, dims, rk, fs0, form, args, stream, dist, norm_sq=None):
    """Warm up, then time args.steps CP-ALS iterations of one numeric form.
    With norm_sq (a tensor sharded over the ranks), each mode's MTTKRP is
    summed over the ranks by an all-reduce on the plan's stream and the fit
    uses the whole tensor's norm.
    Returns dict(ms_per_step, mttkrp_ms (per mode), fits, launches, clocks)."""
    prec = getattr(pkg, FORMS[form][0])
    opts = pkg.make_opts(kernel=args.kernel, precision=prec, stream=stream.cuda_stream)
    fs = [f.clone() for f in fs0]
    lam = torch.ones(rk, dtype=torch.float64, device="cuda")
    plan = pkg.CpalsPlan(t, fs, lam, opts)
    if norm_sq is not None:
        plan.set_reduce(pkg.dist_reduce(dist))
        plan.set_norm_sq(norm_sq)
    fits = plan.iterate(args.warmup, tol=-1.0)
    ms0, calls0 = plan.mttkrp_ms()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    pkg.launch_count(reset=True)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    fits += plan.iterate(args.steps, tol=-1.0)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = pkg.launch_count(reset=True)
    ck = clocks.stop()
    elapsed = ev0.elapsed_time(ev1)
    ms1, calls1 = plan.mttkrp_ms()
    timed_end = len(fits)
    # untimed: the same run continued to args.fit_iters iterations, where the
    # forms' fits are compared (the decomposition's fit, near convergence)
    if args.fit_iters > len(fits):
        fits += plan.iterate(args.fit_iters - len(fits), tol=-1.0)
    plan.destroy()
    del fs, lam
    per_rank = all_ranks(elapsed / args.steps, dist)
    elapsed = max_over_ranks(elapsed, dist)
    return dict(ms_per_step=elapsed / args.steps, mttkrp_ms=list((ms1 - ms0) / max(1, calls1 - calls0)),
                fits=fits, timed_end=timed_end, launches=int(launches), clocks=ck, ms_per_step_per_rank=per_rank)


def c1_leg(pkg, torch, args):
    """This engine on the CPU-runnable workload (the reference's KruskalModel
    initial factors, 20 iterations, tolerance 0): device ms per iteration of
    the plain FP64 plan and the mixed plan, and blco_cpals end to end from
    host buffers (encode + 20 iterations)."""
    import pyoracle as po
    X, fs, lam = c1_inputs()
    out = dict(workload=C1["workload"], desc=C1["desc"])
    t = pkg.Tensor.encode(C1["dims"], X["cidx"], X["vals"])
    for name, prec in (("fp64", pkg.PRECISION_FP64), ("mixed_f32", pkg.PRECISION_MIXED)):
        dfs = [torch.from_numpy(x.copy()).cuda() for x in fs]
        dl = torch.from_numpy(lam.copy()).cuda()
        plan = pkg.CpalsPlan(t, dfs, dl, pkg.make_opts(kernel=args.kernel, precision=prec))
        plan.iterate(2, tol=-1.0)
        plan.destroy()
        dfs = [torch.from_numpy(x.copy()).cuda() for x in fs]
        dl = torch.from_numpy(lam.copy()).cuda()
        plan = pkg.CpalsPlan(t, dfs, dl, pkg.make_opts(kernel=args.kernel, precision=prec))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        fits = plan.iterate(C1["iters"], tol=-1.0)
        e1.record()
        torch.cuda.synchronize()
        plan.destroy()
        out[name] = dict(ms_per_iter=e0.elapsed_time(e1) / C1["iters"], fit=fits[-1])
    t.free()
    f = [x.copy() for x in fs]
    t0 = time.perf_counter()
    t2 = pkg.Tensor.encode(C1["dims"], X["cidx"], X["vals"])
    fit, _ = pkg.cpals(t2, f, lam.copy(), C1["iters"], -1.0, pkg.make_opts(kernel=args.kernel))
    out["e2e_fp64_ms_per_iter"] = (time.perf_counter() - t0) * 1e3 / C1["iters"]
    t2.free()
    out["fit_reference_oracle"] = float(po.cpals(C1["dims"], po.blco_encode(C1["dims"], X["cidx"], X["vals"]),
                                                 [x.copy() for x in fs], lam.copy(), C1["iters"], -1.0)[-1])
    out["note"] = ("device time (CUDA events) of plans whose factors start on the device; e2e: blco_encode from host "
                   "COO + blco_cpals with host factors, wall time / iterations; fit_reference_oracle: the CPU "
                   "restatement of the reference's GPU CP-ALS on the same inputs")
    return out


BATCH = dict(
    workload=("512 independent 3-mode tensors: nnz lognormal(median 2e5, sigma 1) clipped to [1e4, 2e6] and to half "
              "the cells, mode lengths U[100, 50000], uniform coordinates, FP32 U(0,1) values, rank in {8,16,32}"),
    count=512, seed=4)


def batched_leg(pkg, torch, args):
    """Batched CP-ALS of the many-small-tensors workload: device ms per
    sweep of the captured graph, next to per-tensor plans run one after
    another (timed on the first 32 tensors, scaled by nnz)."""
    from blco_b200 import synth
    Xs = synth.batch_tensors_device(args.batch_count, seed=BATCH["seed"])
    nnzs = [int(x["vals"].numel()) for x in Xs]
    ts = [pkg.Tensor.encode_device(x["dims"], x["cidx"], x["vals"]) for x in Xs]
    ranks = [x["rank"] for x in Xs]
    dims = [x["dims"] for x in Xs]
    del Xs
    torch.cuda.empty_cache()
    g = torch.Generator(device="cuda").manual_seed(99)
    fs = [[torch.rand(d, r, dtype=torch.float64, device="cuda", generator=g) for d in dd] for dd, r in zip(dims, ranks)]
    f0 = [[m.clone() for m in f] for f in fs]
    ls = [torch.ones(r, dtype=torch.float64, device="cuda") for r in ranks]
    b = pkg.Batch(ts, fs, ls, tol=0.0)
    b.iterate(args.warmup)
    pkg.launch_count(reset=True)
    b.iterate(args.steps)
    launches = pkg.launch_count(reset=True)
    ms = b.last_ms() / max(1, args.steps)
    mt_ms = min(b.mttkrp_ms() for _ in range(3))
    b.destroy()
    # algorithmic bytes of one sweep's MTTKRPs (FP64): per tensor and mode,
    # the index and value stream once, every other factor once, the output once
    alg = 0
    for dd, r, nz in zip(dims, ranks, nnzs):
        for m in range(len(dd)):
            alg += nz * (8 + 8) + sum(d for i, d in enumerate(dd) if i != m) * r * 8 + dd[m] * r * 8
    peak = peaks()[0]
    # per-tensor plans, one after another, on a prefix of the batch
    k = min(32, len(ts))
    seq = 0.0
    for i in range(k):
        lam = torch.ones(ranks[i], dtype=torch.float64, device="cuda")
        p = pkg.CpalsPlan(ts[i], f0[i], lam)
        p.iterate(2, tol=-1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        p.iterate(3, tol=-1.0)
        torch.cuda.synchronize()
        seq += (time.perf_counter() - t0) / 3
        p.destroy()
    seq_est = seq * 1e3 * sum(nnzs) / sum(nnzs[:k])
    for t in ts:
        t.free()
    return dict(workload=BATCH["workload"], tensors=len(ts), nnz=sum(nnzs), ms_per_sweep=ms, sweeps=args.steps,
                gpu_launches=int(launches), dtype="f64", graph="one CUDA graph per sweep",
                mttkrp_ms_per_sweep=mt_ms,
                roofline=dict(bound="hbm", achieved=alg / (mt_ms * 1e-3) / 1e9, peak=peak, unit="GB/s",
                              frac=alg / (mt_ms * 1e-3) / 1e9 / peak, traffic=None, alg_bytes_per_sweep=int(alg),
                              kernel="k_b_mttkrp, every mode slot of one sweep (CUDA events, outside the graph, "
                                     "best of 3); algorithmic bytes: per tensor and mode the BLCO coordinate "
                                     "(8 B) and value (8 B) of each nonzero, every other factor and the output "
                                     "once"),
                sequential_plans_ms_per_iter_est=seq_est, speedup_vs_sequential=seq_est / ms,
                note="device time (CUDA events on the batch stream); sequential estimate from the first "
                     f"{k} tensors' plans (wall time), scaled by nnz")


WIDE = dict(workload="mttkrp_wide_zipf1.1_2^20x2^20x2^20x4096_nnz100M_r32",
            desc=("keys of 72 bits (the reference's 128-bit build): Zipf(1.1) coordinates over 2^20 x 2^20 x 2^20 "
                  "x 4096, 100M distinct nonzeros, lognormal FP32 values, rank 32, FP64 CP-ALS"),
            dims=[1 << 20, 1 << 20, 1 << 20, 1 << 12], nnz=100_000_000, zipf=1.1, rank=32, seed=7)


def wide_cpu_baseline(args, X, dims, rk):
    """The reference's 128-bit CPU ALTO MTTKRP (oracle/_ref) on a bounded
    sample of the wide workload, all modes, scaled to its nonzeros."""
    import ctypes
    import pyoracle as po
    R = po.ref_lib()
    if R is None:
        return None
    total = int(X["vals"].numel())
    sample = min(args.ref_sample, total)
    cidx = np.ascontiguousarray(np.stack([c[:sample].cpu().numpy().astype(np.uint64) for c in X["cidx"]]))
    vals = np.ascontiguousarray(X["vals"][:sample].cpu().numpy())
    nthreads = os.cpu_count() or 1
    d64 = np.ascontiguousarray(dims, dtype=np.uint64)
    u64p = ctypes.POINTER(ctypes.c_uint64)
    f64p = ctypes.POINTER(ctypes.c_double)
    h = R.ref_alto_create128(len(dims), d64.ctypes.data_as(u64p), sample, cidx.ctypes.data_as(u64p),
                             vals.ctypes.data_as(f64p), nthreads)
    rng = np.random.default_rng(0)
    fs = [rng.random((d, rk)) for d in dims]
    ptrs = (ctypes.c_void_p * len(dims))(*[f.ctypes.data for f in fs])
    for m in range(len(dims)):
        R.ref_alto_mttkrp128(h, m, rk, ptrs)
    t0 = time.perf_counter()
    for m in range(len(dims)):
        R.ref_alto_mttkrp128(h, m, rk, ptrs)
    dt = (time.perf_counter() - t0) * 1e3
    R.ref_alto_destroy128(h, rk)
    how = ("the whole tensor, measured" if sample == total else
           f"the first {sample} nonzeros, scaled linearly to {total} nonzeros")
    return dict(value=dt / sample * total, unit="ms", cores=nthreads, kind="reference",
                sample=(f"reference mttkrp_alto_par on AltoTensor<unsigned __int128> (oracle/_ref), all "
                        f"{len(dims)} modes on {how}, {nthreads} threads; MTTKRP part of the iteration only"))


def wide_leg(pkg, torch, args, peak, with_cpu):
    """FP64 CP-ALS of the wide-key workload: encode, device ms per
    iteration, per-mode MTTKRP time and its roofline, the reference's CPU
    MTTKRP on a sample."""
    from blco_b200 import synth
    dims, nnz, rk = WIDE["dims"], args.wide_nnz, WIDE["rank"]
    X = synth.wide_tensor_device(nnz, dims, WIDE["zipf"], seed=WIDE["seed"])
    torch.cuda.synchronize()
    e0 = time.perf_counter()
    t = pkg.Tensor.encode_device(dims, X["cidx"], X["vals"])
    torch.cuda.synchronize()
    encode_ms = (time.perf_counter() - e0) * 1e3
    cpu = wide_cpu_baseline(args, X, dims, rk) if with_cpu else None
    del X
    torch.cuda.empty_cache()
    inf = t.info()
    g = torch.Generator(device="cuda").manual_seed(4321)
    fs = [torch.rand(d, rk, dtype=torch.float64, device="cuda", generator=g) for d in dims]
    lam = torch.ones(rk, dtype=torch.float64, device="cuda")
    plan = pkg.CpalsPlan(t, fs, lam, pkg.make_opts(kernel=pkg.KERNEL_AUTO))
    plan.iterate(args.warmup, tol=-1.0)
    ms0, c0 = plan.mttkrp_ms()
    pkg.launch_count(reset=True)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record()
    fits = plan.iterate(args.steps, tol=-1.0)
    ev1.record()
    torch.cuda.synchronize()
    launches = pkg.launch_count(reset=True)
    ms1, c1 = plan.mttkrp_ms()
    per_mode = list((ms1 - ms0) / max(1, c1 - c0))
    plan.destroy()
    t.free()
    del fs
    torch.cuda.empty_cache()
    alg = [mttkrp_alg_bytes(dims, nnz, rk, m) for m in range(len(dims))]
    achieved = sum(alg) / (sum(per_mode) * 1e-3) / 1e9
    return dict(workload=WIDE["workload"] if nnz == WIDE["nnz"] else WIDE["workload"] + f"_at_{nnz}_nnz",
                desc=WIDE["desc"], nnz=nnz, key_bits=inf["alto_bits"],
                blocks=inf["block_count"], encode_ms=encode_ms,
                ms_per_step=ev0.elapsed_time(ev1) / args.steps, steps=args.steps, fit_last=fits[-1],
                mttkrp_ms_per_mode=[round(x, 4) for x in per_mode], gpu_launches=int(launches), dtype="f64",
                roofline=dict(bound="hbm", achieved=achieved, peak=peak, unit="GB/s", frac=achieved / peak,
                              traffic=traffic_from_profiles("fp64", nnz, "mttkrp_wide_zipf_2p20x3x4096_r32.md",
                                                            WIDE["nnz"]),
                              kernel="k_mttkrp_wide (one launch per mode), mean over the 4 modes",
                              alg_bytes_per_launch=[int(x) for x in alg]),
                cpu_baseline=cpu)


STREAMED = dict(workload="cpals_streamed_zipf0.9_500kx200kx50kx1k_r64", dims=[500_000, 200_000, 50_000, 1_000],
                zipf=0.9, rank=64, full_nnz=2_000_000_000, residency=8_000_000_000, block=64 << 20,
                values="uniform(0,1) fp32 as fp64, repeated coordinates kept as separate nonzeros")


def pinned_h2d_peak(torch, gib=2, reps=3):
    """Host-to-device GB/s of one pinned copy of `gib` GiB, best of `reps`."""
    hb = torch.empty(gib << 27, dtype=torch.float64).pin_memory()
    db = torch.empty(gib << 27, dtype=torch.float64, device="cuda")
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    best = 0.0
    for _ in range(reps):
        e0.record()
        db.copy_(hb, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, hb.numel() * 8 / (e0.elapsed_time(e1) * 1e-3) / 1e9)
    del hb, db
    return best


def streamed_leg(pkg, torch, args):
    """The out-of-memory streamed CP-ALS: the 4-mode Zipf(0.9) 500k x 200k x
    50k x 1k tensor at rank 64, blocks of 64M nonzeros kept in pinned host
    memory and copied through a ring of device buffers, with the whole
    plan's device memory (factors, workspace, ring) capped at 8e9 bytes.
    Each iteration copies every block once per mode, so the bound is the
    host link: H2D bytes per iteration over the time, against a pinned copy
    measured in the same process.  FP64 and the mixed FP32 form (4-byte
    values streamed from a pinned FP32 copy)."""
    from blco_b200 import synth
    W = STREAMED
    dims, rk, nnz = W["dims"], W["rank"], args.streamed_nnz
    peak = pinned_h2d_peak(torch)
    X = synth.zipf_coo_device(nnz, dims, W["zipf"], seed=args.seed)
    torch.cuda.synchronize()
    o = pkg.make_opts(kernel=10, stream_data=True, residency_bytes=W["residency"])
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    t = pkg.Tensor.encode_device(dims, X["cidx"], X["vals"], W["block"], o)
    torch.cuda.synchronize()
    encode_s = time.perf_counter() - t0
    del X
    torch.cuda.empty_cache()
    info = t.info()
    g = torch.Generator(device="cuda").manual_seed(1234)
    fs0 = [torch.rand(d, rk, dtype=torch.float64, device="cuda", generator=g) for d in dims]
    forms = {}
    for name, prec, bpn in (("fp64", pkg.PRECISION_FP64, 16), ("mixed_f32", pkg.PRECISION_MIXED, 12)):
        fs = [f.clone() for f in fs0]
        lam = torch.ones(rk, dtype=torch.float64, device="cuda")
        plan = pkg.CpalsPlan(t, fs, lam, pkg.make_opts(kernel=10, stream_data=True, residency_bytes=W["residency"],
                                                       precision=prec))
        plan.iterate(1, tol=-1.0)
        torch.cuda.synchronize()
        free_b, total_b = torch.cuda.mem_get_info()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fits = plan.iterate(args.streamed_iters, tol=-1.0)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.streamed_iters
        _, promoted = plan.condition()
        h2d = len(dims) * nnz * bpn
        forms[name] = dict(ms_per_iter=ms, h2d_bytes_per_iter=h2d, h2d_gbs=h2d / (ms * 1e-3) / 1e9,
                           h2d_frac=h2d / (ms * 1e-3) / 1e9 / peak, fit_last=fits[-1],
                           device_bytes_plan=int(plan.device_bytes()),
                           device_bytes_in_use=int(total_b - free_b), promoted_to_fp64=bool(promoted))
        if promoted:  # the guard moved the mixed plan to FP64: FP64 values crossed the link
            forms[name]["h2d_bytes_per_iter"] = h2d = len(dims) * nnz * 16
            forms[name].update(h2d_gbs=h2d / (ms * 1e-3) / 1e9, h2d_frac=h2d / (ms * 1e-3) / 1e9 / peak)
        plan.destroy()
        del fs, lam
    forms["mixed_f32"]["fit_delta_vs_fp64"] = abs(forms["mixed_f32"]["fit_last"] - forms["fp64"]["fit_last"])
    t.free()
    del fs0
    torch.cuda.empty_cache()
    return dict(workload=W["workload"] + (f"_nnz{nnz // 1_000_000}M" if nnz != W["full_nnz"] else "_nnz2B"),
                dims=dims, nnz=nnz, full_nnz=W["full_nnz"], rank=rk, zipf=W["zipf"], values=W["values"],
                residency_bytes=W["residency"], block_nnz=W["block"], blocks=info["block_count"],
                iters_timed=args.streamed_iters, encode_s=encode_s, pinned_h2d_peak_gbs=peak, forms=forms,
                roofline=dict(bound="host link (H2D)", achieved=forms["mixed_f32"]["h2d_gbs"], peak=peak,
                              unit="GB/s", frac=forms["mixed_f32"]["h2d_frac"],
                              peak_kind="pinned 2 GiB host-to-device copy, best of 3, this process"),
                note=("nnz below the configuration's 2B keeps the leg inside the benchmark's time budget "
                      "(--streamed-nnz 2000000000 runs the full size); every block crosses the host link once "
                      "per mode per iteration: 16 B per nonzero (FP64 values) or 12 B (mixed, FP32 values); "
                      "device_bytes_plan is the plan's own count (caller's factors, workspace, ring)"))


def shard_slice(X, world, rank):
    """This rank's share of a tensor whose nonzeros are split over `world`
    ranks: a contiguous range of the nonzero list (every rank draws the
    same tensor), and ||X||^2 of the whole tensor for the fit."""
    n = X["vals"].numel()
    lo, hi = n * rank // world, n * (rank + 1) // world
    norm_sq = float((X["vals"].double() ** 2).sum().item())
    return dict(dims=X["dims"], cidx=[c[lo:hi] for c in X["cidx"]], vals=X["vals"][lo:hi], lo=lo, hi=hi,
                norm_sq=norm_sq)


def run_ours(args, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    pkg = load_pkg()
    from blco_b200 import synth
    selector = pkg.default_selector(margin=0.1) if args.kernel == pkg.KERNEL_LEARNED else None
    dims, nnz, rk = WORKLOAD["dims"], args.nnz, WORKLOAD["rank"]
    # every rank draws the same tensor; with N ranks each encodes and owns a
    # contiguous 1/N of its nonzeros, and each mode's MTTKRP is summed over
    # the ranks (strong scaling: the job is the one tensor)
    X = synth.zipf_tensor_device(nnz, dims, WORKLOAD["zipf"], seed=args.seed)
    norm_sq = None
    Xs = X
    if world > 1:
        Xs = shard_slice(X, world, rank)
        norm_sq = Xs["norm_sq"]
    nnz_local = int(Xs["vals"].numel())
    stream = torch.cuda.current_stream()
    opts = pkg.make_opts(kernel=args.kernel, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    e0 = time.perf_counter()
    t = pkg.Tensor.encode_device(dims, Xs["cidx"], Xs["vals"], 0, opts)
    torch.cuda.synchronize()
    encode_ms = (time.perf_counter() - e0) * 1e3
    del Xs
    # host copies for the end-to-end leg (pinned)
    h_cidx = [c.to(torch.int64).cpu().pin_memory() for c in X["cidx"]]
    h_vals = X["vals"].cpu().pin_memory()
    del X
    torch.cuda.empty_cache()
    g = torch.Generator(device="cuda").manual_seed(1234 + rank)
    fs0 = [torch.rand(d, rk, dtype=torch.float64, device="cuda", generator=g) for d in dims]

    forms = [f.strip() for f in args.forms.split(",") if f.strip()]
    res = {f: time_form(pkg, torch, t, dims, rk, fs0, f, args, stream, dist, norm_sq) for f in forms}
    plain = res.get("fp64")
    chosen = "fp64"
    best = plain["ms_per_step"] if plain else float("inf")
    for f in forms:
        if f == "fp64":
            continue
        dfit = abs(res[f]["fits"][-1] - plain["fits"][-1]) if plain else 0.0
        res[f]["fit_delta_vs_fp64"] = dfit
        if plain:
            n = min(len(res[f]["fits"]), len(plain["fits"]))
            d = np.abs(np.array(res[f]["fits"][:n]) - np.array(plain["fits"][:n]))
            res[f]["fit_delta_max_over_run"] = float(d.max())
            res[f]["fit_delta_at_timed_end"] = float(d[res[f]["timed_end"] - 1])
        if dfit <= 1e-5 and res[f]["ms_per_step"] < best:
            best, chosen = res[f]["ms_per_step"], f
    C = res[chosen]
    _, sv, sf, so, dtype = FORMS[chosen]

    # end-to-end: the public C ABI from host buffers (COO in, factors out), chosen form
    # host factors in pinned memory, as a caller streaming from the host would keep them
    h_fs = []
    for f in fs0:
        hp = torch.empty(f.shape, dtype=torch.float64, pin_memory=True)
        hp.copy_(f)
        h_fs.append(hp.numpy())
    e_iters = args.steps
    h2d = sum(c.numel() * 8 for c in h_cidx) + h_vals.numel() * 8 + sum(f.nbytes for f in h_fs) + rk * 8
    d2h = sum(f.nbytes for f in h_fs) + rk * 8 + e_iters * 8
    cidx_np = [c.numpy().view(np.uint64) for c in h_cidx]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    import ctypes
    L = pkg.lib()
    t0 = time.perf_counter()
    ptrs = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in cidx_np])
    h = ctypes.c_void_p()
    o2 = pkg.make_opts(kernel=args.kernel, precision=getattr(pkg, FORMS[chosen][0]), stream=0)
    d64 = np.ascontiguousarray(dims, dtype=np.uint64)
    st = L.blco_encode(3, d64.ctypes.data, nnz, ptrs, h_vals.numpy().ctypes.data, 0, ctypes.byref(o2),
                       ctypes.byref(h))
    if st != 0:
        raise RuntimeError(L.blco_last_error().decode())
    t2 = pkg.Tensor(h.value)
    t1 = time.perf_counter()
    lam_h = np.ones(rk)
    pkg.cpals(t2, h_fs, lam_h, e_iters, -1.0, o2)
    t3 = time.perf_counter()
    e2e_ms = (t3 - t0) * 1e3 / e_iters
    e2e_split = dict(encode_ms=(t1 - t0) * 1e3, cpals_ms=(t3 - t1) * 1e3)
    t2.free()
    e2e_ms = max_over_ranks(e2e_ms, dist)

    peak, peak_kind = peaks()
    alg = [mttkrp_alg_bytes(dims, nnz, rk, m, 8, sv, sf, so) for m in range(3)]
    achieved = sum(alg) / (sum(C["mttkrp_ms"]) * 1e-3) / 1e9  # GB/s over the three launches
    traffic = traffic_from_profiles(chosen, nnz)
    # the schedule kernel id 21 takes for each mode of the chosen form
    schedules = None
    if selector is not None:
        space = pkg.tune_space()
        dt = {"fp64": pkg.DTYPE_F64, "mixed_f32": pkg.DTYPE_F32, "mixed_bf16": pkg.DTYPE_BF16}[chosen]
        schedules = []
        for m in range(3):
            k, swept = pkg.select(t, m, rk, dt, selector, 0.1)
            schedules.append(dict(mode=m, schedule=k, **space[k], decided_by="sweep" if swept else "network"))
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_full(args, dims, rk, h_cidx, h_vals)
    # rows each mode's MTTKRP gathers with the compressed-fibre kernel, and the rate
    gather = None
    used = [sc["kernel"] for sc in schedules] if schedules else None
    if rank == 0 and (used is None or 4 in used):
        try:
            st = [t.fibre_stats(m) for m in range(3)]
            rows = [x["rows_gathered"] for x in st]
            rates = [r / (ms * 1e-3) / 1e9 for r, ms in zip(rows, C["mttkrp_ms"])]
            nnz_g = nnz_local
            ceil = None if args.no_gather_ceiling else gather_ceiling()
            top = ceil["grows_per_s_zipf"] if ceil else None
            gather = dict(rows_per_mode=rows, fibre_modes=[x["fibre_mode"] for x in st],
                          fibred_share=[x["fibred_nnz"] / nnz_g for x in st], rows_per_nnz=[r / nnz_g for r in rows],
                          grows_per_s=rates, ceiling=ceil,
                          frac_of_ceiling=[r / top for r in rates] if top else None,
                          note=("rows gathered by kernel 4 per mode (the inner modes' rows of every fibred "
                                "nonzero, one fibre-mode row per fibre, every other mode's row of a single-nonzero "
                                "fibre) over the mode's MTTKRP time, against the load-path ceiling measured by "
                                "bin/gather_ceiling in this run; rows of rank x element bytes (128 B for the FP32 "
                                "form at rank 32)"))
        except Exception as e:  # modes the fibre kernel does not serve
            gather = dict(unavailable=str(e))
    c1 = c1_leg(pkg, torch, args) if rank == 0 and not args.no_c1 else None
    t.free()
    del fs0
    torch.cuda.empty_cache()
    batched = None
    if not args.no_batched:
        batched = batched_leg(pkg, torch, args)
    wide = None
    if not args.no_wide:
        wide = wide_leg(pkg, torch, args, peaks()[0], rank == 0 and world == 1 and not args.no_cpu_baseline)
    streamed = None
    if not args.no_streamed and rank == 0 and world == 1:
        streamed = streamed_leg(pkg, torch, args)
    if rank == 0:
        forms_out = {}
        for f, r in res.items():
            a_f = [mttkrp_alg_bytes(dims, nnz, rk, m, 8, FORMS[f][1], FORMS[f][2], FORMS[f][3]) for m in range(3)]
            forms_out[f] = dict(ms_per_step=r["ms_per_step"], mttkrp_ms_per_mode=[round(x, 4) for x in r["mttkrp_ms"]],
                                mttkrp_gbs=sum(a_f) / (sum(r["mttkrp_ms"]) * 1e-3) / 1e9, fit_last=r["fits"][-1],
                                fit_delta_vs_fp64=r.get("fit_delta_vs_fp64", 0.0),
                                fit_delta_at_timed_end=r.get("fit_delta_at_timed_end", 0.0),
                                fit_delta_max_over_run=r.get("fit_delta_max_over_run", 0.0), fit_iters=len(r["fits"]))
        line = {
            "metric": METRIC, "value": C["ms_per_step"], "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": C["ms_per_step"], "higher_is_better": False, "scaling": "strong",
            "vs_baseline": None, "dtype": dtype, "data": "synthetic",
            "config": dict(workload=WORKLOAD["workload"], dims=dims, nnz=nnz, rank=rk, zipf=WORKLOAD["zipf"],
                           values=WORKLOAD["values"], form=chosen, kernel=args.kernel, schedules=schedules,
                           parallelism=(f"nnz-sharded x{world}: each rank owns a contiguous 1/{world} of the "
                                        "nonzeros; each mode's MTTKRP all-reduced over NCCL on the plan's stream"
                                        if world > 1 else "single"),
                           l2="inputs larger than L2 (3.2 GB stream, >= 0.5 GB factors)"),
            "forms": forms_out,
            "plain_fp64_ms_per_step": plain["ms_per_step"] if plain else None,
            "speedup_vs_plain": (plain["ms_per_step"] / C["ms_per_step"]) if plain else None,
            "encode_ms": encode_ms,
            "roofline": dict(bound="hbm", achieved=achieved, peak=peak, unit="GB/s", frac=achieved / peak,
                             traffic=traffic, peak_kind=peak_kind + " (hbm_gbs burst copy)",
                             kernel=(f"MTTKRP of one mode, {chosen}, the schedule of each mode in "
                                     "config.schedules (kernel 4: k_mttkrp_fib); mean over the 3 modes; traffic = "
                                     "DRAM read + write per mode (ncu, profiles/)"),
                             alg_bytes_per_launch=[int(x) for x in alg], gather=gather),
            "cpu_baseline": cpu,
            "e2e": dict(value=e2e_ms, unit="ms", h2d_bytes_per_step=int(h2d / e_iters),
                        d2h_bytes_per_step=int(d2h / e_iters),
                        note=(f"blco_encode from pinned host COO + blco_cpals({e_iters} iters, {chosen}) with pinned "
                              "host factors; job time / iterations; bytes are per iteration"
                              + ("; with N ranks every rank runs the whole tensor this way (the host entry point "
                                 "takes no exchange hook), max over ranks" if world > 1 else "")), **e2e_split),
            "ms_per_step_per_rank": C["ms_per_step_per_rank"],
            "allreduce": (dict(bytes_per_mode=[int(d * rk * 8) for d in dims], bytes_per_iter=int(sum(dims) * rk * 8),
                               note="each mode's I_m x R MTTKRP result summed over the ranks (FP64: the plain "
                                    "form, and the mixed form's fibre schedule, which sums rows in FP64; 4-byte "
                                    "sums where a mixed mode runs a tile schedule)")
                          if world > 1 else None),
            "gpu_launches": C["launches"],
            "clocks": C["clocks"],
            "batched": batched,
            "wide": wide,
            "c1": c1,
            "streamed": streamed,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def mttkrp_leg(pkg, torch, args):
    """One MTTKRP per mode of the benchmark tensor (args.nnz nonzeros) with
    factors of --mttkrp-dtype, each mode's schedule from --kernel, timed with
    CUDA events: the kernels the ncu summaries capture."""
    from blco_b200 import synth
    dims, rk = WORKLOAD["dims"], WORKLOAD["rank"]
    X = synth.zipf_tensor_device(args.nnz, dims, WORKLOAD["zipf"], seed=args.seed)
    t = pkg.Tensor.encode_device(dims, X["cidx"], X["vals"])
    del X
    torch.cuda.empty_cache()
    g = torch.Generator(device="cuda").manual_seed(1)
    fs = [torch.rand(d, rk, dtype=torch.float64, device="cuda", generator=g) for d in dims]
    dt = args.mttkrp_dtype
    if dt != "f64":
        fs = [f.to(torch.float32 if dt == "f32" else torch.bfloat16) for f in fs]
    code = {"f64": pkg.DTYPE_F64, "f32": pkg.DTYPE_F32, "bf16": pkg.DTYPE_BF16}[dt]
    o = pkg.make_opts(kernel=args.kernel)
    sv, sf, so = {"f64": (8, 8, 8), "f32": (4, 4, 4), "bf16": (4, 2, 4)}[dt]
    modes = []
    for m in range(3):
        out = torch.zeros(dims[m], rk, dtype=torch.float64 if dt == "f64" else torch.float32, device="cuda")
        ts = []
        for _ in range(args.mttkrp_reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            pkg.mttkrp_ex(t, m, fs, out, code, o)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        alg = mttkrp_alg_bytes(dims, args.nnz, rk, m, 8, sv, sf, so)
        modes.append(dict(mode=m, ms=ts, alg_bytes=int(alg), gbs=alg / (min(ts) * 1e-3) / 1e9))
    t.free()
    return dict(nnz=args.nnz, dtype=dt, kernel=args.kernel, modes=modes)


def gram_leg(pkg, torch, args):
    """The mixed form's Gram of a 2M x 32 FP32 factor, tensor-core and
    CUDA-core engines (twice each: a warm-up, then the captured launch)."""
    U = torch.rand(2_000_000, 32, dtype=torch.float32, device="cuda") - 0.3
    ref = U.double().T @ U.double()
    out = {}
    for tc in (True, False):
        for _ in range(2):
            G = pkg.gram_f32(U, tensor_cores=tc)
        out["tensor_cores" if tc else "cuda_cores"] = (torch.linalg.norm(G - ref) / torch.linalg.norm(ref)).item()
    return dict(rows=2_000_000, rank=32, rel_err=out)


def run_only(args, local):
    """One leg alone on one GPU (the commands of the ncu summaries)."""
    import torch
    torch.cuda.set_device(local)
    pkg = load_pkg()
    if args.only == "mttkrp":
        out = mttkrp_leg(pkg, torch, args)
    elif args.only == "gram":
        out = gram_leg(pkg, torch, args)
    elif args.only == "streamed":
        out = streamed_leg(pkg, torch, args)
    elif args.only == "batched":
        out = batched_leg(pkg, torch, args)
    elif args.only == "wide":
        out = wide_leg(pkg, torch, args, peaks()[0], not args.no_cpu_baseline)
    else:
        out = c1_leg(pkg, torch, args)
    print(json.dumps({args.only: out}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nnz", type=int, default=WORKLOAD["nnz"])
    ap.add_argument("--kernel", type=int, default=21,
                    help="MTTKRP kernel id; 21 (default) = the committed learned schedule selector")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--ref-sample", type=int, default=WORKLOAD["nnz"],
                    help="--impl reference: nonzeros of the CPU CP-ALS run (the whole tensor by default; fewer are "
                         "scaled to it)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched many-small-tensors leg")
    ap.add_argument("--no-wide", action="store_true", help="skip the wide-key (128-bit BLCO) leg")
    ap.add_argument("--no-c1", action="store_true", help="skip the CPU-runnable workload leg")
    ap.add_argument("--no-gather-ceiling", action="store_true", help="skip the live gather-ceiling probe")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="--impl reference: skip the reference's own GPU CP-ALS on the full workload")
    ap.add_argument("--ref-gpu-wide", action="store_true",
                    help="--impl reference: also time the reference's GPU CP-ALS on the wide-key workload")
    ap.add_argument("--no-streamed", action="store_true", help="skip the streamed (out-of-memory) leg")
    ap.add_argument("--streamed-nnz", type=int, default=500_000_000,
                    help="nonzeros of the streamed leg (the configuration's full size is 2000000000)")
    ap.add_argument("--streamed-iters", type=int, default=2)
    ap.add_argument("--only", choices=["mttkrp", "gram", "streamed", "batched", "wide", "c1"],
                    help="run one leg alone and print its JSON object")
    ap.add_argument("--wide-nnz", type=int, default=WIDE["nnz"], help="nonzeros of the wide-key leg")
    ap.add_argument("--batch-count", type=int, default=BATCH["count"], help="tensors of the batched leg")
    ap.add_argument("--mttkrp-dtype", default="f32", choices=["f64", "f32", "bf16"])
    ap.add_argument("--mttkrp-reps", type=int, default=1)
    ap.add_argument("--fit-iters", type=int, default=40,
                    help="iterations after which the forms' fits are compared (the timed steps, then untimed)")
    ap.add_argument("--forms", default="fp64,mixed_f32,mixed_bf16")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.only:
        run_only(args, local)
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
