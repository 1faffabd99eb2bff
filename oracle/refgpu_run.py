"""Child-process runner for the reference's GPU code (test infrastructure).

The reference exits the process on any CUDA error (src/utils.cu:131-137), so
every call to oracle/_ref/libblco_refgpu.so runs in a fresh interpreter:

    python oracle/refgpu_run.py request.npz result.npz

request.npz holds op ("cpals" | "mttkrp"), dims, cidx, vals, factors f0..fN,
lam, rank, the reference flags, optionally wide (1: the 128-bit build's
encoding) and iters (MTTKRP repetitions); result.npz receives the outputs.  The
reference's own printout goes to this process's stdout/stderr.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(req_path, res_path):
    r = dict(np.load(req_path))
    G = ctypes.CDLL(os.path.join(HERE, "_ref", "libblco_refgpu.so"))
    u64p = ctypes.POINTER(ctypes.c_uint64)
    f64p = ctypes.POINTER(ctypes.c_double)
    dims = np.ascontiguousarray(r["dims"], dtype=np.uint64)
    cidx = np.ascontiguousarray(r["cidx"], dtype=np.uint64)
    vals = np.ascontiguousarray(r["vals"], dtype=np.float64)
    n = len(dims)
    fs = [np.ascontiguousarray(r[f"f{m}"], dtype=np.float64).copy() for m in range(n)]
    ptrs = (ctypes.c_void_p * n)(*[f.ctypes.data for f in fs])
    rank = int(r["rank"])
    wide = int(r["wide"]) if "wide" in r else 0
    cpals_fn = G.refgpu_cpals128 if wide else G.refgpu_cpals
    mttkrp_fn = G.refgpu_mttkrp128 if wide else G.refgpu_mttkrp
    iters = int(r["iters"]) if "iters" in r else 1
    out = {}
    if str(r["op"]) == "cpals":
        lam = np.ascontiguousarray(r["lam"], dtype=np.float64).copy()
        cpals_fn.restype = ctypes.c_double
        fit = cpals_fn(ctypes.c_int(n), dims.ctypes.data_as(u64p), ctypes.c_uint64(cidx.shape[1]),
                             cidx.ctypes.data_as(u64p), vals.ctypes.data_as(f64p), ctypes.c_int(rank), ptrs,
                             lam.ctypes.data_as(f64p), ctypes.c_int(int(r["maxiter"])),
                             ctypes.c_double(float(r["tol"])), ctypes.c_int(int(r["kernel"])),
                             ctypes.c_int(int(r["nprtn"])), ctypes.c_int(int(r["thread_cf"])))
        out["fit"] = np.float64(fit)
        out["lam"] = lam
    else:
        mttkrp_fn(ctypes.c_int(n), dims.ctypes.data_as(u64p), ctypes.c_uint64(cidx.shape[1]),
                  cidx.ctypes.data_as(u64p), vals.ctypes.data_as(f64p), ctypes.c_int(rank), ptrs,
                  ctypes.c_int(int(r["mode"])), ctypes.c_int(int(r["kernel"])), ctypes.c_int(iters),
                  ctypes.c_int(int(r["nprtn"])), ctypes.c_int(int(r["thread_cf"])))
    for m in range(n):
        out[f"f{m}"] = fs[m]
    sys.stdout.flush()
    np.savez(res_path, **out)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
