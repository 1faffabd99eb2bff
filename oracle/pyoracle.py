"""ctypes bindings for the CPU oracle (test infrastructure only).

Loads oracle/liboracle.so (the C restatement in blco_oracle.c) and, when it
was built, oracle/_ref/libblco_ref.so (the reference's own CPU code compiled
from its sources by `make -C oracle ref`).  Only tests/, the smoke check in
__graft_entry__.py and bench.py's CPU-baseline leg use this module; the
product path never does.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_u64p = ctypes.POINTER(ctypes.c_uint64)
_f64p = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int)


def _p(a, t):
    return a.ctypes.data_as(t)


def _ptr_array(arrs):
    return (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (run make -C oracle)")
        L = ctypes.CDLL(path)
        L.orc_pdep.restype = ctypes.c_uint64
        L.orc_pdep.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.orc_pext.restype = ctypes.c_uint64
        L.orc_pext.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.orc_alto_masks.restype = ctypes.c_int
        L.orc_blco_encode.restype = ctypes.c_int
        L.orc_blco_encode128.restype = ctypes.c_int
        L.orc_pinv_sym.restype = ctypes.c_int
        L.orc_cpals.restype = ctypes.c_int
        L.orc_cpals_coo.restype = ctypes.c_int
        _lib = L
    return _lib


def ref_lib():
    """The reference's own CPU code, or None when oracle/_ref was not built."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libblco_ref.so")
        if not os.path.exists(path):
            return None
        R = ctypes.CDLL(path)
        R.ref_blco_encode.restype = ctypes.c_int
        R.ref_blco_encode128.restype = ctypes.c_int
        R.ref_alto_create.restype = ctypes.c_void_p
        R.ref_alto_create.argtypes = [ctypes.c_int, _u64p, ctypes.c_uint64, _u64p, _f64p, ctypes.c_int]
        R.ref_alto_mttkrp.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        R.ref_alto_destroy.argtypes = [ctypes.c_void_p, ctypes.c_int]
        R.ref_alto_create128.restype = ctypes.c_void_p
        R.ref_alto_create128.argtypes = [ctypes.c_int, _u64p, ctypes.c_uint64, _u64p, _f64p, ctypes.c_int]
        R.ref_alto_mttkrp128.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        R.ref_alto_destroy128.argtypes = [ctypes.c_void_p, ctypes.c_int]
        R.ref_tns_import.restype = ctypes.c_void_p
        R.ref_tns_import.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), _u64p, _u64p]
        R.ref_tns_copy.argtypes = [ctypes.c_void_p, _u64p, _f64p]
        R.ref_tns_free.argtypes = [ctypes.c_void_p]
        R.ref_cpd_alto.restype = ctypes.c_int
        R.ref_cpd_alto.argtypes = [ctypes.c_int, _u64p, ctypes.c_uint64, _u64p, _f64p, ctypes.c_int, ctypes.c_void_p,
                                   _f64p, ctypes.c_int, ctypes.c_double, ctypes.c_int, _f64p, _f64p, _f64p]
        _ref = R
    return _ref


def ref_cpd_alto(dims, cidx, vals, factors, lam, iters, epsilon=0.0, nthreads=None):
    """The reference's CPU CP-ALS (cpd_alto, include/cpd.hpp:44-187) through
    oracle/_ref: factors (list of FP64 arrays) and lam are updated in place.
    Returns dict(iters, ms_per_iter, mttkrp_ms_per_iter, fit, threads) from
    its own report (the "Per iteration" line)."""
    R = ref_lib()
    if R is None:
        raise RuntimeError("oracle/_ref/libblco_ref.so is not built")
    dims = np.ascontiguousarray(dims, dtype=np.uint64)
    cidx = np.ascontiguousarray(cidx, dtype=np.uint64)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    nthreads = nthreads or (os.cpu_count() or 1)
    for f in factors:
        assert f.flags.c_contiguous and f.dtype == np.float64
    ptrs = (ctypes.c_void_p * len(factors))(*[f.ctypes.data for f in factors])
    out = np.zeros(3)
    n = R.ref_cpd_alto(len(dims), _p(dims, _u64p), cidx.shape[1], _p(cidx, _u64p), _p(vals, _f64p),
                       factors[0].shape[1], ptrs, _p(lam, _f64p), int(iters), float(epsilon), int(nthreads),
                       _p(out[0:1], _f64p), _p(out[1:2], _f64p), _p(out[2:3], _f64p))
    if n < 0:
        raise RuntimeError("cpd_alto report not found")
    return dict(iters=n, ms_per_iter=float(out[0]), mttkrp_ms_per_iter=float(out[1]), fit=float(out[2]),
                threads=nthreads)


def ref_import_tns(path):
    """The reference's .tns reader (ImportSparseTensor, src/sptensor.cpp:162)
    through oracle/_ref: (dims, cidx (nmodes x nnz, 0-based), vals)."""
    R = ref_lib()
    if R is None:
        raise RuntimeError("oracle/_ref/libblco_ref.so is not built")
    nm = ctypes.c_int()
    dims = np.zeros(8, dtype=np.uint64)
    nnz = np.zeros(1, dtype=np.uint64)
    h = R.ref_tns_import(os.fsencode(path), ctypes.byref(nm), _p(dims, _u64p), _p(nnz, _u64p))
    n = int(nnz[0])
    cidx = np.zeros((nm.value, n), dtype=np.uint64)
    vals = np.zeros(n, dtype=np.float64)
    R.ref_tns_copy(h, _p(cidx, _u64p), _p(vals, _f64p))
    R.ref_tns_free(h)
    return [int(d) for d in dims[:nm.value]], cidx, vals


def alto_masks(dims):
    dims = np.ascontiguousarray(dims, dtype=np.uint64)
    out = np.zeros(len(dims), dtype=np.uint64)
    bits = lib().orc_alto_masks(ctypes.c_int(len(dims)), _p(dims, _u64p), _p(out, _u64p))
    if bits < 0:
        raise ValueError("ALTO key wider than 64 bits")
    return out, bits


def _encode_with(fn, dims, cidx, vals, max_block_size, with_alto):
    dims = np.ascontiguousarray(dims, dtype=np.uint64)
    cidx = np.ascontiguousarray(cidx, dtype=np.uint64)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    nmodes, nnz = cidx.shape
    coords = np.zeros(nnz, dtype=np.uint64)
    ovals = np.zeros(nnz, dtype=np.float64)
    masks = np.zeros(nmodes, dtype=np.uint64)
    pos = np.zeros(nmodes, dtype=np.int32)
    nb = np.zeros(1, dtype=np.uint64)
    B = max_block_size if max_block_size else max(nnz, 1)
    offs = np.zeros(nnz // B + 2, dtype=np.uint64)
    if with_alto:
        amasks = np.zeros(nmodes, dtype=np.uint64)
        rc = fn(ctypes.c_int(nmodes), _p(dims, _u64p), ctypes.c_uint64(nnz), _p(cidx, _u64p),
                _p(vals, _f64p), ctypes.c_uint64(max_block_size), _p(coords, _u64p),
                _p(ovals, _f64p), _p(masks, _u64p), _p(pos, _i32p), _p(amasks, _u64p),
                _p(nb, _u64p), _p(offs, _u64p))
        extra = amasks
    else:
        bcoords = np.zeros((nnz // B + 2) * nmodes, dtype=np.uint64)
        rc = fn(ctypes.c_int(nmodes), _p(dims, _u64p), ctypes.c_uint64(nnz), _p(cidx, _u64p),
                _p(vals, _f64p), ctypes.c_uint64(max_block_size), _p(coords, _u64p),
                _p(ovals, _f64p), _p(masks, _u64p), _p(pos, _i32p), _p(nb, _u64p),
                _p(offs, _u64p), _p(bcoords, _u64p))
        extra = bcoords[: int(nb[0]) * nmodes].reshape(-1, nmodes)
    if rc != 0:
        raise ValueError("encode rejected the input")
    n_blocks = int(nb[0])
    return dict(coords=coords, vals=ovals, mode_masks=masks, mode_pos=pos,
                nblocks=n_blocks, block_offsets=offs[: n_blocks + 1].copy(), extra=extra)


def blco_encode(dims, cidx, vals, max_block_size=0):
    """Oracle encoder; returns dict with coords, vals, mode_masks, mode_pos,
    nblocks, block_offsets and alto_masks."""
    r = _encode_with(lib().orc_blco_encode, dims, cidx, vals, max_block_size, True)
    r["alto_masks"] = r.pop("extra")
    return r


def ref_blco_encode(dims, cidx, vals, max_block_size=0):
    """The reference encoder (oracle/_ref); same fields plus block_coords."""
    R = ref_lib()
    if R is None:
        raise FileNotFoundError("oracle/_ref not built")
    r = _encode_with(R.ref_blco_encode, dims, cidx, vals, max_block_size, False)
    r["block_coords"] = r.pop("extra")
    return r


def _encode128_with(fn, dims, cidx, vals, max_block_size, oracle):
    dims = np.ascontiguousarray(dims, dtype=np.uint64)
    cidx = np.ascontiguousarray(cidx, dtype=np.uint64)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    nmodes, nnz = cidx.shape
    coords = np.zeros(nnz, dtype=np.uint64)
    ovals = np.zeros(nnz, dtype=np.float64)
    masks = np.zeros(nmodes, dtype=np.uint64)
    pos = np.zeros(nmodes, dtype=np.int32)
    nb = np.zeros(1, dtype=np.uint64)
    offs = np.zeros(nnz + 2, dtype=np.uint64)
    bcoords = np.zeros((nnz + 1) * nmodes, dtype=np.uint64)
    args = [ctypes.c_int(nmodes), _p(dims, _u64p), ctypes.c_uint64(nnz), _p(cidx, _u64p), _p(vals, _f64p),
            ctypes.c_uint64(max_block_size), _p(coords, _u64p), _p(ovals, _f64p), _p(masks, _u64p),
            _p(pos, _i32p)]
    lo = np.zeros(nmodes, dtype=np.uint64)
    hi = np.zeros(nmodes, dtype=np.uint64)
    if oracle:
        args += [_p(lo, _u64p), _p(hi, _u64p)]
    args += [_p(nb, _u64p), _p(offs, _u64p), _p(bcoords, _u64p)]
    if fn(*args) != 0:
        raise ValueError("encode rejected the input")
    n_blocks = int(nb[0])
    r = dict(coords=coords, vals=ovals, mode_masks=masks, mode_pos=pos, nblocks=n_blocks,
             block_offsets=offs[: n_blocks + 1].copy(),
             block_coords=bcoords[: n_blocks * nmodes].reshape(-1, nmodes).copy())
    if oracle:
        r["alto_masks_lo"], r["alto_masks_hi"] = lo, hi
    return r


def blco_encode128(dims, cidx, vals, max_block_size=0):
    """Oracle encoder with 128-bit ALTO keys (the cpd128 build): coords,
    vals, mode_masks, mode_pos, nblocks, block_offsets, block_coords,
    alto_masks_lo / alto_masks_hi."""
    return _encode128_with(lib().orc_blco_encode128, dims, cidx, vals, max_block_size, True)


def ref_blco_encode128(dims, cidx, vals, max_block_size=0):
    """The reference encoder with 128-bit keys (oracle/_ref)."""
    R = ref_lib()
    if R is None:
        raise FileNotFoundError("oracle/_ref not built")
    return _encode128_with(R.ref_blco_encode128, dims, cidx, vals, max_block_size, False)


def mttkrp_blco128(enc, factors, mode, out=None):
    """MTTKRP over a blocked encoding (row = field | block coordinate)."""
    factors = [np.ascontiguousarray(f, dtype=np.float64) for f in factors]
    rank = factors[0].shape[1]
    nmodes = len(factors)
    if out is None:
        out = np.zeros((factors[mode].shape[0], rank), dtype=np.float64)
    masks = np.ascontiguousarray(enc["mode_masks"], dtype=np.uint64)
    pos = np.ascontiguousarray(enc["mode_pos"], dtype=np.int32)
    offs = np.ascontiguousarray(enc["block_offsets"], dtype=np.uint64)
    bc = np.ascontiguousarray(enc["block_coords"], dtype=np.uint64).reshape(-1)
    coords = np.ascontiguousarray(enc["coords"], dtype=np.uint64)
    vals = np.ascontiguousarray(enc["vals"], dtype=np.float64)
    lib().orc_mttkrp_blco128(ctypes.c_int(nmodes), _p(masks, _u64p), _p(pos, _i32p),
                             ctypes.c_uint64(enc["nblocks"]), _p(offs, _u64p), _p(bc, _u64p),
                             _p(coords, _u64p), _p(vals, _f64p), _ptr_array(factors), ctypes.c_int(rank),
                             ctypes.c_int(mode), _p(out, _f64p))
    return out


def mttkrp_coo(cidx, vals, factors, mode, out=None):
    cidx = np.ascontiguousarray(cidx, dtype=np.uint64)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    factors = [np.ascontiguousarray(f, dtype=np.float64) for f in factors]
    nmodes, nnz = cidx.shape
    rank = factors[0].shape[1]
    if out is None:
        out = np.zeros((factors[mode].shape[0], rank), dtype=np.float64)
    lib().orc_mttkrp_coo(ctypes.c_int(nmodes), ctypes.c_uint64(nnz), _p(cidx, _u64p),
                         _p(vals, _f64p), ctypes.c_int(rank), _ptr_array(factors),
                         ctypes.c_int(mode), _p(out, _f64p))
    return out


def mttkrp_blco(enc, factors, mode, out=None):
    factors = [np.ascontiguousarray(f, dtype=np.float64) for f in factors]
    rank = factors[0].shape[1]
    nmodes = len(factors)
    if out is None:
        out = np.zeros((factors[mode].shape[0], rank), dtype=np.float64)
    masks = np.ascontiguousarray(enc["mode_masks"], dtype=np.uint64)
    pos = np.ascontiguousarray(enc["mode_pos"], dtype=np.int32)
    coords = np.ascontiguousarray(enc["coords"], dtype=np.uint64)
    vals = np.ascontiguousarray(enc["vals"], dtype=np.float64)
    lib().orc_mttkrp_blco(ctypes.c_int(nmodes), _p(masks, _u64p), _p(pos, _i32p),
                          ctypes.c_uint64(len(coords)), _p(coords, _u64p), _p(vals, _f64p),
                          ctypes.c_int(rank), _ptr_array(factors), ctypes.c_int(mode),
                          _p(out, _f64p))
    return out


def pinv_sym(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    p = np.zeros_like(a)
    lib().orc_pinv_sym(ctypes.c_int(a.shape[0]), _p(a, _f64p), _p(p, _f64p))
    return p


def cpals(dims, enc, factors, lam, maxiter, tol):
    """Oracle CP-ALS (GPU semantics).  factors/lam are updated in place;
    returns the list of per-iteration fits."""
    dims = np.ascontiguousarray(dims, dtype=np.uint64)
    masks = np.ascontiguousarray(enc["mode_masks"], dtype=np.uint64)
    pos = np.ascontiguousarray(enc["mode_pos"], dtype=np.int32)
    coords = np.ascontiguousarray(enc["coords"], dtype=np.uint64)
    vals = np.ascontiguousarray(enc["vals"], dtype=np.float64)
    for f in factors:
        assert f.flags.c_contiguous and f.dtype == np.float64
    rank = factors[0].shape[1]
    fits = np.zeros(max(maxiter, 1), dtype=np.float64)
    it = lib().orc_cpals(ctypes.c_int(len(dims)), _p(dims, _u64p), _p(masks, _u64p),
                         _p(pos, _i32p), ctypes.c_uint64(len(coords)), _p(coords, _u64p),
                         _p(vals, _f64p), ctypes.c_int(rank), _ptr_array(factors),
                         _p(lam, _f64p), ctypes.c_int(maxiter), ctypes.c_double(tol),
                         _p(fits, _f64p))
    return list(fits[:it])


def cpals_coo(dims, cidx, vals, factors, lam, maxiter, tol):
    """Oracle CP-ALS with the MTTKRP taken from the COO tensor (any key
    width).  factors/lam are updated in place; returns the fits."""
    dims = np.ascontiguousarray(dims, dtype=np.uint64)
    cidx = np.ascontiguousarray(cidx, dtype=np.uint64)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    for f in factors:
        assert f.flags.c_contiguous and f.dtype == np.float64
    rank = factors[0].shape[1]
    fits = np.zeros(max(maxiter, 1), dtype=np.float64)
    it = lib().orc_cpals_coo(ctypes.c_int(len(dims)), _p(dims, _u64p), ctypes.c_uint64(cidx.shape[1]),
                             _p(cidx, _u64p), _p(vals, _f64p), ctypes.c_int(rank), _ptr_array(factors),
                             _p(lam, _f64p), ctypes.c_int(maxiter), ctypes.c_double(tol), _p(fits, _f64p))
    return list(fits[:it])


def kruskal_random_init(dims, rank, seed, nthreads):
    factors = [np.zeros((int(d), rank), dtype=np.float64) for d in dims]
    lam = np.zeros(rank, dtype=np.float64)
    dims = np.ascontiguousarray(dims, dtype=np.uint64)
    lib().orc_kruskal_random_init(ctypes.c_int(len(dims)), _p(dims, _u64p), ctypes.c_int(rank),
                                  ctypes.c_uint(seed), ctypes.c_int(nthreads),
                                  _ptr_array(factors), _p(lam, _f64p))
    return factors, lam


def refgpu_available():
    """True when the reference's GPU build (oracle/_ref/libblco_refgpu.so,
    `make -C oracle ref-gpu`) is present.  It needs a B200 to run."""
    return os.path.exists(os.path.join(HERE, "_ref", "libblco_refgpu.so"))


def _refgpu_call(req, log_path=None, timeout=600):
    """Runs one reference call in a child interpreter (the reference exits
    the process on CUDA errors); returns the result arrays."""
    import subprocess
    import sys
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        qp, rp = os.path.join(d, "req.npz"), os.path.join(d, "res.npz")
        np.savez(qp, **req)
        p = subprocess.run([sys.executable, os.path.join(HERE, "refgpu_run.py"), qp, rp],
                           capture_output=True, text=True, timeout=timeout)
        if log_path:
            with open(log_path, "a") as f:
                f.write(p.stdout + p.stderr)
        if p.returncode != 0 or not os.path.exists(rp):
            tail = (p.stdout + p.stderr)[-2000:]
            raise RuntimeError(f"reference GPU call failed (exit {p.returncode}):\n{tail}")
        return dict(np.load(rp))


def _req(dims, cidx, vals, factors, **kw):
    r = dict(dims=np.asarray(dims, dtype=np.uint64), cidx=np.asarray(cidx, dtype=np.uint64),
             vals=np.asarray(vals, dtype=np.float64), rank=np.int64(factors[0].shape[1]))
    for m, f in enumerate(factors):
        r[f"f{m}"] = np.asarray(f, dtype=np.float64)
    for k, v in kw.items():
        r[k] = np.asarray(v)
    return r


def refgpu_cpals(dims, cidx, vals, factors, lam, maxiter, tol, kernel=10, nprtn=8, thread_cf=2, log_path=None,
                 wide=False, timeout=600):
    """Runs the reference cpals_blco_dev (wide: on the 128-bit build's
    encoding); factors/lam updated in place; returns the final fit."""
    res = _refgpu_call(_req(dims, cidx, vals, factors, op="cpals", lam=lam, maxiter=maxiter, tol=tol,
                            kernel=kernel, nprtn=nprtn, thread_cf=thread_cf, wide=int(wide)), log_path, timeout)
    for m, f in enumerate(factors):
        f[:] = res[f"f{m}"]
    lam[:] = res["lam"]
    return float(res["fit"])


def refgpu_mttkrp(dims, cidx, vals, factors, mode, kernel=1, nprtn=8, thread_cf=2, log_path=None, wide=False,
                  iters=1):
    """Runs the reference mttkrp_alto_dev `iters` times into a zeroed target
    factor (wide: on the 128-bit build's encoding); returns the sum of the
    MTTKRPs.  The reference prints its per-iteration time to log_path."""
    fs = [np.array(f, dtype=np.float64) for f in factors]
    fs[mode][:] = 0.0
    res = _refgpu_call(_req(dims, cidx, vals, fs, op="mttkrp", mode=mode, kernel=kernel, nprtn=nprtn,
                            thread_cf=thread_cf, wide=int(wide), iters=iters), log_path)
    return res[f"f{mode}"]
