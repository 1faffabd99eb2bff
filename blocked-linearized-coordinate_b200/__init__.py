"""Python binding of libblco_b200 (ctypes over the C ABI in include/blco.h).

The engine is the CUDA/C++ library lib/libblco_b200.so built for sm_100a by
`make -C blocked-linearized-coordinate_b200`.  This module only marshals
pointers: host arrays are numpy arrays, device arrays are torch CUDA tensors
(torch is used for device memory and streams, nothing else).  Every call
raises BlcoError when the library returns a non-zero status; there is no
fallback path.

Entry points mirror the reference's in-process interface
(jeewhanchoi/blocked-linearized-coordinate):
  encode / encode_device   gen_blcotensor_host<u64> (include/blco.hpp:196)
  mttkrp / mttkrp_host     mttkrp_alto_dev_onemode (src/alto_dev.cu:1955)
  cpals                    cpals_blco_dev (src/cpd_gpu.cu:21)
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libblco_b200.so")
MAX_MODES = 5

OK = 0
ERR_INVALID = 1
ERR_UNSUPPORTED = 2
ERR_CUDA = 3
ERR_NOMEM = 4
ERR_TIMEOUT = 5
ERR_IO = 6
ERR_STATE = 7

KERNEL_AUTO = 10
KERNEL_LVL1 = 1
KERNEL_LVL2 = 2
KERNEL_LVL3 = 3
KERNEL_FIBRE = 4
SOLVE_AUTO = 0
SOLVE_PINV = 1
GUARD_COND = 3e4
KERNEL_BATCHED = 11
KERNEL_BATCHED_V2 = 12
KERNEL_ATOMIC = 13

PRECISION_FP64 = 0
PRECISION_MIXED = 1
PRECISION_MIXED_BF16 = 2

KERNEL_TUNED = 20
KERNEL_LEARNED = 21
TUNE_CONFIGS = 14
MLP_FEATURES = 25
DTYPE_F64 = 0
DTYPE_F32 = 1
DTYPE_BF16 = 2

# Every symbol include/blco.h declares.
EXPORTS = (
    "blco_opts_init", "blco_status_string", "blco_last_error", "blco_version",
    "blco_encode", "blco_encode_device", "blco_encode_device_noalloc", "blco_tensor_free", "blco_tensor_get_info",
    "blco_tensor_copy_out", "blco_tensor_device_arrays", "blco_mttkrp", "blco_mttkrp_ex", "blco_mttkrp_host",
    "blco_cpals", "blco_cpals_plan_create", "blco_cpals_plan_iterate",
    "blco_cpals_plan_mttkrp_ms", "blco_cpals_plan_condition", "blco_cpals_plan_device_bytes", "blco_cpals_plan_destroy", "blco_batch_create",
    "blco_batch_iterate",
    "blco_batch_destroy", "blco_batch_last_ms", "blco_batch_mttkrp_ms", "blco_tune_space", "blco_autotune", "blco_tune_features",
    "blco_mlp_create", "blco_mlp_num_params", "blco_mlp_set_params", "blco_mlp_get_params", "blco_mlp_predict",
    "blco_mlp_grad", "blco_mlp_train", "blco_mlp_destroy", "blco_selector_set", "blco_select", "blco_gram_f32",
    "blco_encode_tns", "blco_gram_tc_timeout_check", "blco_parse_decimal", "blco_launch_count", "blco_cpals_plan_set_reduce",
    "blco_cpals_plan_set_norm_sq", "blco_tensor_fibre_stats",
)


class BlcoError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{msg} [status {status}]")
        self.status = status


class Opts(ctypes.Structure):
    _fields_ = [
        ("kernel", ctypes.c_int),
        ("nprtn", ctypes.c_int),
        ("thread_cf", ctypes.c_int),
        ("stream_data", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("verbose", ctypes.c_int),
        ("device", ctypes.c_int),
        ("residency_bytes", ctypes.c_uint64),
        ("stream", ctypes.c_void_p),
        ("gram_tensor_cores", ctypes.c_int),
        ("solve", ctypes.c_int),
        ("guard_cond", ctypes.c_double),
    ]


class TensorInfo(ctypes.Structure):
    _fields_ = [
        ("nmodes", ctypes.c_int),
        ("dims", ctypes.c_uint64 * MAX_MODES),
        ("nnz", ctypes.c_uint64),
        ("block_count", ctypes.c_uint64),
        ("max_block_size", ctypes.c_uint64),
        ("mode_masks", ctypes.c_uint64 * MAX_MODES),
        ("mode_pos", ctypes.c_int * MAX_MODES),
        ("alto_masks", ctypes.c_uint64 * MAX_MODES),
        ("alto_bits", ctypes.c_int),
        ("device", ctypes.c_int),
        ("resident", ctypes.c_int),
        ("alto_masks_hi", ctypes.c_uint64 * MAX_MODES),
    ]


_lib = None


def lib():
    """Load the library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is not built; run make -C {HERE}")
        L = ctypes.CDLL(LIB_PATH)
        vp, u64, i32, f64 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_double
        L.blco_status_string.restype = ctypes.c_char_p
        L.blco_last_error.restype = ctypes.c_char_p
        L.blco_version.restype = ctypes.c_char_p
        L.blco_launch_count.restype = u64
        L.blco_launch_count.argtypes = [i32]
        L.blco_opts_init.argtypes = [vp]
        L.blco_encode.argtypes = [i32, vp, u64, vp, vp, u64, vp, vp]
        L.blco_encode_device.argtypes = [i32, vp, u64, vp, vp, u64, vp, vp]
        L.blco_encode_device_noalloc.argtypes = [i32, vp, u64, vp, vp, vp, vp, vp]
        L.blco_tensor_free.argtypes = [vp]
        L.blco_tensor_get_info.argtypes = [vp, vp]
        L.blco_tensor_copy_out.argtypes = [vp, vp, vp, vp, vp]
        L.blco_tensor_device_arrays.argtypes = [vp, vp, vp]
        L.blco_mttkrp.argtypes = [vp, i32, i32, vp, vp, vp]
        L.blco_mttkrp_host.argtypes = [vp, i32, i32, vp, vp, vp]
        L.blco_mttkrp_ex.argtypes = [vp, i32, i32, i32, vp, vp, vp]
        L.blco_cpals.argtypes = [vp, i32, vp, vp, i32, f64, vp, vp, vp, vp]
        L.blco_cpals_plan_create.argtypes = [vp, i32, vp, vp, vp, vp]
        L.blco_cpals_plan_iterate.argtypes = [vp, i32, f64, vp, vp]
        L.blco_cpals_plan_mttkrp_ms.argtypes = [vp, vp, vp]
        L.blco_cpals_plan_condition.argtypes = [vp, vp, vp]
        L.blco_cpals_plan_device_bytes.argtypes = [vp, vp]
        L.blco_tensor_fibre_stats.argtypes = [vp, i32, vp]
        L.blco_cpals_plan_destroy.argtypes = [vp]
        L.blco_batch_create.argtypes = [i32, vp, vp, vp, vp, f64, vp, vp]
        L.blco_batch_iterate.argtypes = [vp, i32, vp, vp]
        L.blco_batch_destroy.argtypes = [vp]
        L.blco_batch_last_ms.argtypes = [vp, vp]
        L.blco_tune_space.argtypes = [vp]
        L.blco_autotune.argtypes = [vp, i32, i32, i32, i32, vp, vp, vp]
        L.blco_tune_features.argtypes = [vp, i32, i32, i32, vp]
        L.blco_mlp_create.argtypes = [i32, u64, i32, vp]
        L.blco_mlp_num_params.argtypes = [vp, vp]
        L.blco_mlp_set_params.argtypes = [vp, vp, i32]
        L.blco_mlp_get_params.argtypes = [vp, vp, i32]
        L.blco_mlp_predict.argtypes = [vp, vp, i32, vp]
        L.blco_mlp_grad.argtypes = [vp, vp, vp, vp, i32, vp, vp]
        L.blco_mlp_train.argtypes = [vp, vp, vp, vp, i32, i32, i32, ctypes.c_float, u64, vp]
        L.blco_mlp_destroy.argtypes = [vp]
        L.blco_selector_set.argtypes = [vp, ctypes.c_float]
        L.blco_select.argtypes = [vp, i32, i32, i32, vp, ctypes.c_float, vp, vp, vp]
        L.blco_gram_f32.argtypes = [vp, u64, i32, vp, i32, i32, vp]
        L.blco_encode_tns.argtypes = [ctypes.c_char_p, u64, vp, vp, vp]
        L.blco_parse_decimal.argtypes = [ctypes.c_char_p, i32, vp, vp]
        _lib = L
    return _lib


def _check(status):
    if status != OK:
        raise BlcoError(status, lib().blco_last_error().decode() or lib().blco_status_string(status).decode())


def version():
    return lib().blco_version().decode()


def launch_count(reset=False):
    return int(lib().blco_launch_count(1 if reset else 0))


def make_opts(kernel=KERNEL_AUTO, nprtn=0, thread_cf=2, stream_data=False, precision=PRECISION_FP64,
              verbose=False, device=0, residency_bytes=0, stream=None, gram_tensor_cores=None, solve=SOLVE_AUTO,
              guard_cond=0.0):
    o = Opts()
    lib().blco_opts_init(ctypes.byref(o))
    o.kernel, o.nprtn, o.thread_cf = kernel, nprtn, thread_cf
    o.stream_data, o.precision, o.verbose = int(stream_data), precision, int(verbose)
    o.device, o.residency_bytes = device, residency_bytes
    # None: the default engine per rank; True / False: tensor / CUDA cores
    o.gram_tensor_cores = 0 if gram_tensor_cores is None else (1 if gram_tensor_cores else -1)
    o.solve, o.guard_cond = int(solve), float(guard_cond)
    if stream is None:
        try:
            import torch
            if torch.cuda.is_available():
                stream = torch.cuda.current_stream(device).cuda_stream
        except ImportError:
            stream = None
    o.stream = stream
    return o


def _u64arr(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def _ptrs(ptr_list):
    return (ctypes.c_void_p * len(ptr_list))(*ptr_list)


class TnsInfo(ctypes.Structure):
    _fields_ = [("nmodes", ctypes.c_int), ("dims", ctypes.c_uint64 * 5), ("nnz", ctypes.c_uint64),
                ("lines", ctypes.c_uint64), ("host_parsed", ctypes.c_uint64)]


class Tensor:
    """An encoded BLCO tensor owned by the library."""

    def __init__(self, handle):
        self._h = ctypes.c_void_p(handle)

    @property
    def handle(self):
        return self._h

    @classmethod
    def encode(cls, dims, cidx, vals, max_block_size=0, opts=None):
        """Encode host COO arrays: cidx is (nmodes, nnz) 0-based, vals (nnz,)."""
        dims = _u64arr(dims)
        cidx = _u64arr(cidx)
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        nmodes, nnz = cidx.shape
        ptrs = _ptrs([cidx[n].ctypes.data for n in range(nmodes)])
        h = ctypes.c_void_p()
        o = opts if opts is not None else make_opts()
        _check(lib().blco_encode(nmodes, dims.ctypes.data, nnz, ptrs, vals.ctypes.data, max_block_size,
                                 ctypes.byref(o), ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def encode_device(cls, dims, d_cidx, d_vals, max_block_size=0, opts=None):
        """Encode COO arrays already on the GPU (torch int64/uint64 and float64)."""
        dims = _u64arr(dims)
        nmodes = len(d_cidx)
        nnz = int(d_vals.numel())
        ptrs = _ptrs([int(c.data_ptr()) for c in d_cidx])
        h = ctypes.c_void_p()
        o = opts if opts is not None else make_opts()
        _check(lib().blco_encode_device(nmodes, dims.ctypes.data, nnz, ptrs, int(d_vals.data_ptr()),
                                        max_block_size, ctypes.byref(o), ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def encode_tns(cls, path, max_block_size=0, opts=None):
        """Parse a .tns file on the GPU and encode it (blco_encode_tns).
        Returns (Tensor, dict(nmodes, dims, nnz, lines, host_parsed))."""
        h = ctypes.c_void_p()
        inf = TnsInfo()
        o = opts if opts is not None else make_opts()
        _check(lib().blco_encode_tns(os.fsencode(path), max_block_size, ctypes.byref(o), ctypes.byref(h),
                                     ctypes.byref(inf)))
        n = inf.nmodes
        return cls(h.value), dict(nmodes=n, dims=list(inf.dims[:n]), nnz=inf.nnz, lines=inf.lines,
                                  host_parsed=inf.host_parsed)

    def info(self):
        inf = TensorInfo()
        _check(lib().blco_tensor_get_info(self._h, ctypes.byref(inf)))
        n = inf.nmodes
        return dict(nmodes=n, dims=list(inf.dims[:n]), nnz=inf.nnz, block_count=inf.block_count,
                    max_block_size=inf.max_block_size, mode_masks=list(inf.mode_masks[:n]),
                    mode_pos=list(inf.mode_pos[:n]), alto_masks=list(inf.alto_masks[:n]),
                    alto_masks_hi=list(inf.alto_masks_hi[:n]), alto_bits=inf.alto_bits, device=inf.device,
                    resident=bool(inf.resident))

    def copy_out(self):
        inf = self.info()
        nnz, nb, n = inf["nnz"], inf["block_count"], inf["nmodes"]
        coords = np.zeros(nnz, dtype=np.uint64)
        vals = np.zeros(nnz, dtype=np.float64)
        offs = np.zeros(nb + 1, dtype=np.uint64)
        bcoords = np.zeros(max(nb * n, 1), dtype=np.uint64)
        _check(lib().blco_tensor_copy_out(self._h, coords.ctypes.data, vals.ctypes.data, offs.ctypes.data,
                                          bcoords.ctypes.data))
        return dict(coords=coords, vals=vals, block_offsets=offs, block_coords=bcoords[: nb * n].reshape(nb, n),
                    **inf)

    def fibre_stats(self, mode):
        """Statistics of the mode's compressed-fibre copy (kernel id 4):
        dict(fibre_mode, fibred_nnz, single_nnz, fibres, rows_gathered)."""
        st = np.zeros(5, dtype=np.uint64)
        _check(lib().blco_tensor_fibre_stats(self.handle, mode, st.ctypes.data))
        return dict(fibre_mode=int(st[0]), fibred_nnz=int(st[1]), single_nnz=int(st[2]), fibres=int(st[3]),
                    rows_gathered=int(st[4]))

    def free(self):
        if self._h and self._h.value:
            _check(lib().blco_tensor_free(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


NOALLOC_MAX_NNZ = 1_900_000  # BLCO_NOALLOC_MAX_NNZ in include/blco.h


def encode_device_noalloc(dims, d_cidx, d_vals, d_coords_out, d_vals_out, stream=None):
    """Allocation-free encode (blco_encode_device_noalloc): COO torch CUDA
    arrays in, BLCO coordinates/values written to the caller's torch CUDA
    arrays (uint64/int64 and float64, nnz entries).  Uses the library's
    fixed device scratch array; no device memory is allocated."""
    dims = _u64arr(dims)
    nnz = int(d_vals.numel())
    ptrs = _ptrs([int(c.data_ptr()) for c in d_cidx])
    if stream is None:
        import torch
        stream = torch.cuda.current_stream().cuda_stream
    _check(lib().blco_encode_device_noalloc(len(d_cidx), dims.ctypes.data, nnz, ptrs, int(d_vals.data_ptr()),
                                            int(d_coords_out.data_ptr()), int(d_vals_out.data_ptr()), stream))


def mttkrp(t, mode, factors, out, opts=None):
    """out (torch CUDA float64, dims[mode] x R) += MTTKRP; factors are torch
    CUDA float64 row-major matrices (factors[mode] may be None)."""
    rank = int(out.shape[1])
    ptrs = _ptrs([int(f.data_ptr()) if f is not None else 0 for f in factors])
    o = opts if opts is not None else make_opts()
    _check(lib().blco_mttkrp(t.handle, mode, rank, ptrs, int(out.data_ptr()), ctypes.byref(o)))


def mttkrp_ex(t, mode, factors, out, factor_dtype, opts=None):
    """Mixed-precision MTTKRP: out (torch CUDA float32) += MTTKRP with
    torch CUDA float32 or bfloat16 factors."""
    rank = int(out.shape[1])
    ptrs = _ptrs([int(f.data_ptr()) if f is not None else 0 for f in factors])
    o = opts if opts is not None else make_opts()
    _check(lib().blco_mttkrp_ex(t.handle, mode, rank, factor_dtype, ptrs, int(out.data_ptr()), ctypes.byref(o)))


def mttkrp_host(t, mode, factors, out=None, opts=None):
    """Host numpy version; returns out (+)= MTTKRP."""
    factors = [np.ascontiguousarray(f, dtype=np.float64) for f in factors]
    rank = factors[0].shape[1]
    if out is None:
        out = np.zeros((factors[mode].shape[0], rank), dtype=np.float64)
    ptrs = _ptrs([f.ctypes.data for f in factors])
    o = opts if opts is not None else make_opts()
    _check(lib().blco_mttkrp_host(t.handle, mode, rank, ptrs, out.ctypes.data, ctypes.byref(o)))
    return out


def cpals(t, factors, lam, maxiter, tol, opts=None):
    """CP-ALS with host numpy factors (updated in place).  Returns
    (final_fit, per-iteration fits)."""
    for f in factors:
        if not (f.flags.c_contiguous and f.dtype == np.float64):
            raise ValueError("factors must be C-contiguous float64")
    rank = factors[0].shape[1]
    fits = np.zeros(max(maxiter, 1), dtype=np.float64)
    fit = ctypes.c_double()
    iters = ctypes.c_int()
    ptrs = _ptrs([f.ctypes.data for f in factors])
    o = opts if opts is not None else make_opts()
    _check(lib().blco_cpals(t.handle, rank, ptrs, lam.ctypes.data, maxiter, tol, ctypes.byref(o),
                            ctypes.byref(fit), fits.ctypes.data, ctypes.byref(iters)))
    return fit.value, list(fits[: iters.value])


# int fn(void* ctx, void* d_buf, uint64_t count, int dtype, void* stream)
REDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int,
                             ctypes.c_void_p)


class _DeviceBuf:
    """A CUDA array view of a raw device pointer (no copy)."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = dict(shape=(int(count),), typestr=typestr, data=(int(ptr), False),
                                             version=2)


def dist_reduce(dist, group=None, via_host=False, view=None):
    """A reduce hook for CpalsPlan.set_reduce from a torch.distributed
    process group: the MTTKRP buffer is summed over the ranks on the plan's
    stream (dist.all_reduce; NCCL puts it on that stream's timeline).  With
    via_host the sum goes through host copies (for the gloo backend).
    view(ptr, count, dtype) -> tensor overrides the device view (tests)."""
    import torch

    def fn(ptr, count, dtype, stream):
        tdt = torch.float64 if dtype == DTYPE_F64 else torch.float32
        if view is not None:
            t = view(ptr, count, dtype)
        else:
            t = torch.as_tensor(_DeviceBuf(ptr, count, "<f8" if dtype == DTYPE_F64 else "<f4"), device="cuda")
            assert t.dtype == tdt
        ctx = torch.cuda.stream(torch.cuda.ExternalStream(stream)) if stream and t.is_cuda else None
        if ctx is not None:
            ctx.__enter__()
        try:
            if via_host and t.is_cuda:
                h = t.cpu()
                dist.all_reduce(h, group=group)
                t.copy_(h)
            else:
                dist.all_reduce(t, group=group)
        finally:
            if ctx is not None:
                ctx.__exit__(None, None, None)

    return fn


class CpalsPlan:
    """Device-resident CP-ALS over torch CUDA factors (owned by the caller)."""

    def __init__(self, t, factors, lam, opts=None):
        self._t = t
        self._keep = (factors, lam)
        self.nmodes = len(factors)
        ptrs = _ptrs([int(f.data_ptr()) for f in factors])
        h = ctypes.c_void_p()
        o = opts if opts is not None else make_opts()
        self._opts = o
        _check(lib().blco_cpals_plan_create(t.handle, int(factors[0].shape[1]), ptrs, int(lam.data_ptr()),
                                            ctypes.byref(o), ctypes.byref(h)))
        self._h = h

    def iterate(self, iters, tol=-1.0):
        fits = np.zeros(max(iters, 1), dtype=np.float64)
        done = ctypes.c_int()
        _check(lib().blco_cpals_plan_iterate(self._h, iters, tol, fits.ctypes.data, ctypes.byref(done)))
        return list(fits[: done.value])

    def set_reduce(self, fn):
        """Sharded tensor: fn(d_ptr, count, dtype, stream) must sum the
        MTTKRP buffer over the ranks on that stream (see dist_reduce);
        None removes the hook."""
        if fn is None:
            self._reduce = None
            _check(lib().blco_cpals_plan_set_reduce(self._h, None, None))
            return

        def cb(ctx, ptr, count, dtype, stream):
            try:
                fn(ptr, count, dtype, stream)
                return 0
            except Exception:  # reported as a failed exchange
                import traceback
                traceback.print_exc()
                return 1

        self._reduce = REDUCE_FN(cb)  # kept alive with the plan
        _check(lib().blco_cpals_plan_set_reduce(self._h, self._reduce, None))

    def set_norm_sq(self, norm_sq):
        """||X||^2 of the whole (sharded) tensor, for the fit."""
        _check(lib().blco_cpals_plan_set_norm_sq(self._h, ctypes.c_double(float(norm_sq))))

    def mttkrp_ms(self):
        ms = np.zeros(self.nmodes, dtype=np.float64)
        calls = ctypes.c_int()
        _check(lib().blco_cpals_plan_mttkrp_ms(self._h, ms.ctypes.data, ctypes.byref(calls)))
        return ms, calls.value

    def device_bytes(self):
        """Device bytes the plan holds (factors, workspace, streamed ring)."""
        b = ctypes.c_uint64()
        _check(lib().blco_cpals_plan_device_bytes(self._h, ctypes.byref(b)))
        return b.value

    def condition(self):
        """(condition estimate of every mode's last solve, promoted to FP64)."""
        c = np.zeros(self.nmodes, dtype=np.float64)
        pr = ctypes.c_int()
        _check(lib().blco_cpals_plan_condition(self._h, c.ctypes.data, ctypes.byref(pr)))
        return c, bool(pr.value)

    def destroy(self):
        if self._h and self._h.value:
            _check(lib().blco_cpals_plan_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Batch:
    """Batched CP-ALS over many resident tensors (blco_batch_*).

    tensors: list of Tensor; factors[t]: list of torch CUDA float64
    (dims[n], rank_t) tensors; lams[t]: torch CUDA float64 (rank_t,).
    Factors and lambdas are updated in place."""

    def __init__(self, tensors, factors, lams, tol=1e-5, opts=None):
        T = len(tensors)
        self.count = T
        self._keep = (tensors, factors, lams)
        ranks = (ctypes.c_int * T)(*[int(f[0].shape[1]) for f in factors])
        rows = [_ptrs([int(m.data_ptr()) for m in f]) for f in factors]
        self._rows = rows
        fptrs = (ctypes.c_void_p * T)(*[ctypes.cast(r, ctypes.c_void_p).value for r in rows])
        lptrs = _ptrs([int(l.data_ptr()) for l in lams])
        hs = _ptrs([int(t.handle.value) for t in tensors])
        o = opts if opts is not None else make_opts()
        h = ctypes.c_void_p()
        _check(lib().blco_batch_create(T, hs, ranks, fptrs, lptrs, float(tol), ctypes.byref(o), ctypes.byref(h)))
        self._h = h

    def iterate(self, iters):
        """Run `iters` sweeps; returns (fits (iters, count), iterations per tensor)."""
        fits = np.zeros((max(iters, 1), self.count), dtype=np.float64)
        done = np.zeros(self.count, dtype=np.int32)
        _check(lib().blco_batch_iterate(self._h, iters, fits.ctypes.data, done.ctypes.data))
        return fits[:iters], done

    def last_ms(self):
        """Device milliseconds of the sweeps of the last iterate call."""
        ms = ctypes.c_double()
        _check(lib().blco_batch_last_ms(self._h, ctypes.byref(ms)))
        return ms.value

    def mttkrp_ms(self):
        """Device milliseconds of one sweep's MTTKRP launches alone."""
        ms = ctypes.c_double()
        _check(lib().blco_batch_mttkrp_ms(self._h, ctypes.byref(ms)))
        return ms.value

    def destroy(self):
        if self._h and self._h.value:
            _check(lib().blco_batch_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class TuneConfig(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int), ("hot_chunk", ctypes.c_int), ("interleave", ctypes.c_int)]


def tune_space():
    """The autotuner's schedules: list of dict(kernel, hot_chunk, interleave)."""
    arr = (TuneConfig * TUNE_CONFIGS)()
    _check(lib().blco_tune_space(arr))
    return [dict(kernel=c.kernel, hot_chunk=c.hot_chunk, interleave=c.interleave) for c in arr]


def autotune(t, mode, rank, factor_dtype=DTYPE_F64, reps=3, opts=None):
    """Exhaustive sweep: (ms per schedule as numpy float32, -1 = not valid; best index)."""
    ms = np.zeros(TUNE_CONFIGS, dtype=np.float32)
    best = ctypes.c_int()
    o = opts if opts is not None else make_opts()
    _check(lib().blco_autotune(t.handle, mode, rank, factor_dtype, reps, ctypes.byref(o), ms.ctypes.data,
                               ctypes.byref(best)))
    return ms, best.value


def tune_features(t, mode, rank, factor_dtype=DTYPE_F64):
    f = np.zeros(MLP_FEATURES, dtype=np.float32)
    _check(lib().blco_tune_features(t.handle, mode, rank, factor_dtype, f.ctypes.data))
    return f


class Mlp:
    """The schedule selector network (blco_mlp_*), trained on the GPU by the
    library's kernels."""

    def __init__(self, hidden=64, seed=0, device=0):
        h = ctypes.c_void_p()
        _check(lib().blco_mlp_create(hidden, seed, device, ctypes.byref(h)))
        self._h = h
        n = ctypes.c_int()
        _check(lib().blco_mlp_num_params(h, ctypes.byref(n)))
        self.nparams = n.value
        self.hidden = hidden

    @property
    def handle(self):
        return self._h

    def params(self):
        p = np.zeros(self.nparams, dtype=np.float32)
        _check(lib().blco_mlp_get_params(self._h, p.ctypes.data, self.nparams))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(lib().blco_mlp_set_params(self._h, p.ctypes.data, int(p.size)))

    def predict(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.zeros((X.shape[0], TUNE_CONFIGS), dtype=np.float32)
        _check(lib().blco_mlp_predict(self._h, X.ctypes.data, X.shape[0], out.ctypes.data))
        return out

    def grad(self, X, Y, M):
        X, Y, M = (np.ascontiguousarray(a, dtype=np.float32) for a in (X, Y, M))
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = ctypes.c_float()
        _check(lib().blco_mlp_grad(self._h, X.ctypes.data, Y.ctypes.data, M.ctypes.data, X.shape[0], g.ctypes.data,
                                   ctypes.byref(loss)))
        return g, loss.value

    def train(self, X, Y, M, epochs=200, batch=64, lr=1e-3, seed=0):
        X, Y, M = (np.ascontiguousarray(a, dtype=np.float32) for a in (X, Y, M))
        loss = ctypes.c_float()
        _check(lib().blco_mlp_train(self._h, X.ctypes.data, Y.ctypes.data, M.ctypes.data, X.shape[0], epochs, batch,
                                    ctypes.c_float(lr), seed, ctypes.byref(loss)))
        return loss.value

    def destroy(self):
        if self._h and self._h.value:
            _check(lib().blco_mlp_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def selector_set(net, margin=0.1):
    _check(lib().blco_selector_set(net.handle if net is not None else None, ctypes.c_float(margin)))


def select(t, mode, rank, factor_dtype=DTYPE_F64, net=None, margin=0.1, opts=None):
    """(schedule index, used_sweep) as kernel id 21 would choose."""
    cfg = ctypes.c_int()
    sw = ctypes.c_int()
    o = opts if opts is not None else make_opts()
    _check(lib().blco_select(t.handle, mode, rank, factor_dtype, net.handle if net is not None else None,
                             ctypes.c_float(margin), ctypes.byref(o), ctypes.byref(cfg), ctypes.byref(sw)))
    return cfg.value, bool(sw.value)


def gram_tc_timeout_check(device=0):
    """(status of a tensor-core Gram launch whose completion wait is made to
    run out, status of an ordinary launch after it)."""
    a, b = ctypes.c_int(), ctypes.c_int()
    _check(lib().blco_gram_tc_timeout_check(device, ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


def gram_f32(U, tensor_cores=True):
    """G = U^T U (torch CUDA float64) for a torch CUDA float32 matrix U (I x R, R <= 64)."""
    import torch
    U = U.contiguous()
    R = int(U.shape[1])
    G = torch.empty(R, R, dtype=torch.float64, device=U.device)
    stream = torch.cuda.current_stream(U.device).cuda_stream
    _check(lib().blco_gram_f32(int(U.data_ptr()), int(U.shape[0]), R, int(G.data_ptr()), int(bool(tensor_cores)),
                               U.device.index or 0, stream))
    return G


_default_net = None


def default_selector(margin=0.1, path=None):
    """Load the committed trained selector (selector/selector_params.npz,
    made by selector/train_selector.py) and make it the network kernel id
    21 uses.  Returns the network; the module keeps it alive."""
    global _default_net
    path = path or os.path.join(HERE, "selector", "selector_params.npz")
    d = np.load(path)
    net = Mlp(hidden=int(d["hidden"]), seed=0)
    net.set_params(d["params"])
    selector_set(net, margin)
    _default_net = net
    return net


def parse_decimal(text):
    """The GPU loader's decimal conversion, run on the host:
    (status, value, consumed); status 0 decided, 1 left to strtod, 2 none."""
    b = text.encode() if isinstance(text, str) else bytes(text)
    out = ctypes.c_double()
    used = ctypes.c_int()
    st = lib().blco_parse_decimal(b, len(b), ctypes.byref(out), ctypes.byref(used))
    return st, out.value, used.value
