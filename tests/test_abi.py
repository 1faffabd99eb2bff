"""CPU tests of the C-ABI library: it loads, exports every declared symbol
and reports errors as status codes (no GPU work is launched here)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT, gpu_available


def declared_symbols():
    with open(os.path.join(ROOT, "include", "blco.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(blco_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree(blco):
    assert declared_symbols() == sorted(blco.EXPORTS)


def test_library_exports_every_declared_symbol(blco):
    L = blco.lib()
    for name in declared_symbols():
        assert hasattr(L, name), name


def test_host_only_calls(blco):
    assert blco.version().startswith("blco_b200")
    o = blco.make_opts(stream=0)
    assert o.kernel == blco.KERNEL_AUTO and o.thread_cf == 2 and o.precision == blco.PRECISION_FP64
    L = blco.lib()
    assert L.blco_status_string(blco.ERR_INVALID).decode() == "invalid argument"
    assert L.blco_status_string(99).decode() == "unknown status"


def test_argument_errors_are_status_codes(blco):
    L = blco.lib()
    h = ctypes.c_void_p()
    # nmodes out of range is rejected before any CUDA call
    st = L.blco_encode(0, None, 0, None, None, 0, None, ctypes.byref(h))
    assert st == blco.ERR_INVALID
    assert "nmodes" in L.blco_last_error().decode()
    st = L.blco_encode(6, None, 0, None, None, 0, None, ctypes.byref(h))
    assert st == blco.ERR_INVALID
    assert L.blco_mttkrp(None, 0, 4, None, None, None) == blco.ERR_INVALID
    assert L.blco_cpals(None, 4, None, None, 5, 0.0, None, None, None, None) == blco.ERR_INVALID
    assert L.blco_tensor_free(None) == blco.OK


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU error path")
def test_no_device_is_an_error_not_a_crash(blco):
    import numpy as np
    with pytest.raises(blco.BlcoError) as e:
        blco.Tensor.encode([4, 4], np.zeros((2, 1), dtype=np.uint64), np.ones(1), opts=blco.make_opts(stream=0))
    assert e.value.status in (blco.ERR_CUDA, blco.ERR_UNSUPPORTED)
