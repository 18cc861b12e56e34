"""CPU checks of the C ABI boundary: the library loads, exports every function declared in
include/pme_recip.h, and rejects bad arguments before touching the GPU."""
import ctypes
import os
import re

import pytest

from gpu_recip_b200 import _capi
from gpu_recip_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not hdr.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:PME_API\s+)?(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*(pme_[a-z0-9_]+)\s*\(", text, re.M):
            names.append(m.group(1))
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    B.build()
    return _capi.load()


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("pme_create", "pme_spread_charge", "pme_r2c_fft", "pme_scalar_sum", "pme_c2r_fft",
                 "pme_gather_force", "pme_calc_self_energy", "pme_eval_ortho"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    raw = ctypes.CDLL(_capi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(raw, n)]
    assert not missing, missing
    # and the Python bindings cover them all
    assert sorted(set(declared_functions()) - set(_capi.SIGNATURES)) == []


def test_status_strings(lib):
    assert lib.pme_status_string(0) == b"PME_OK"
    assert lib.pme_status_string(-2) == b"PME_EUNSUPPORTED"
    assert lib.pme_version() >= 100


@pytest.mark.parametrize("args,status", [
    ((64, 64, 64, 5, 2, 1, 0), _capi.PME_EINVAL),          # order
    ((64, 64, 64, 4, 2, 2, 0), _capi.PME_EUNSUPPORTED),    # multi-node
    ((64, 64, 64, 4, 7, 1, 0), _capi.PME_EINVAL),          # fft type
    ((3, 64, 64, 4, 2, 1, 0), _capi.PME_EINVAL),           # grid < order
    ((64, 64, 1024, 4, 2, 1, 0), _capi.PME_EINVAL),        # grid > 512
    ((64, 49, 64, 4, 2, 1, 0), _capi.PME_EUNSUPPORTED),    # prime factor 7
])
def test_create_validates_before_gpu(lib, args, status):
    h = ctypes.c_void_p()
    rc = lib.pme_create(*args, ctypes.c_void_p(0), ctypes.byref(h))
    assert rc == status
    assert h.value is None
    assert lib.pme_last_error_string()


def test_null_handle_rejected(lib):
    assert lib.pme_r2c_fft(None) == _capi.PME_EINVAL
    assert lib.pme_destroy(None) == _capi.PME_OK


def test_trace_buffer_sizing_host_logic():
    """The trace hook's buffer check (no GPU needed): 14 entries per CTA plus the 32 step stamps
    of a single-system trace must fit, and only an int64 CUDA buffer is accepted."""
    import torch
    from gpu_recip_b200.pme import TRACE_STEP_STAMPS, _trace_ctas

    class Buf:
        def __init__(self, n, dtype=torch.int64, cuda=True):
            self.n, self.dtype, self.is_cuda = n, dtype, cuda

        def numel(self):
            return self.n

    assert _trace_ctas(Buf(100 * 14 + TRACE_STEP_STAMPS), 0, TRACE_STEP_STAMPS) == 100
    assert _trace_ctas(Buf(100 * 14), 0, 0) == 100
    assert _trace_ctas(Buf(100 * 14 + TRACE_STEP_STAMPS), 64, TRACE_STEP_STAMPS) == 64
    for bad in (Buf(100 * 14), Buf(13), Buf(100 * 14 + 40, torch.int32), Buf(100 * 14 + 40, cuda=False)):
        with pytest.raises(ValueError):
            _trace_ctas(bad, 100, TRACE_STEP_STAMPS)
