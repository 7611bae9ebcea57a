"""CPU-side checks of the C ABI library: it loads, and it exports every
entry point declared in include/itp2d_gpu.h. No device calls."""
import ctypes

from itp2d_b200 import capi


def test_library_exports_header_symbols():
    L = capi.lib()
    names = capi.header_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings():
    L = capi.lib()
    for code in range(9):
        s = L.itp2d_status_string(code)
        assert s and s != b"unknown status"
    assert L.itp2d_status_string(99) == b"unknown status"


def test_invalid_arguments_rejected_before_device_use():
    L = capi.lib()
    out = ctypes.c_void_p()
    # sizes and enums are validated before any CUDA call
    assert L.itp2d_ctx_create(1, 16, 0.1, 4, 0, 0.0, 1, 0, None, ctypes.byref(out)) == capi.E_INVALID
    assert L.itp2d_ctx_create(16, 16, 0.1, 4, 7, 0.0, 1, 0, None, ctypes.byref(out)) == capi.E_INVALID
    assert L.itp2d_ctx_create(22, 16, 0.1, 4, 0, 0.0, 1, 0, None, ctypes.byref(out)) == capi.E_UNSUPPORTED
    assert L.itp2d_ctx_create(8192, 16, 0.1, 4, 1, 1.0, 1, 0, None, ctypes.byref(out)) == capi.E_UNSUPPORTED
    assert L.itp2d_propagate(None) == capi.E_INVALID
