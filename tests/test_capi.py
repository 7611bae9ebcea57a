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


def test_impurity_arguments_rejected_before_device_use():
    L = capi.lib()
    V = ctypes.c_void_p(1)  # never dereferenced: every case below returns before a CUDA call
    imp = ctypes.c_void_p(1)
    add = L.itp2d_add_gaussian_impurities
    assert add(0, 16, 0.1, 1, imp, V, None) == capi.E_INVALID       # empty grid
    assert add(16, 16, 0.0, 1, imp, V, None) == capi.E_INVALID      # dx <= 0
    assert add(16, 16, 0.1, -1, imp, V, None) == capi.E_INVALID     # negative count
    assert add(16, 16, 0.1, 1, None, V, None) == capi.E_INVALID     # no impurity list
    assert add(16, 16, 0.1, 1, imp, None, None) == capi.E_INVALID   # no potential
    assert add(16, 16, 0.1, 0, None, V, None) == capi.OK            # nothing to add
