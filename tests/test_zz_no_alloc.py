"""The allocation-free eigensolver entry point, for callers that cannot
allocate device memory (their memory manager owns the device, or they cannot
afford cudaMalloc's synchronisation). It must give the same results as the
allocating entry point itp2d_hermitian_eigensolve, call after call, even
though every call reuses one fixed device array.

This file is collected last on purpose: it runs after every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 128  # ITP2D_NOALLOC_MAX_N in include/itp2d_gpu.h


@pytest.fixture(scope="module")
def L():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from itp2d_b200 import capi
    lib = capi.lib()
    dp = C.POINTER(C.c_double)
    lib.itp2d_hermitian_eigensolve_noalloc.argtypes = [C.c_int, dp, dp, dp]
    lib.itp2d_hermitian_eigensolve_noalloc.restype = C.c_int
    return lib


def _noalloc(L, M):
    """Calls the C ABI entry point directly (column-major input, upper triangle)."""
    n = M.shape[0]
    a = np.ascontiguousarray(np.asarray(M, dtype=np.complex128).T)
    ev = np.empty(n)
    vec = np.empty((n, n), dtype=np.complex128)
    st = L.itp2d_hermitian_eigensolve_noalloc(n, a.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                                              ev.ctypes.data_as(C.POINTER(C.c_double)),
                                              vec.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)))
    return st, ev, vec.T.copy()


def _hermitian(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return X @ X.conj().T / n + np.eye(n)


def test_noalloc_matches_allocating_entry_point(L):
    from itp2d_b200 import capi
    # two calls in a row, the second smaller than the first, so leftovers of
    # the first call sit in the shared array when the second one runs
    for n, seed in [(MAX_N, 1), (37, 2)]:
        M = _hermitian(n, seed)
        st, ev, U = _noalloc(L, M)
        assert st == capi.OK
        ev_ref, U_ref = capi.hermitian_eigensolve(M)
        scale = np.max(np.abs(ev_ref))
        assert np.max(np.abs(ev - ev_ref)) < 1e-13 * scale
        # eigenvectors agree up to a phase (the eigenvalues here are distinct)
        overlap = np.abs(np.sum(np.conj(U_ref) * U, axis=0))
        assert np.max(np.abs(overlap - 1)) < 1e-12
        assert np.max(np.abs(U.conj().T @ U - np.eye(n))) < 2e-14
        assert np.max(np.abs(M @ U - U * ev[None, :])) < 1e-12 * scale


def test_noalloc_rejects_sizes_beyond_the_maximum(L):
    from itp2d_b200 import capi
    st, _, _ = _noalloc(L, np.eye(MAX_N + 1, dtype=complex))
    assert st == capi.E_INVALID
