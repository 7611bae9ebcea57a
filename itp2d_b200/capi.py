"""ctypes binding of the C ABI in include/itp2d_gpu.h (libitp2d_b200.so).

This is a thin host-side mirror used by the tests and the benchmark; the
native C++ host layer (itp2d_b200/host) sits on the same ABI. Every call
raises ``ITP2DError`` on a non-zero status; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libitp2d_b200.so")
HEADER = os.path.join(ROOT, "include", "itp2d_gpu.h")

OK = 0
E_INVALID, E_CUDA, E_OOM = 1, 2, 3
E_NONPOSITIVE_EIGENVALUE, E_NONNORMAL_EIGENVALUE, E_EIGENSOLVER = 4, 5, 6
E_TIMEOUT, E_UNSUPPORTED = 7, 8
PERIODIC, DIRICHLET = 0, 1
FP64, FP32 = 0, 1
ORTHO_DEFAULT, ORTHO_HIGHMEM, ORTHO_CHOLESKY = 0, 1, 2
BETWEEN_LOWDIN, BETWEEN_CHOLESKY = 0, 1
COL_SMEM, COL_TMA = 0, 1
CONTRACT_AUTO, CONTRACT_FP64, CONTRACT_TC_STAGED = 0, 1, 2
FP64_DMMA, FP64_INT8 = 0, 1
TRANSFORMS = ["FFT", "iFFT", "FFTx", "iFFTx", "FFTy", "iFFTy", "DST", "iDST", "DSTx", "iDSTx",
              "DSTy", "iDSTy", "DCT", "iDCT", "DCTx", "iDCTx", "DCTy", "iDCTy"]

_lib = None


class ITP2DError(RuntimeError):
    def __init__(self, status: int, what: str, bad_index: int = -1, bad_value: float = 0.0):
        msg = lib().itp2d_status_string(status).decode() if _lib is not None else str(status)
        super().__init__(f"{what}: {msg} (status {status})")
        self.status, self.bad_index, self.bad_value = status, bad_index, bad_value


def header_symbols() -> list:
    """Function names declared in include/itp2d_gpu.h."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*\**\s+\**(itp2d_[a-z0-9_]+)\s*\(",
                                 txt, flags=re.M)))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ITP2DError(E_INVALID, f"{LIB_PATH} missing; build it with python -m itp2d_b200.build")
        L = C.CDLL(LIB_PATH)
        vp, i, d, dp, ip = C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.itp2d_ctx_create.argtypes = [i, i, d, i, i, d, i, i, vp, C.POINTER(vp)]
        L.itp2d_ctx_destroy.argtypes = [vp]
        L.itp2d_set_potential.argtypes = [vp, dp]
        L.itp2d_set_time_step.argtypes = [vp, d]
        L.itp2d_upload_states.argtypes = [vp, dp]
        L.itp2d_download_states.argtypes = [vp, dp]
        L.itp2d_device_states.argtypes = [vp, C.POINTER(vp)]
        L.itp2d_propagate.argtypes = [vp]
        L.itp2d_orthonormalize.argtypes = [vp, i, ip, dp]
        L.itp2d_energies.argtypes = [vp, dp, dp, dp, dp]
        L.itp2d_apply_hamiltonian.argtypes = [vp]
        L.itp2d_transform.argtypes = [vp, i]
        L.itp2d_synchronize.argtypes = [vp]
        L.itp2d_set_contraction.argtypes = [vp, i]
        L.itp2d_set_precision.argtypes = [vp, i]
        L.itp2d_set_fp32_orthonormalization.argtypes = [vp, i]
        L.itp2d_orthonormalization_counts.argtypes = [vp] + [C.POINTER(C.c_longlong)] * 3
        L.itp2d_set_fp32_between.argtypes = [vp, i]
        L.itp2d_set_fp32_eig_sweeps.argtypes = [vp, i]
        L.itp2d_set_fp64_engine.argtypes = [vp, i]
        L.itp2d_int8_contractions.argtypes = [vp]
        L.itp2d_int8_contractions.restype = C.c_longlong
        L.itp2d_fp32_capped_eigensolves.argtypes = [vp]
        L.itp2d_fp32_capped_eigensolves.restype = C.c_longlong
        L.itp2d_rayleigh_ritz.argtypes = [vp, dp]
        L.itp2d_set_column_variant.argtypes = [vp, i]
        L.itp2d_triangular_rotations.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        L.itp2d_column_variant.argtypes = [vp]
        L.itp2d_overlap_matrix.argtypes = [vp, dp]
        L.itp2d_launch_count.argtypes = [vp]
        L.itp2d_launch_count.restype = C.c_longlong
        L.itp2d_set_timing.argtypes = [vp, i]
        L.itp2d_phase_times.argtypes = [vp, dp]
        L.itp2d_phase_stats.argtypes = [vp, dp, C.POINTER(C.c_longlong)]
        L.itp2d_last_sweeps.argtypes = [vp]
        L.itp2d_total_sweeps.argtypes = [vp]
        L.itp2d_total_sweeps.restype = C.c_longlong
        L.itp2d_precision_sweeps.argtypes = [vp, i]
        L.itp2d_precision_sweeps.restype = C.c_longlong
        L.itp2d_device_fp32_peak.argtypes = [dp]
        L.itp2d_hermitian_eigensolve.argtypes = [i, dp, dp, dp]
        L.itp2d_device_fp64_peak.argtypes = [dp]
        L.itp2d_add_gaussian_impurities.argtypes = [i, i, C.c_double, i, vp, vp, vp]
        L.itp2d_status_string.argtypes = [i]
        L.itp2d_status_string.restype = C.c_char_p
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _check(st, what):
    if st != OK:
        raise ITP2DError(st, what)


def device_fp32_peak() -> float:
    """Measured FP32 FFMA TFLOP/s of the current device."""
    t = C.c_double(0.0)
    _check(lib().itp2d_device_fp32_peak(C.byref(t)), "itp2d_device_fp32_peak")
    return t.value


def add_gaussian_impurities(sx: int, sy: int, dx: float, impurities_ptr: int, n: int, V_ptr: int,
                            stream: int = 0) -> None:
    """V += Gaussian impurities on the device (itp2d_add_gaussian_impurities);
    impurities_ptr points to n rows (x, y, A, w) and V_ptr to sx * sy doubles,
    both device memory (for example torch tensors' data_ptr())."""
    _check(lib().itp2d_add_gaussian_impurities(sx, sy, dx, n, C.c_void_p(impurities_ptr), C.c_void_p(V_ptr),
                                               C.c_void_p(stream) if stream else None),
           "itp2d_add_gaussian_impurities")


def device_fp64_peak() -> float:
    """Measured FP64 DMMA TFLOP/s of the current device."""
    t = C.c_double(0.0)
    _check(lib().itp2d_device_fp64_peak(C.byref(t)), "itp2d_device_fp64_peak")
    return t.value


def hermitian_eigensolve(A: np.ndarray):
    """Eigenvalues (ascending) and eigenvectors (columns) of a Hermitian
    matrix through itp2d_hermitian_eigensolve; reads the upper triangle."""
    n = A.shape[0]
    a = np.ascontiguousarray(np.asarray(A, dtype=np.complex128).T)  # column-major
    ev = np.empty(n)
    vec = np.empty((n, n), dtype=np.complex128)
    _check(lib().itp2d_hermitian_eigensolve(n, _dp(a.view(np.float64)), _dp(ev), _dp(vec.view(np.float64))),
           "itp2d_hermitian_eigensolve")
    return ev, vec.T.copy()


PHASES = ["propagate", "overlap", "eigensolve", "rotation", "energies"]


def triangular_rotations(handle) -> dict:
    """Rotations by an upper-triangular W per precision, {"fp64": n, "fp32": n}."""
    a, b = C.c_longlong(0), C.c_longlong(0)
    _check(lib().itp2d_triangular_rotations(handle, C.byref(a), C.byref(b)), "itp2d_triangular_rotations")
    return {"fp64": a.value, "fp32": b.value}


def phase_stats(handle) -> dict:
    """Phase device times and call counts of a context handle, by precision."""
    ms = np.zeros(10)
    calls = np.zeros(10, dtype=np.int64)
    _check(lib().itp2d_phase_stats(handle, _dp(ms), calls.ctypes.data_as(C.POINTER(C.c_longlong))),
           "itp2d_phase_stats")
    return {prec: {ph: (float(ms[p * 5 + i]), int(calls[p * 5 + i])) for i, ph in enumerate(PHASES)}
            for p, prec in enumerate(["fp64", "fp32"])}


class Context:
    """One device-resident state set (the three seams of ITPSystem::step)."""

    def __init__(self, sx, sy, dx, num_states, boundary=PERIODIC, B=0.0, halforder=1, precision=FP64,
                 stream=None):
        self.sx, self.sy, self.dx, self.k = sx, sy, float(dx), num_states
        self.precision = precision
        h = C.c_void_p()
        st = lib().itp2d_ctx_create(sx, sy, float(dx), num_states, boundary, float(B), halforder, precision,
                                    C.c_void_p(stream) if stream else None, C.byref(h))
        _check(st, "itp2d_ctx_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().itp2d_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_potential(self, V):
        if V is None:
            _check(lib().itp2d_set_potential(self.h, None), "itp2d_set_potential")
            return
        a = np.ascontiguousarray(V, dtype=np.float64).reshape(-1)
        assert a.size == self.sx * self.sy
        _check(lib().itp2d_set_potential(self.h, _dp(a)), "itp2d_set_potential")

    def set_time_step(self, eps):
        _check(lib().itp2d_set_time_step(self.h, float(eps)), "itp2d_set_time_step")

    def upload(self, psi):
        a = np.ascontiguousarray(psi, dtype=np.complex128)
        assert a.shape == (self.k, self.sy, self.sx), a.shape
        _check(lib().itp2d_upload_states(self.h, _dp(a.view(np.float64))), "itp2d_upload_states")

    def download(self):
        out = np.empty((self.k, self.sy, self.sx), dtype=np.complex128)
        _check(lib().itp2d_download_states(self.h, _dp(out.view(np.float64))), "itp2d_download_states")
        return out

    def device_states(self) -> int:
        p = C.c_void_p()
        _check(lib().itp2d_device_states(self.h, C.byref(p)), "itp2d_device_states")
        return p.value

    def propagate(self):
        _check(lib().itp2d_propagate(self.h), "itp2d_propagate")

    def orthonormalize(self, algo=ORTHO_DEFAULT):
        bi, bv = C.c_int(-1), C.c_double(0.0)
        st = lib().itp2d_orthonormalize(self.h, algo, C.byref(bi), C.byref(bv))
        if st != OK:
            raise ITP2DError(st, "itp2d_orthonormalize", bi.value, bv.value)

    def set_fp32_orthonormalization(self, canonical_every):
        _check(lib().itp2d_set_fp32_orthonormalization(self.h, int(canonical_every)),
               "itp2d_set_fp32_orthonormalization")

    def set_column_variant(self, variant):
        """Column pass of 256/512-point lines: COL_SMEM, COL_TMA, or -1 (tuned)."""
        _check(lib().itp2d_set_column_variant(self.h, int(variant)), "itp2d_set_column_variant")

    @property
    def column_variant(self) -> int:
        return lib().itp2d_column_variant(self.h)

    def rayleigh_ritz(self):
        """One Rayleigh-Ritz step on the (orthonormal) resident states; returns
        the ascending Ritz values."""
        theta = np.empty(self.k)
        _check(lib().itp2d_rayleigh_ritz(self.h, theta.ctypes.data_as(C.POINTER(C.c_double))),
               "itp2d_rayleigh_ritz")
        return theta

    def set_fp32_between(self, method):
        """BETWEEN_LOWDIN or BETWEEN_CHOLESKY between the canonical calls."""
        _check(lib().itp2d_set_fp32_between(self.h, int(method)), "itp2d_set_fp32_between")

    def set_fp32_eig_sweeps(self, max_sweeps):
        """FP32 canonical steps: at most max_sweeps Jacobi sweeps, finished by a
        Cholesky step (0: full eigensolve)."""
        _check(lib().itp2d_set_fp32_eig_sweeps(self.h, int(max_sweeps)), "itp2d_set_fp32_eig_sweeps")

    def set_fp64_engine(self, engine):
        """FP64_DMMA (default) or FP64_INT8 for the rotation of FP64 states."""
        _check(lib().itp2d_set_fp64_engine(self.h, int(engine)), "itp2d_set_fp64_engine")

    def int8_contractions(self) -> int:
        """Rotations of FP64 states run on the int8 tensor cores since creation."""
        return lib().itp2d_int8_contractions(self.h)

    def capped_eigensolves(self) -> int:
        """Canonical FP32 steps finished by the Cholesky step since creation."""
        return lib().itp2d_fp32_capped_eigensolves(self.h)

    def orthonormalization_counts(self):
        """(canonical, Lowdin, Cholesky) orthonormalisations since creation."""
        a, b, c = C.c_longlong(0), C.c_longlong(0), C.c_longlong(0)
        _check(lib().itp2d_orthonormalization_counts(self.h, C.byref(a), C.byref(b), C.byref(c)),
               "itp2d_orthonormalization_counts")
        return a.value, b.value, c.value

    def set_precision(self, precision):
        _check(lib().itp2d_set_precision(self.h, precision), "itp2d_set_precision")
        self.precision = precision

    def set_contraction(self, engine=CONTRACT_AUTO):
        _check(lib().itp2d_set_contraction(self.h, engine), "itp2d_set_contraction")

    def overlap_matrix(self):
        S = np.empty((self.k, self.k), dtype=np.complex128)
        _check(lib().itp2d_overlap_matrix(self.h, _dp(S.view(np.float64))), "itp2d_overlap_matrix")
        return S

    def energies(self):
        E, s, r, ei = (np.empty(self.k) for _ in range(4))
        _check(lib().itp2d_energies(self.h, _dp(E), _dp(s), _dp(r), _dp(ei)), "itp2d_energies")
        return E, s, r, ei

    def apply_hamiltonian(self):
        _check(lib().itp2d_apply_hamiltonian(self.h), "itp2d_apply_hamiltonian")

    def transform(self, kind):
        if isinstance(kind, str):
            kind = TRANSFORMS.index(kind)
        _check(lib().itp2d_transform(self.h, kind), "itp2d_transform")

    def synchronize(self):
        _check(lib().itp2d_synchronize(self.h), "itp2d_synchronize")

    @property
    def launches(self) -> int:
        return lib().itp2d_launch_count(self.h)

    def set_timing(self, on=True):
        _check(lib().itp2d_set_timing(self.h, int(on)), "itp2d_set_timing")

    def phase_times(self) -> dict:
        t = np.zeros(5)
        _check(lib().itp2d_phase_times(self.h, _dp(t)), "itp2d_phase_times")
        return dict(zip(["propagate", "overlap", "eigensolve", "rotation", "energies"], t.tolist()))

    def phase_stats(self) -> dict:
        """{precision: {phase: (ms, calls)}} with precision "fp64" / "fp32"."""
        return phase_stats(self.h)

    @property
    def last_sweeps(self) -> int:
        return lib().itp2d_last_sweeps(self.h)
