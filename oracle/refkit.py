"""ctypes access to the itp2d reference compiled into oracle/_ref/libitp2d_ref.so.
TEST INFRASTRUCTURE ONLY (the checker and the reference CPU baseline).

The library is built by ``make -C oracle`` from the unmodified reference
sources plus the oracle shims; see oracle/Makefile and oracle/ref_harness.cpp.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libitp2d_ref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        # The bundled OpenBLAS is a pthreads build; the reference calls it from
        # inside OpenMP loops, so keep BLAS single-threaded (must be set before
        # the library initialises) and let the reference's OpenMP loops use
        # the cores.
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} not built (run: make -C oracle)")
        L = C.CDLL(LIB_PATH)
        vp, d, i, dp = C.c_void_p, C.c_double, C.c_int, C.POINTER(C.c_double)
        L.refkit_create.restype = vp
        L.refkit_create.argtypes = [i, i, d, i, d, i, d, i, i, C.c_char_p, dp, i]
        for name in ["refkit_destroy", "refkit_propagate", "refkit_apply_hamiltonian"]:
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = None
        for name in ["refkit_get_potential", "refkit_set_states", "refkit_get_states"]:
            getattr(L, name).argtypes = [vp, dp]
            getattr(L, name).restype = None
        L.refkit_kvalues.argtypes = [vp, dp, dp, dp, dp]
        L.refkit_init_gaussian.argtypes = [vp, C.c_ulong]
        L.refkit_set_time_step.argtypes = [vp, d]
        L.refkit_orthonormalize.argtypes = [vp]
        L.refkit_orthonormalize.restype = i
        L.refkit_how_orthonormal.argtypes = [vp]
        L.refkit_how_orthonormal.restype = d
        L.refkit_energies.argtypes = [vp, dp, dp, dp]
        L.refkit_transform.argtypes = [vp, i]
        L.refkit_ortho_times.argtypes = [vp, dp]
        L.refkit_ortho_times.restype = None
        L.refkit_normalization_factor.argtypes = [vp, i]
        L.refkit_normalization_factor.restype = d
        L.refsys_create.restype = vp
        L.refsys_create.argtypes = [C.POINTER(RefSysParams), dp, dp]
        for name in ["refsys_destroy", "refsys_step"]:
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = None
        for name in ["refsys_is_finished", "refsys_error_flag", "refsys_total_steps",
                     "refsys_num_finally_converged"]:
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = i
        L.refsys_eps.argtypes = [vp]
        L.refsys_eps.restype = d
        L.refsys_last_energies.argtypes = [vp, dp, dp]
        L.refsys_last_energies.restype = i
        L.refsys_get_states.argtypes = [vp, dp]
        L.refsys_times.argtypes = [vp, dp]
        L.ref_add_gaussian_impurities.argtypes = [i, i, d, i, dp, dp]
        L.ref_add_gaussian_impurities.restype = None
        L.ref_add_impurities.argtypes = [i, i, i, d, i, dp, d, d, dp]
        L.ref_add_impurities.restype = None
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def add_gaussian_impurities(sx: int, sy: int, dx: float, impurities: np.ndarray, V: np.ndarray) -> np.ndarray:
    """V plus the impurities (rows x, y, A, w) through the reference's
    GaussianImpurities::add_noise (noise.cpp:24-40); returns a new [sy][sx] array."""
    imp = np.ascontiguousarray(impurities, dtype=np.float64).reshape(-1, 4)
    out = np.ascontiguousarray(V, dtype=np.float64).copy()
    assert out.shape == (sy, sx)
    lib().ref_add_gaussian_impurities(sx, sy, dx, imp.shape[0], _dp(imp), _dp(out))
    return out


def add_impurities(shape: int, sx: int, sy: int, dx: float, rows: np.ndarray, p0: float, p1: float,
                   V: np.ndarray) -> np.ndarray:
    """V plus n impurities of one shape (1 Coulomb, 2 hemisphere, 3 delta)
    through the reference's add_noise (noise.cpp:42-87); returns a new array."""
    width = 3 if shape == 3 else 2
    r = np.ascontiguousarray(rows, dtype=np.float64).reshape(-1, width)
    out = np.ascontiguousarray(V, dtype=np.float64).copy()
    lib().ref_add_impurities(shape, sx, sy, dx, r.shape[0], _dp(r), float(p0), float(p1), _dp(out))
    return out


class RefSysParams(C.Structure):
    _fields_ = [
        ("sx", C.c_int), ("sy", C.c_int), ("len", C.c_double), ("boundary", C.c_int),
        ("B", C.c_double), ("halforder", C.c_int), ("num_states", C.c_int), ("wanted", C.c_int),
        ("ignore_lowest", C.c_int), ("num_eps", C.c_int), ("eps", C.c_double * 8),
        ("eps_divisor", C.c_double), ("max_steps", C.c_int), ("min_eps", C.c_double),
        ("seed", C.c_ulong), ("ortho_highmem", C.c_int), ("threads", C.c_int), ("recover", C.c_int),
        ("potential", C.c_char * 128), ("timestep_test", C.c_char * 128), ("final_test", C.c_char * 128),
    ]


class RefKit:
    """The reference operators for one grid, applied seam by seam."""

    def __init__(self, sx, sy, length, boundary, B, halforder, eps, num_states,
                 potential="harmonic(1)", extra_potential=None, highmem=False, threads=1):
        self.sx, self.sy, self.k = sx, sy, num_states
        self._extra = None
        ep = None
        if extra_potential is not None:
            self._extra = np.ascontiguousarray(extra_potential, dtype=np.float64).reshape(-1)
            ep = _dp(self._extra)
        self.h = lib().refkit_create(sx, sy, float(length), int(boundary), float(B), int(halforder),
                                     float(eps), int(num_states), int(highmem), potential.encode(), ep,
                                     int(threads))

    def close(self):
        if self.h:
            lib().refkit_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def potential(self) -> np.ndarray:
        out = np.empty((self.sy, self.sx))
        lib().refkit_get_potential(self.h, _dp(out))
        return out

    def kvalues(self):
        fkx, dkx = np.empty(self.sx), np.empty(self.sx)
        fky, dky = np.empty(self.sy), np.empty(self.sy)
        lib().refkit_kvalues(self.h, _dp(fkx), _dp(fky), _dp(dkx), _dp(dky))
        return fkx, fky, dkx, dky

    def set_states(self, psi: np.ndarray) -> None:
        a = np.ascontiguousarray(psi, dtype=np.complex128)
        assert a.shape == (self.k, self.sy, self.sx)
        lib().refkit_set_states(self.h, _dp(a.view(np.float64)))

    def states(self) -> np.ndarray:
        out = np.empty((self.k, self.sy, self.sx), dtype=np.complex128)
        lib().refkit_get_states(self.h, _dp(out.view(np.float64)))
        return out

    def init_gaussian(self, seed: int) -> None:
        lib().refkit_init_gaussian(self.h, seed)

    def set_time_step(self, eps: float) -> None:
        lib().refkit_set_time_step(self.h, float(eps))

    def propagate(self) -> None:
        lib().refkit_propagate(self.h)

    def orthonormalize(self) -> int:
        return lib().refkit_orthonormalize(self.h)

    def ortho_times(self) -> dict:
        """Accumulated seconds of this kit's orthonormalisations, by phase
        (StateSet timers, stateset.hpp:77-80)."""
        t = np.empty(4)
        lib().refkit_ortho_times(self.h, _dp(t))
        return dict(zip(["dot", "eigensolve", "lincomb", "total"], t.tolist()))

    def how_orthonormal(self) -> float:
        return lib().refkit_how_orthonormal(self.h)

    def energies(self):
        E, s, Ei = np.empty(self.k), np.empty(self.k), np.empty(self.k)
        lib().refkit_energies(self.h, _dp(E), _dp(s), _dp(Ei))
        return E, s, Ei

    def apply_hamiltonian(self) -> None:
        lib().refkit_apply_hamiltonian(self.h)

    def transform(self, kind: int) -> None:
        lib().refkit_transform(self.h, int(kind))

    def normalization_factor(self, kind: int) -> float:
        return lib().refkit_normalization_factor(self.h, int(kind))


class RefSystem:
    """The reference ITPSystem driven through its step() loop."""

    def __init__(self, sx, sy, length, boundary, B, halforder, num_states, wanted, eps_values,
                 eps_divisor=2.0, timestep_test="abschange(1e-10)", final_test="absstdev(1e-8)",
                 potential="harmonic(1)", extra_potential=None, init_states=None, max_steps=100000,
                 min_eps=1e-9, seed=12345, highmem=True, threads=None, ignore_lowest=0, recover=False):
        p = RefSysParams()
        p.sx, p.sy, p.len, p.boundary, p.B = sx, sy, float(length), int(boundary), float(B)
        p.halforder, p.num_states, p.wanted, p.ignore_lowest = halforder, num_states, wanted, ignore_lowest
        p.num_eps = len(eps_values)
        for i, e in enumerate(eps_values[:8]):
            p.eps[i] = e
        p.eps_divisor, p.max_steps, p.min_eps, p.seed = eps_divisor, max_steps, min_eps, seed
        p.ortho_highmem, p.recover = int(highmem), int(recover)
        p.threads = threads if threads else (os.cpu_count() or 1)
        p.potential, p.timestep_test, p.final_test = potential.encode(), timestep_test.encode(), final_test.encode()
        self.p = p
        self.k, self.sx, self.sy = num_states, sx, sy
        ep = ip = None
        self._keep = []
        if extra_potential is not None:
            a = np.ascontiguousarray(extra_potential, dtype=np.float64).reshape(-1)
            self._keep.append(a)
            ep = _dp(a)
        if init_states is not None:
            b = np.ascontiguousarray(init_states, dtype=np.complex128)
            self._keep.append(b)
            ip = _dp(b.view(np.float64))
        self.h = lib().refsys_create(C.byref(p), ep, ip)

    def close(self):
        if self.h:
            lib().refsys_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self):
        lib().refsys_step(self.h)

    @property
    def finished(self) -> bool:
        return bool(lib().refsys_is_finished(self.h))

    @property
    def error_flag(self) -> bool:
        return bool(lib().refsys_error_flag(self.h))

    @property
    def total_steps(self) -> int:
        return lib().refsys_total_steps(self.h)

    @property
    def eps(self) -> float:
        return lib().refsys_eps(self.h)

    @property
    def num_converged(self) -> int:
        return lib().refsys_num_finally_converged(self.h)

    def energies(self):
        E, s = np.empty(self.k), np.empty(self.k)
        n = lib().refsys_last_energies(self.h, _dp(E), _dp(s))
        return E[:n], s[:n]

    def states(self) -> np.ndarray:
        out = np.empty((self.k, self.sy, self.sx), dtype=np.complex128)
        lib().refsys_get_states(self.h, _dp(out.view(np.float64)))
        return out

    def times(self) -> dict:
        t = np.empty(7)
        lib().refsys_times(self.h, _dp(t))
        keys = ["total", "propagation", "orthonormalization", "dot", "eigensolve", "lincomb", "convtest"]
        return dict(zip(keys, t.tolist()))
