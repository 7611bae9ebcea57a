"""ctypes binding of the native ITP driver (include/itp2d_host.h).

``ITPSystem(Parameters(...))`` mirrors the reference ITPSystem
(itpsystem.hpp:55-156): ``step()`` until ``finished``, then the sorted
energies. All work runs in libitp2d_b200.so; there is no Python fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import capi


class _Params(C.Structure):
    _fields_ = [
        ("sx", C.c_int), ("sy", C.c_int), ("length", C.c_double), ("boundary", C.c_int), ("B", C.c_double),
        ("halforder", C.c_int), ("num_states", C.c_int), ("wanted", C.c_int), ("ignore_lowest", C.c_int),
        ("num_eps", C.c_int), ("eps", C.c_double * 16), ("eps_divisor", C.c_double), ("exhaust_eps", C.c_int),
        ("max_steps", C.c_int), ("min_eps", C.c_double), ("seed", C.c_ulong), ("ortho_algorithm", C.c_int),
        ("recover", C.c_int), ("precision", C.c_int), ("fp32_switch", C.c_double),
        ("potential", C.c_char * 128), ("timestep_test", C.c_char * 128), ("final_test", C.c_char * 128),
        ("fp32_canonical_every", C.c_int), ("fp32_between", C.c_int), ("switch_rayleigh_ritz", C.c_int),
        ("fp32_switch_span", C.c_int), ("fp32_eig_sweeps", C.c_int),
        ("fp32_canonical_delay", C.c_int), ("fp64_engine", C.c_int),
    ]


_bound = False


def _lib():
    global _bound
    L = capi.lib()
    if not _bound:
        vp, i, d, dp, ip = C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.itp2d_parameters_default.argtypes = [C.POINTER(_Params)]
        L.itp2d_system_create.argtypes = [C.POINTER(_Params), dp, dp, vp, C.POINTER(vp)]
        for n in ["itp2d_system_destroy", "itp2d_system_step"]:
            getattr(L, n).argtypes = [vp]
        L.itp2d_system_run.argtypes = [vp, i]
        L.itp2d_system_run_device.argtypes = [vp, i]
        L.itp2d_system_device_iterations.argtypes = [vp]
        L.itp2d_system_reset.argtypes = [vp, dp]
        for n in ["itp2d_system_is_finished", "itp2d_system_error_flag", "itp2d_system_total_steps",
                  "itp2d_system_num_converged", "itp2d_system_in_fp32"]:
            getattr(L, n).argtypes = [vp]
            getattr(L, n).restype = i
        L.itp2d_system_eps.argtypes = [vp]
        L.itp2d_system_eps.restype = d
        L.itp2d_system_energies.argtypes = [vp, dp, dp, dp, ip]
        L.itp2d_system_energy_history.argtypes = [vp, i, dp]
        L.itp2d_system_download_states.argtypes = [vp, dp]
        L.itp2d_system_times.argtypes = [vp, dp]
        L.itp2d_system_last_error.argtypes = [vp]
        L.itp2d_system_last_error.restype = C.c_char_p
        L.itp2d_system_context.argtypes = [vp]
        L.itp2d_system_context.restype = vp
        L.itp2d_install_signal_handlers.argtypes = []
        L.itp2d_abort_flag.restype = ip
        L.itp2d_save_flag.restype = ip
        L.itp2d_system_set_flags.argtypes = [vp, ip, ip]
        L.itp2d_system_set_save_callback.argtypes = [vp, _SaveFn, vp]
        L.itp2d_system_saves.argtypes = [vp]
        _bound = True
    return L


# void (*)(void* user, const double* states, const int* order, int k, int sx, int sy, int step);
# sig_atomic_t is an int on the platforms this library builds for
_SaveFn = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_int, C.c_int, C.c_int,
                      C.c_int)


def install_signal_handlers() -> None:
    """SIGINT raises the library's abort flag (a second SIGINT exits with
    status 1), SIGUSR1 its save flag, as the reference's program does
    (itp2d.cpp:40-66). Replaces Python's own SIGINT handler."""
    st = _lib().itp2d_install_signal_handlers()
    if st != capi.OK:
        raise capi.ITP2DError(st, "itp2d_install_signal_handlers")


def abort_flag():
    """The library's process-wide abort flag (a ctypes int pointer)."""
    return _lib().itp2d_abort_flag()


def save_flag():
    """The library's process-wide save flag (a ctypes int pointer)."""
    return _lib().itp2d_save_flag()


@dataclass
class Parameters:
    """Mirror of the reference Parameters (parameters.hpp:37-211), with the
    reference defaults (parameters.cpp:25-55)."""
    sx: int = 64
    sy: int = 64
    length: float = 12.0
    boundary: int = capi.PERIODIC
    B: float = 0.0
    halforder: int = 5
    num_states: int = 25
    wanted: int = 16
    ignore_lowest: int = 0
    eps: list = field(default_factory=list)
    eps_divisor: float = 5.0
    exhaust_eps: bool = False
    max_steps: int = 50
    min_eps: float = 1e-9
    seed: int = 0x20120131
    ortho_algorithm: int = capi.ORTHO_DEFAULT
    recover: bool = False
    precision: int = capi.FP64
    fp32_switch: float = 0.0
    fp32_canonical_every: int = 0
    fp32_between: int = capi.BETWEEN_LOWDIN
    switch_rayleigh_ritz: bool = False
    fp32_switch_span: int = 0
    fp32_eig_sweeps: int = 0
    fp32_canonical_delay: int = 0
    fp64_engine: int = capi.FP64_DMMA
    potential: str = "harmonic"
    timestep_test: str = "relstdev(1e-3,1e-4)"
    final_test: str = "relstdev(1e-3,0)"

    def _raw(self) -> _Params:
        p = _Params()
        _lib().itp2d_parameters_default(C.byref(p))
        for k in ["sx", "sy", "length", "boundary", "B", "halforder", "num_states", "wanted", "ignore_lowest",
                  "eps_divisor", "max_steps", "min_eps", "seed", "ortho_algorithm", "precision", "fp32_switch",
                  "fp32_canonical_every", "fp32_between", "fp32_switch_span", "fp32_eig_sweeps", "fp32_canonical_delay", "fp64_engine"]:
            setattr(p, k, getattr(self, k))
        p.exhaust_eps, p.recover = int(self.exhaust_eps), int(self.recover)
        p.switch_rayleigh_ritz = int(self.switch_rayleigh_ritz)
        if len(self.eps) > 16:
            raise ValueError("at most 16 explicit time steps")
        p.num_eps = len(self.eps)
        for i, e in enumerate(self.eps):
            p.eps[i] = e
        p.potential, p.timestep_test, p.final_test = (self.potential.encode(), self.timestep_test.encode(),
                                                      self.final_test.encode())
        return p


class ITPSystem:
    def __init__(self, params: Parameters, extra_potential=None, init_states=None, stream=None):
        self.params = params
        self.k = params.num_states
        self._raw = params._raw()
        G = params.sx * params.sy
        ep = ip = None
        self._keep = []
        if extra_potential is not None:
            a = np.ascontiguousarray(extra_potential, dtype=np.float64).reshape(-1)
            assert a.size == G
            self._keep.append(a)
            ep = a.ctypes.data_as(C.POINTER(C.c_double))
        if init_states is not None:
            b = np.ascontiguousarray(init_states, dtype=np.complex128)
            assert b.shape == (self.k, params.sy, params.sx)
            self._keep.append(b)
            ip = b.view(np.float64).ctypes.data_as(C.POINTER(C.c_double))
        h = C.c_void_p()
        st = _lib().itp2d_system_create(C.byref(self._raw), ep, ip, C.c_void_p(stream) if stream else None,
                                        C.byref(h))
        if st != capi.OK:
            raise capi.ITP2DError(st, "itp2d_system_create")
        self.h = h
        self._keep = []

    def close(self):
        if getattr(self, "h", None):
            _lib().itp2d_system_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self, init_states=None):
        """Restart from new initial states (None: fresh noise), reusing device memory."""
        ip = None
        if init_states is not None:
            b = np.ascontiguousarray(init_states, dtype=np.complex128)
            assert b.shape == (self.k, self.params.sy, self.params.sx)
            ip = b.view(np.float64).ctypes.data_as(C.POINTER(C.c_double))
        st = _lib().itp2d_system_reset(self.h, ip)
        if st != capi.OK:
            raise capi.ITP2DError(st, "itp2d_system_reset: " + self.last_error)

    def step(self):
        st = _lib().itp2d_system_step(self.h)
        if st != capi.OK:
            raise capi.ITP2DError(st, "itp2d_system_step: " + self.last_error)

    def run(self, max_iterations=1 << 30):
        st = _lib().itp2d_system_run(self.h, int(max_iterations))
        if st != capi.OK:
            raise capi.ITP2DError(st, "itp2d_system_run: " + self.last_error)

    def run_device(self, max_phases=1 << 30):
        """Solve with the FP64 iterations on the device (itp2d_system_run_device)."""
        st = _lib().itp2d_system_run_device(self.h, int(max_phases))
        if st != capi.OK:
            raise capi.ITP2DError(st, "itp2d_system_run_device: " + self.last_error)

    @property
    def device_iterations(self) -> int:
        return _lib().itp2d_system_device_iterations(self.h)

    @property
    def finished(self) -> bool:
        return bool(_lib().itp2d_system_is_finished(self.h))

    @property
    def error_flag(self) -> bool:
        return bool(_lib().itp2d_system_error_flag(self.h))

    @property
    def total_steps(self) -> int:
        return _lib().itp2d_system_total_steps(self.h)

    @property
    def num_converged(self) -> int:
        return _lib().itp2d_system_num_converged(self.h)

    @property
    def eps(self) -> float:
        return _lib().itp2d_system_eps(self.h)

    @property
    def in_fp32(self) -> bool:
        return bool(_lib().itp2d_system_in_fp32(self.h))

    @property
    def last_error(self) -> str:
        return _lib().itp2d_system_last_error(self.h).decode()

    def energies(self):
        E, s, r = np.empty(self.k), np.empty(self.k), np.empty(self.k)
        idx = np.empty(self.k, dtype=np.int32)
        n = _lib().itp2d_system_energies(self.h, E.ctypes.data_as(C.POINTER(C.c_double)),
                                         s.ctypes.data_as(C.POINTER(C.c_double)),
                                         r.ctypes.data_as(C.POINTER(C.c_double)),
                                         idx.ctypes.data_as(C.POINTER(C.c_int)))
        return E[:n], s[:n], r[:n], idx[:n]

    def energy_history(self, step: int):
        E = np.empty(self.k)
        n = _lib().itp2d_system_energy_history(self.h, step, E.ctypes.data_as(C.POINTER(C.c_double)))
        return E[:n]

    def states(self):
        out = np.empty((self.k, self.params.sy, self.params.sx), dtype=np.complex128)
        st = _lib().itp2d_system_download_states(self.h, out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)))
        if st != capi.OK:
            raise capi.ITP2DError(st, "itp2d_system_download_states")
        return out

    def times(self) -> dict:
        t = np.zeros(7)
        _lib().itp2d_system_times(self.h, t.ctypes.data_as(C.POINTER(C.c_double)))
        return dict(zip(["total", "propagation", "orthonormalization", "dot", "eigensolve", "lincomb",
                         "convtest"], t.tolist()))

    def write_datafile(self, filename: str, clobber: bool = False, save_states: bool = True):
        """The reference's HDF5 datafile of this solve (--save final states):
        itp2d_system_write_datafile, read back with itp2d_b200.datafile."""
        from . import datafile
        datafile.write_system_datafile(self, filename, clobber, save_states)

    def context_handle(self) -> int:
        return _lib().itp2d_system_context(self.h)

    def set_flags(self, abort=None, save=None):
        """The abort and save flags this system reads (itpsystem.hpp:59-62):
        ctypes int objects or pointers (abort_flag() / save_flag()), or None."""
        def ptr(f):
            if f is None:
                return None
            return f if isinstance(f, C.POINTER(C.c_int)) else C.pointer(f)
        self._flags = (abort, save)  # keeps caller-owned ints alive
        st = _lib().itp2d_system_set_flags(self.h, ptr(abort), ptr(save))
        if st != capi.OK:
            raise capi.ITP2DError(st, "itp2d_system_set_flags")

    def set_save_callback(self, fn):
        """fn(states (k, sy, sx) complex128 copy in storage order, order (storage
        indices by ascending energy, or None), step) runs where the reference's
        save_states writes its datafile (itpsystem.cpp:374-389)."""
        if fn is None:
            self._save_cb = _SaveFn()
        else:
            def cb(_user, states, order, k, sx, sy, step):
                a = np.ctypeslib.as_array(states, shape=(k * sy * sx * 2,)).view(np.complex128)
                o = np.ctypeslib.as_array(order, shape=(k,)).copy() if order else None
                fn(a.reshape(k, sy, sx).copy(), o, step)
            self._save_cb = _SaveFn(cb)
        st = _lib().itp2d_system_set_save_callback(self.h, self._save_cb, None)
        if st != capi.OK:
            raise capi.ITP2DError(st, "itp2d_system_set_save_callback")

    @property
    def saves(self) -> int:
        return _lib().itp2d_system_saves(self.h)


class _RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("error_flag", C.c_int), ("iterations", C.c_int), ("converged", C.c_int),
                ("num_energies", C.c_int), ("t_submit", C.c_double), ("t_start", C.c_double),
                ("t_finish", C.c_double), ("footprint_bytes", C.c_double)]


class _ServerStats(C.Structure):
    _fields_ = [("queued", C.c_int), ("running", C.c_int), ("peak_running", C.c_int), ("completed", C.c_int),
                ("bytes_in_use", C.c_double), ("peak_bytes_in_use", C.c_double), ("budget_bytes", C.c_double),
                ("busy_seconds", C.c_double), ("overlap_seconds", C.c_double)]


_server_bound = False


def _server_lib():
    global _server_bound
    L = _lib()
    if not _server_bound:
        vp, i, d, dp = C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_double)
        L.itp2d_server_create.argtypes = [i, d, C.POINTER(vp)]
        L.itp2d_server_submit.argtypes = [vp, C.POINTER(_Params), dp, dp, C.POINTER(C.c_longlong)]
        L.itp2d_server_wait.argtypes = [vp, C.c_longlong, d, C.POINTER(_RequestInfo), dp, dp]
        L.itp2d_server_forget.argtypes = [vp, C.c_longlong]
        L.itp2d_server_get_stats.argtypes = [vp, C.POINTER(_ServerStats)]
        L.itp2d_server_last_error.argtypes = [vp]
        L.itp2d_server_last_error.restype = C.c_char_p
        L.itp2d_server_destroy.argtypes = [vp]
        L.itp2d_ctx_footprint.argtypes = [i, i, i, i, d, i]
        L.itp2d_ctx_footprint.restype = C.c_longlong
        _server_bound = True
    return L


def footprint(params: Parameters) -> int:
    """Device bytes a solve of these parameters allocates (itp2d_ctx_footprint)."""
    return _server_lib().itp2d_ctx_footprint(params.sx, params.sy, params.num_states, params.boundary,
                                             float(params.B), params.halforder)


class Server:
    """The serving loop of include/itp2d_host.h: requests queued as they
    arrive, admitted by device footprint, up to max_active solves at once on
    their own streams, each retired when it finishes."""

    def __init__(self, max_active: int, memory_budget_bytes: float):
        h = C.c_void_p()
        st = _server_lib().itp2d_server_create(int(max_active), float(memory_budget_bytes), C.byref(h))
        if st != capi.OK:
            raise capi.ITP2DError(st, "itp2d_server_create")
        self.h = h
        self.k = {}

    def submit(self, params: Parameters, extra_potential=None, init_states=None) -> int:
        raw = params._raw()
        ep = ip = None
        if extra_potential is not None:
            a = np.ascontiguousarray(extra_potential, dtype=np.float64).reshape(-1)
            ep = a.ctypes.data_as(C.POINTER(C.c_double))
        if init_states is not None:
            b = np.ascontiguousarray(init_states, dtype=np.complex128)
            ip = b.view(np.float64).ctypes.data_as(C.POINTER(C.c_double))
        rid = C.c_longlong(0)
        st = _server_lib().itp2d_server_submit(self.h, C.byref(raw), ep, ip, C.byref(rid))
        if st != capi.OK:
            raise capi.ITP2DError(st, "itp2d_server_submit")
        self.k[rid.value] = params.num_states
        return rid.value

    def wait(self, rid: int, timeout: float = 3600.0) -> dict:
        """Sorted energies, deviations and timing of a finished request;
        raises ITP2DError(E_TIMEOUT) if it does not finish within timeout s."""
        k = self.k[rid]
        info = _RequestInfo()
        E, sig = np.empty(k), np.empty(k)
        st = _server_lib().itp2d_server_wait(self.h, rid, float(timeout), C.byref(info),
                                             E.ctypes.data_as(C.POINTER(C.c_double)),
                                             sig.ctypes.data_as(C.POINTER(C.c_double)))
        if st != capi.OK:
            raise capi.ITP2DError(st, "itp2d_server_wait")
        out = {f: getattr(info, f) for f, _ in _RequestInfo._fields_}
        out["E"], out["sigma"] = E, sig
        return out

    def forget(self, rid: int) -> None:
        _server_lib().itp2d_server_forget(self.h, rid)
        self.k.pop(rid, None)

    def stats(self) -> dict:
        s = _ServerStats()
        _server_lib().itp2d_server_get_stats(self.h, C.byref(s))
        return {f: getattr(s, f) for f, _ in _ServerStats._fields_}

    @property
    def last_error(self) -> str:
        return _server_lib().itp2d_server_last_error(self.h).decode()

    def close(self):
        if getattr(self, "h", None):
            _server_lib().itp2d_server_destroy(self.h)
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


_batch_bound = False


def _batch_lib():
    global _batch_bound
    L = _server_lib()
    if not _batch_bound:
        vp, i, d, dp = C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_double)
        L.itp2d_batch_create.argtypes = [i, C.POINTER(_Params), C.POINTER(dp), C.POINTER(dp), C.POINTER(vp)]
        L.itp2d_batch_run.argtypes = [vp, i]
        L.itp2d_batch_result.argtypes = [vp, i, C.POINTER(_RequestInfo), dp, dp]
        L.itp2d_batch_size.argtypes = [vp]
        L.itp2d_batch_finished.argtypes = [vp]
        L.itp2d_batch_stats.argtypes = [vp, C.POINTER(C.c_longlong), dp]
        L.itp2d_batch_last_error.argtypes = [vp]
        L.itp2d_batch_last_error.restype = C.c_char_p
        L.itp2d_batch_destroy.argtypes = [vp]
        _batch_bound = True
    return L


class Batch:
    """The batched form of include/itp2d_host.h: many independent solves
    stepped together, one batched eigensolve launch per iteration."""

    def __init__(self, params: list, extra_potentials=None, init_states=None):
        n = len(params)
        raws = (_Params * n)(*[p._raw() for p in params])
        dp = C.POINTER(C.c_double)
        keep = []

        def ptrs(arrs, cplx):
            if arrs is None:
                return None
            out = (dp * n)()
            for j, a in enumerate(arrs):
                if a is None:
                    out[j] = None
                    continue
                b = np.ascontiguousarray(a, dtype=np.complex128 if cplx else np.float64)
                keep.append(b)
                out[j] = (b.view(np.float64) if cplx else b).ctypes.data_as(dp)
            return out
        h = C.c_void_p()
        st = _batch_lib().itp2d_batch_create(n, raws, ptrs(extra_potentials, False), ptrs(init_states, True),
                                             C.byref(h))
        if st != capi.OK:
            raise capi.ITP2DError(st, "itp2d_batch_create")
        self.h = h
        self.k = [p.num_states for p in params]

    def run(self, max_iterations: int = 1 << 30):
        st = _batch_lib().itp2d_batch_run(self.h, int(max_iterations))
        if st != capi.OK:
            raise capi.ITP2DError(st, "itp2d_batch_run: " + _batch_lib().itp2d_batch_last_error(self.h).decode())

    def result(self, i: int) -> dict:
        k = self.k[i]
        info = _RequestInfo()
        E, sig = np.empty(k), np.empty(k)
        st = _batch_lib().itp2d_batch_result(self.h, i, C.byref(info), E.ctypes.data_as(C.POINTER(C.c_double)),
                                             sig.ctypes.data_as(C.POINTER(C.c_double)))
        if st != capi.OK:
            raise capi.ITP2DError(st, "itp2d_batch_result")
        out = {f: getattr(info, f) for f, _ in _RequestInfo._fields_}
        out["E"], out["sigma"] = E, sig
        return out

    @property
    def finished(self) -> bool:
        return bool(_batch_lib().itp2d_batch_finished(self.h))

    def stats(self) -> dict:
        it, sec = C.c_longlong(0), C.c_double(0.0)
        _batch_lib().itp2d_batch_stats(self.h, C.byref(it), C.byref(sec))
        return {"iterations": it.value, "seconds": sec.value}

    def close(self):
        if getattr(self, "h", None):
            _batch_lib().itp2d_batch_destroy(self.h)
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
