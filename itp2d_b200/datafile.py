"""ctypes binding of include/itp2d_datafile.h: the reference's HDF5 datafile
(``Datafile``, datafile.cpp:32-467) and the --copy-states reader
(``StateSet::init_from_datafile``, stateset.cpp:86-109), both implemented in
libitp2d_b200.so without an HDF5 library. Host-only: no device is needed.

    f = Datafile("run.h5", sx, sy, dx, clobber=True)
    f.add_attribute("num_states", 64)
    f.write_stateset(states, step=10, sort_order=order)
    f.close()
    psi0 = init_states("run.h5", 64, sx, sy, dx)      # --copy-states
    E = read("run.h5", "final_energies")
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi

E_IO = 9
_bound = False


class DatafileError(RuntimeError):
    def __init__(self, status: int, what: str):
        msg = capi.lib().itp2d_datafile_last_error().decode(errors="replace")
        super().__init__(f"{what}: {msg} (status {status})")
        self.status = status


def _lib():
    global _bound
    L = capi.lib()
    if not _bound:
        vp, i, d, dp, ip, s = C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_char_p
        ll, llp = C.c_longlong, C.POINTER(C.c_longlong)
        L.itp2d_datafile_create.argtypes = [s, i, i, d, i, C.POINTER(vp)]
        L.itp2d_datafile_flush.argtypes = [vp]
        L.itp2d_datafile_set_chunking.argtypes = [vp, i]
        L.itp2d_datafile_close.argtypes = [vp]
        L.itp2d_datafile_add_attribute_int.argtypes = [vp, s, i]
        L.itp2d_datafile_add_attribute_double.argtypes = [vp, s, d]
        L.itp2d_datafile_add_attribute_ulong.argtypes = [vp, s, C.c_ulong]
        L.itp2d_datafile_add_attribute_string.argtypes = [vp, s, s]
        L.itp2d_datafile_write_state.argtypes = [vp, ll, ll, dp]
        L.itp2d_datafile_write_stateset.argtypes = [vp, dp, i, i, ip]
        L.itp2d_datafile_write_time_step_history.argtypes = [vp, i, d]
        for n in ["itp2d_datafile_write_energy_history", "itp2d_datafile_write_deviation_history"]:
            getattr(L, n).argtypes = [vp, dp, i, i]
        for n in ["itp2d_datafile_write_energies", "itp2d_datafile_write_energy_standard_deviations",
                  "itp2d_datafile_write_noise_realization"]:
            getattr(L, n).argtypes = [vp, dp, i]
        L.itp2d_datafile_write_potential.argtypes = [vp, dp]
        L.itp2d_datafile_save_states.argtypes = [vp, dp, ip, i, i, i, i]
        L.itp2d_datafile_save_states.restype = None
        L.itp2d_system_write_datafile.argtypes = [vp, s, i, i]
        L.itp2d_datafile_init_states.argtypes = [s, i, i, i, d, dp]
        L.itp2d_datafile_dataset_shape.argtypes = [s, s, ip, llp, llp]
        L.itp2d_datafile_read_values.argtypes = [s, s, dp, ll, llp]
        L.itp2d_datafile_read_attribute.argtypes = [s, s, s, dp]
        L.itp2d_datafile_read_string_attribute.argtypes = [s, s, s, C.c_char_p, i]
        L.itp2d_datafile_header_message.argtypes = [s, s, i, i, C.c_char_p, i, ip]
        L.itp2d_datafile_last_error.restype = C.c_char_p
        _bound = True
    return L


def _check(st: int, what: str):
    if st != capi.OK:
        raise DatafileError(st, what)


def _b(x):
    return None if x is None else (x.encode() if isinstance(x, str) else x)


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Datafile:
    """Datafile (datafile.hpp:38-147): the file exists from construction on and
    is rewritten as a whole by flush() and close()."""

    def __init__(self, filename: str, sx: int, sy: int, dx: float, clobber: bool = False):
        self.sx, self.sy = sx, sy
        h = C.c_void_p()
        _check(_lib().itp2d_datafile_create(_b(filename), sx, sy, dx, int(clobber), C.byref(h)),
               "itp2d_datafile_create")
        self.h = h

    def set_chunking(self, deflate_level: int = 9):
        """The reference's storage from now on: one element per chunk,
        deflated (a negative level: contiguous, the default)."""
        _check(_lib().itp2d_datafile_set_chunking(self.h, deflate_level), "set_chunking")

    def add_attribute(self, name: str, value, kind: str = None):
        """kind: "int", "double", "ulong" or "string" (default: from the value's type)."""
        L = _lib()
        if kind is None:
            kind = "string" if isinstance(value, str) else "int" if isinstance(value, (int, np.integer)) else "double"
        fn = {"int": L.itp2d_datafile_add_attribute_int, "double": L.itp2d_datafile_add_attribute_double,
              "ulong": L.itp2d_datafile_add_attribute_ulong,
              "string": L.itp2d_datafile_add_attribute_string}[kind]
        _check(fn(self.h, _b(name), _b(value) if kind == "string" else value), f"add_attribute({name})")

    def write_state(self, n: int, m: int, state):
        a = np.ascontiguousarray(state, dtype=np.complex128).reshape(self.sy, self.sx)
        _check(_lib().itp2d_datafile_write_state(self.h, n, m, _dp(a.view(np.float64))), "write_state")

    def write_stateset(self, states, step: int, sort_order=None):
        a = np.ascontiguousarray(states, dtype=np.complex128)
        k = a.shape[0]
        o = None
        if sort_order is not None:
            o = np.ascontiguousarray(sort_order, dtype=np.int32)
            assert o.size == k
        _check(_lib().itp2d_datafile_write_stateset(self.h, _dp(a.view(np.float64)), k, step,
                                                    None if o is None else o.ctypes.data_as(C.POINTER(C.c_int))),
               "write_stateset")

    def write_time_step_history(self, step: int, eps: float):
        _check(_lib().itp2d_datafile_write_time_step_history(self.h, step, eps), "write_time_step_history")

    def _row(self, fn, values, index):
        a = np.ascontiguousarray(values, dtype=np.float64)
        _check(fn(self.h, _dp(a), a.size, index), fn.__name__)

    def write_energy_history(self, values, index: int):
        self._row(_lib().itp2d_datafile_write_energy_history, values, index)

    def write_deviation_history(self, values, index: int):
        self._row(_lib().itp2d_datafile_write_deviation_history, values, index)

    def _vec(self, fn, values):
        a = np.ascontiguousarray(values, dtype=np.float64)
        _check(fn(self.h, _dp(a), a.size), fn.__name__)

    def write_energies(self, values):
        self._vec(_lib().itp2d_datafile_write_energies, values)

    def write_energy_standard_deviations(self, values):
        self._vec(_lib().itp2d_datafile_write_energy_standard_deviations, values)

    def write_noise_realization(self, values):
        self._vec(_lib().itp2d_datafile_write_noise_realization, values)

    def write_potential(self, V):
        a = np.ascontiguousarray(V, dtype=np.float64).reshape(self.sy, self.sx)
        _check(_lib().itp2d_datafile_write_potential(self.h, _dp(a)), "write_potential")

    def save_states(self, states, order, step: int):
        """The save-callback entry (itp2d_datafile_save_states) called directly."""
        a = np.ascontiguousarray(states, dtype=np.complex128)
        o = None if order is None else np.ascontiguousarray(order, dtype=np.int32)
        _lib().itp2d_datafile_save_states(self.h, _dp(a.view(np.float64)),
                                          None if o is None else o.ctypes.data_as(C.POINTER(C.c_int)),
                                          a.shape[0], self.sx, self.sy, step)

    def flush(self):
        _check(_lib().itp2d_datafile_flush(self.h), "flush")

    def close(self):
        if getattr(self, "h", None):
            h, self.h = self.h, None
            _check(_lib().itp2d_datafile_close(h), "close")

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def write_system_datafile(system, filename: str, clobber: bool = False, save_states: bool = True):
    """The datafile of a solve run by itp2d_b200.system.ITPSystem
    (itp2d_system_write_datafile)."""
    _check(_lib().itp2d_system_write_datafile(system.h, _b(filename), int(clobber), int(save_states)),
           "itp2d_system_write_datafile")


def init_states(filename: str, num_states: int, sx: int, sy: int, dx: float) -> np.ndarray:
    """--copy-states: the last saved state set, checked against the grid."""
    out = np.empty((num_states, sy, sx), dtype=np.complex128)
    _check(_lib().itp2d_datafile_init_states(_b(filename), num_states, sx, sy, dx, _dp(out.view(np.float64))),
           "itp2d_datafile_init_states")
    return out


def shape(filename: str, dataset: str):
    """(dims tuple, numeric values per element)."""
    r = C.c_int()
    dims = (C.c_longlong * 8)()
    per = C.c_longlong()
    _check(_lib().itp2d_datafile_dataset_shape(_b(filename), _b(dataset), C.byref(r), dims, C.byref(per)),
           f"shape({dataset})")
    return tuple(dims[i] for i in range(r.value)), per.value


def read(filename: str, dataset: str) -> np.ndarray:
    """Every numeric value of a dataset as float64, shaped dims + (values per
    element,) when an element holds more than one value."""
    dims, per = shape(filename, dataset)
    n = C.c_longlong()
    total = int(np.prod(dims, dtype=np.int64)) * per
    out = np.empty(max(total, 1), dtype=np.float64)
    _check(_lib().itp2d_datafile_read_values(_b(filename), _b(dataset), _dp(out), total, C.byref(n)),
           f"read({dataset})")
    assert n.value == total
    return out[:total].reshape(tuple(dims) + ((per,) if per != 1 else ()))


def attribute(filename: str, name: str, obj: str = "/") -> float:
    v = C.c_double()
    _check(_lib().itp2d_datafile_read_attribute(_b(filename), _b(obj), _b(name), C.byref(v)), f"attribute({name})")
    return v.value


def string_attribute(filename: str, name: str, obj: str = "/") -> str:
    buf = C.create_string_buffer(65536)
    _check(_lib().itp2d_datafile_read_string_attribute(_b(filename), _b(obj), _b(name), buf, len(buf)),
           f"string_attribute({name})")
    return buf.value.decode(errors="replace")


def header_message(filename: str, obj: str, mtype: int, index: int = 0) -> bytes:
    """Body of the index-th object-header message of type mtype."""
    size = C.c_int()
    buf = C.create_string_buffer(65536)
    _check(_lib().itp2d_datafile_header_message(_b(filename), _b(obj), mtype, index, buf, len(buf),
                                                C.byref(size)), f"header_message({obj}, {mtype})")
    return buf.raw[:size.value]
