"""The HDF5 datafile (include/itp2d_datafile.h) on the CPU: the reference's
Datafile (datafile.cpp:32-467) and StateSet::init_from_datafile
(stateset.cpp:86-109) without an HDF5 library.

Pinning. No HDF5 library or h5py is installed, but the image holds a file
written by the HDF5 library itself (scipy's MATLAB 7.3 test file, an HDF5
file behind a 512-byte user block). The reader must read it to the values
that scipy.io.loadmat gives for the same matrix in the 7.1 format, and the
writer's encodings of the shared structures (superblock fields, double
datatype, version 1 dataspace, fill value, string attribute, local heap free
list) must equal that file's byte for byte. A small walker written here from
the format specification, independent of the library's reader, checks the
root group of a written file."""
import ctypes as C
import os
import re
import struct

import numpy as np
import pytest

from itp2d_b200 import capi
from itp2d_b200 import datafile as D

SCIPY_DATA = None
try:
    import scipy.io
    SCIPY_DATA = os.path.join(os.path.dirname(scipy.io.__file__), "matlab", "tests", "data")
except ImportError:  # pragma: no cover
    pass
LIBHDF5_FILE = os.path.join(SCIPY_DATA or "", "testhdf5_7.4_GLNX86.mat")
V71_FILE = os.path.join(SCIPY_DATA or "", "testdouble_7.1_GLNX86.mat")
needs_libhdf5_file = pytest.mark.skipif(not os.path.exists(LIBHDF5_FILE), reason="no HDF5-library file in this image")

MSG_SPACE, MSG_TYPE, MSG_FILL, MSG_LAYOUT, MSG_ATTR = 1, 3, 5, 8, 12


def test_library_exports_datafile_header_symbols():
    txt = open(os.path.join(capi.ROOT, "include", "itp2d_datafile.h")).read()
    names = sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*\**\s+\**(itp2d_[a-z0-9_]+)\s*\(",
                                  txt, flags=re.M)))
    assert len(names) == 26
    lib = capi.lib()
    for n in names:
        assert hasattr(lib, n), n


@needs_libhdf5_file
def test_reader_reads_a_file_written_by_the_hdf5_library():
    assert D.shape(LIBHDF5_FILE, "testdouble") == ((9, 1), 1)
    v = D.read(LIBHDF5_FILE, "testdouble").ravel()
    ref = scipy.io.loadmat(V71_FILE)["testdouble"].ravel()
    assert np.array_equal(v, ref)  # 0, pi/4, ..., 2 pi
    assert D.string_attribute(LIBHDF5_FILE, "MATLAB_class", "testdouble") == "double"


def _real_superblock():
    b = open(LIBHDF5_FILE, "rb").read()
    at = b.find(b"\x89HDF\r\n\x1a\n")
    return b, at


@needs_libhdf5_file
def test_writer_encodings_match_the_hdf5_library(tmp_path):
    p = str(tmp_path / "enc.h5")
    with D.Datafile(p, 4, 2, 0.5, clobber=True) as f:
        f.add_attribute("MATLAB_class", "double")
        for i in range(9):  # a 9 x 1 double dataset, the shape of the library's file
            f.write_energy_history([i * 0.25], i)
        f.write_energies([1.0])
    # datatype (IEEE double), version 1 dataspace of 9 x 1, fill value
    for t in (MSG_TYPE, MSG_SPACE, MSG_FILL):
        assert D.header_message(p, "energy_history", t) == D.header_message(LIBHDF5_FILE, "testdouble", t), t
    # the scalar C-string attribute, name, type, space and value
    mine = [D.header_message(p, "/", MSG_ATTR, i) for i in range(5)]
    assert D.header_message(LIBHDF5_FILE, "testdouble", MSG_ATTR, 0) in mine
    # superblock: signature, versions, sizes of offsets and lengths, group internal K
    real, at = _real_superblock()
    ours = open(p, "rb").read()
    assert ours[:16] == real[at:at + 16]
    assert ours[18:20] == real[at + 18:at + 20]
    # local heap: the library marks "no further free block" with offset 1
    heap = ours.find(b"HEAP")
    assert struct.unpack_from("<Q", ours, heap + 16)[0] == 1
    rheap = real.find(b"HEAP")
    _, free, data = struct.unpack_from("<QQQ", real, rheap + 8)
    base = struct.unpack_from("<Q", real, at + 24)[0]  # the user block's size
    assert struct.unpack_from("<Q", real, base + data + free)[0] == 1  # the free block's "next"


def _states(rng, k, sy, sx):
    return rng.normal(size=(k, sy, sx)) + 1j * rng.normal(size=(k, sy, sx))


def test_round_trip_every_dataset_and_attribute(tmp_path):
    p = str(tmp_path / "run.h5")
    sx, sy, dx, k = 6, 4, 0.5, 3
    rng = np.random.default_rng(7)
    st = _states(rng, k, sy, sx)
    V = rng.normal(size=(sy, sx))
    with D.Datafile(p, sx, sy, dx, clobber=True) as f:
        f.add_attribute("num_states", k)
        f.add_attribute("random_seed", 2 ** 40 + 5, "ulong")
        f.add_attribute("magnetic_field_strength", 0.5)
        f.add_attribute("potential", "harmonic(1)")
        f.add_attribute("empty", "")
        f.write_stateset(st, 7, [2, 0, 1])
        f.write_stateset(st, 9)
        f.write_time_step_history(1, 0.1)
        f.write_time_step_history(5, 0.05)
        f.write_energy_history([1, 2, 3], 0)
        f.write_energy_history([1.5, 2.5, 3.5], 2)  # row 1 stays zero, like an extended HDF5 dataset
        f.write_deviation_history([0.1, 0.2, 0.3], 0)
        f.write_energies([1, 2, 3.25])
        f.write_energy_standard_deviations([1e-3, 2e-3, 3e-3])
        f.write_potential(V)
        f.write_noise_realization([])
    assert D.shape(p, "states") == ((2, k), 2 * sx * sy)
    assert D.shape(p, "potential_values") == ((), sx * sy)
    s = D.read(p, "states").reshape(2, k, sy, sx, 2)
    c = s[..., 0] + 1j * s[..., 1]
    assert np.array_equal(c[0], st[[2, 0, 1]]) and np.array_equal(c[1], st)
    assert np.array_equal(D.read(p, "state_history"), [[7, 0], [9, 1]])
    assert np.array_equal(D.read(p, "time_step_history"), [[1, 0.1], [5, 0.05]])
    assert np.array_equal(D.read(p, "energy_history"), [[1, 2, 3], [0, 0, 0], [1.5, 2.5, 3.5]])
    assert np.array_equal(D.read(p, "deviation_history"), [[0.1, 0.2, 0.3]])
    assert np.array_equal(D.read(p, "final_energies"), [1, 2, 3.25])
    assert np.array_equal(D.read(p, "final_energy_standard_deviations"), [1e-3, 2e-3, 3e-3])
    assert np.array_equal(D.read(p, "potential_values").reshape(sy, sx), V)
    assert D.read(p, "noise_data").shape == (0,)
    assert D.attribute(p, "num_states") == k and D.attribute(p, "random_seed") == 2 ** 40 + 5
    assert (D.attribute(p, "grid_sizex"), D.attribute(p, "grid_sizey"), D.attribute(p, "grid_delta")) == (sx, sy, dx)
    assert D.string_attribute(p, "potential") == "harmonic(1)" and D.string_attribute(p, "empty") == ""
    for name in ["states", "energy_history", "potential_values", "noise_data"]:
        assert len(D.string_attribute(p, "description", name)) > 20


def test_write_state_grows_with_zero_fill(tmp_path):
    p = str(tmp_path / "s.h5")
    rng = np.random.default_rng(3)
    a = _states(rng, 1, 2, 3)[0]
    with D.Datafile(p, 3, 2, 1.0, clobber=True) as f:
        f.write_state(1, 2, a)
    s = D.read(p, "states").reshape(2, 3, 2, 3, 2)
    c = s[..., 0] + 1j * s[..., 1]
    assert np.array_equal(c[1, 2], a)
    c[1, 2] = 0
    assert not np.any(c)


def _copy_states_file(path, k, sx, sy, dx, st):
    with D.Datafile(path, sx, sy, dx, clobber=True) as f:
        f.add_attribute("num_states", k)
        f.write_stateset(st, 3)
        f.write_stateset(st[::-1], 4)


def test_init_states_checks_the_grid_like_the_reference(tmp_path):
    p = str(tmp_path / "c.h5")
    sx, sy, dx, k = 8, 6, 0.25, 4
    st = _states(np.random.default_rng(5), k, sy, sx)
    _copy_states_file(p, k, sx, sy, dx, st)
    assert np.array_equal(D.init_states(p, k, sx, sy, dx), st[::-1])  # the last slot
    for args, what in [((k + 1, sx, sy, dx), "num_states"), ((k, sx + 1, sy, dx), "grid_sizex"),
                       ((k, sx, sy + 2, dx), "grid_sizey"), ((k, sx, sy, dx * 2), "grid_delta")]:
        with pytest.raises(D.DatafileError) as e:
            D.init_states(p, *args)
        assert e.value.status == capi.E_INVALID
        assert f"value for {what} does not match" in str(e.value)


def test_create_is_exclusive_unless_clobber(tmp_path):
    p = str(tmp_path / "x.h5")
    D.Datafile(p, 2, 2, 1.0).close()
    with pytest.raises(D.DatafileError) as e:
        D.Datafile(p, 2, 2, 1.0)
    assert e.value.status == D.E_IO
    D.Datafile(p, 2, 2, 1.0, clobber=True).close()
    with pytest.raises(D.DatafileError):
        D.Datafile(str(tmp_path / "no" / "such" / "dir.h5"), 2, 2, 1.0, clobber=True)
    with D.Datafile(str(tmp_path / "y.h5"), 2, 2, 1.0) as f:
        f.add_attribute("a", 1)
        with pytest.raises(D.DatafileError):
            f.add_attribute("a", 2)  # createAttribute on an existing name fails


def test_reader_rejects_what_it_cannot_read(tmp_path):
    p = tmp_path / "junk.h5"
    p.write_bytes(b"not an hdf5 file" * 64)
    with pytest.raises(D.DatafileError) as e:
        D.read(str(p), "states")
    assert e.value.status == D.E_IO
    q = str(tmp_path / "ok.h5")
    D.Datafile(q, 2, 2, 1.0).close()
    with pytest.raises(D.DatafileError) as e:
        D.read(q, "states")
    assert e.value.status == capi.E_INVALID  # no such dataset
    with pytest.raises(D.DatafileError):
        D.attribute(q, "description")  # a string is not a number
    # a truncated file fails cleanly
    b = open(q, "rb").read()
    (tmp_path / "cut.h5").write_bytes(b[:200])
    with pytest.raises(D.DatafileError):
        D.attribute(str(tmp_path / "cut.h5"), "grid_sizex")


def test_save_states_callback_writes_a_slot_per_call(tmp_path):
    """itp2d_datafile_save_states is the driver's save callback
    (itp2d_system_set_save_callback) with the datafile as its user pointer;
    each call appends a slot in energy order and flushes."""
    p = str(tmp_path / "cb.h5")
    sx, sy, k = 4, 4, 3
    st = _states(np.random.default_rng(11), k, sy, sx)
    f = D.Datafile(p, sx, sy, 0.5, clobber=True)
    f.save_states(st, [1, 2, 0], 5)
    assert D.shape(p, "states")[0] == (1, k)  # on disk before close
    f.save_states(st, None, 6)
    f.close()
    s = D.read(p, "states").reshape(2, k, sy, sx, 2)
    c = s[..., 0] + 1j * s[..., 1]
    assert np.array_equal(c[0], st[[1, 2, 0]]) and np.array_equal(c[1], st)
    assert np.array_equal(D.read(p, "state_history"), [[5, 0], [6, 1]])
    fn = C.cast(capi.lib().itp2d_datafile_save_states, C.c_void_p).value
    assert fn  # a plain function pointer, usable as an itp2d_save_states_fn


def _walk_root(path):
    """Root-group links of a version 0 superblock file, read straight from the
    format specification (superblock -> root symbol-table entry -> B-tree leaf
    -> symbol-table node -> local heap)."""
    b = open(path, "rb").read()
    assert b[:8] == b"\x89HDF\r\n\x1a\n" and b[8] == 0
    leaf_k, internal_k = struct.unpack_from("<HH", b, 16)
    base, _, eof, _ = struct.unpack_from("<QQQQ", b, 24)
    assert eof == len(b)
    _, root, cache, _, btree, heap = struct.unpack_from("<QQIIQQ", b, 56)
    assert cache == 1
    assert b[heap:heap + 4] == b"HEAP"
    hsize, hfree, hdata = struct.unpack_from("<QQQ", b, heap + 8)
    assert b[btree:btree + 4] == b"TREE" and b[btree + 4] == 0 and b[btree + 5] == 0
    n = struct.unpack_from("<H", b, btree + 6)[0]
    links = []
    for i in range(n):
        snod = struct.unpack_from("<Q", b, btree + 32 + 16 * i)[0]
        assert b[snod:snod + 4] == b"SNOD"
        for j in range(struct.unpack_from("<H", b, snod + 6)[0]):
            off, hdr = struct.unpack_from("<QQ", b, snod + 8 + 40 * j)
            name = b[hdata + off:b.index(b"\0", hdata + off)].decode()
            assert b[hdr] == 1  # version 1 object header
            links.append(name)
        last = struct.unpack_from("<Q", b, btree + 40 + 16 * i)[0]
        assert b[hdata + last:b.index(b"\0", hdata + last)].decode() == links[-1]
    return leaf_k, internal_k, links


def test_independent_walk_of_a_written_file(tmp_path):
    p = str(tmp_path / "w.h5")
    with D.Datafile(p, 4, 4, 0.5, clobber=True) as f:
        f.write_energies([1.0, 2.0])
        f.write_time_step_history(1, 0.5)
        f.write_noise_realization([0.5])
        f.write_stateset(np.ones((2, 4, 4), complex), 1)
        f.write_energy_history([1.0, 2.0], 0)
        f.write_deviation_history([1.0, 2.0], 0)
        f.write_energy_standard_deviations([1.0, 2.0])
        f.write_potential(np.zeros((4, 4)))
    leaf_k, internal_k, links = _walk_root(p)
    assert links == sorted(links)  # a symbol-table node lists names in order
    assert set(links) == {"deviation_history", "energy_history", "final_energies", "final_energy_standard_deviations",
                          "noise_data", "potential_values", "state_history", "states", "time_step_history"}
    assert len(links) <= 2 * leaf_k and internal_k == 16


def _decode_type(b, p):
    """A datatype message body decoded from the specification's field tables
    (classes 0, 1, 6 version 1 and 10 version 2), independent of the library."""
    cls, ver = b[p] & 15, b[p] >> 4
    size = struct.unpack_from("<I", b, p + 4)[0]
    if cls == 0:
        return ("int", size, bool(b[p + 1] & 8)), p + 12
    if cls == 1:
        assert b[p + 1:p + 4] == bytes([0x20, 63, 0]) and size == 8
        return ("double",), p + 20
    if cls == 6:
        assert ver == 1
        n = struct.unpack_from("<H", b, p + 1)[0]
        q, members = p + 8, []
        for _ in range(n):
            end = b.index(b"\0", q)
            name = b[q:end].decode()
            q += (end - q + 8) // 8 * 8
            off = struct.unpack_from("<I", b, q)[0]
            assert b[q + 4] == 0  # no member dimensions
            t, q = _decode_type(b, q + 32)
            members.append((name, off, t))
        return ("compound", size, members), q
    if cls == 10:
        assert ver == 2
        nd = b[p + 8]
        dims = struct.unpack_from(f"<{nd}I", b, p + 12)
        perm = struct.unpack_from(f"<{nd}I", b, p + 12 + 4 * nd)
        assert perm == tuple(range(nd))
        t, q = _decode_type(b, p + 12 + 8 * nd)
        return ("array", size, dims, t), q
    raise AssertionError(f"class {cls}")


def test_compound_and_array_encodings_follow_the_specification(tmp_path):
    p = str(tmp_path / "t.h5")
    sx, sy = 5, 3
    with D.Datafile(p, sx, sy, 0.5, clobber=True) as f:
        f.write_stateset(np.zeros((2, sy, sx), complex), 1)
        f.write_time_step_history(1, 0.5)
        f.write_potential(np.zeros((sy, sx)))
    dbl = ("double",)
    cplx = ("compound", 16, [("r", 0, dbl), ("i", 8, dbl)])
    expect = {
        "states": ("array", 16 * sx * sy, (sy, sx), cplx),
        "state_history": ("compound", 8, [("step", 0, ("int", 4, True)), ("index", 4, ("int", 4, True))]),
        "time_step_history": ("compound", 16, [("step", 0, ("int", 4, True)), ("time_step", 8, dbl)]),
        "potential_values": ("array", 8 * sx * sy, (sy, sx), dbl),
    }
    for name, want in expect.items():
        body = D.header_message(p, name, MSG_TYPE)
        got, end = _decode_type(body, 0)
        assert got == want, name
        assert len(body) - end < 8  # only the message's padding follows


def test_reader_refuses_a_directory(tmp_path):
    with pytest.raises(D.DatafileError) as e:
        D.read(str(tmp_path), "states")
    assert e.value.status == D.E_IO


def test_truncated_and_corrupted_files_fail_cleanly(tmp_path):
    """Every truncation, and a flipped byte anywhere, gives a status or
    values, never a crash (the reader bounds-checks every field)."""
    p = str(tmp_path / "good.h5")
    with D.Datafile(p, 5, 3, 0.5, clobber=True) as f:
        f.add_attribute("num_states", 2)
        f.write_stateset(np.ones((2, 3, 5), complex), 1, [1, 0])
        f.write_energy_history([1.0, 2.0], 0)
        f.write_time_step_history(1, 0.5)
    good = open(p, "rb").read()
    q = tmp_path / "bad.h5"
    for cut in range(0, len(good), 37):
        q.write_bytes(good[:cut])
        with pytest.raises(D.DatafileError):
            D.read(str(q), "states")
    for i in range(0, len(good), 13):
        b = bytearray(good)
        b[i] ^= 0xFF
        q.write_bytes(bytes(b))
        for call in (lambda: D.read(str(q), "states"), lambda: D.attribute(str(q), "num_states"),
                     lambda: D.string_attribute(str(q), "description", "states")):
            try:
                call()
            except D.DatafileError:
                pass


def _write_run(path, chunk_level=None):
    sx, sy, k = 6, 4, 40
    rng = np.random.default_rng(21)
    st = _states(rng, k, sy, sx)
    with D.Datafile(path, sx, sy, 0.5, clobber=True) as f:
        if chunk_level is not None:
            f.set_chunking(chunk_level)
        f.add_attribute("num_states", k)
        f.write_stateset(st, 3)
        f.write_stateset(st[::-1], 5, np.arange(k)[::-1])  # 80 chunks: a two-level chunk index
        for i in range(30):  # 30 x 40 = 1200 chunks of one double
            f.write_energy_history(rng.normal(size=k), i)
        f.write_time_step_history(1, 0.5)
        f.write_energies(rng.normal(size=k))
        f.write_potential(rng.normal(size=(sy, sx)))
        f.write_noise_realization([])
        f.write_state(3, 1, st[7])  # grows states to 4 slots, zero-filled
    return st


def test_chunked_deflated_storage_reads_like_contiguous(tmp_path):
    """The reference's storage (one element per chunk, deflate 9, unlimited
    maximum sizes, datafile.cpp:76-88) holds the same values as the
    contiguous default, and --copy-states reads it."""
    a, b = str(tmp_path / "contiguous.h5"), str(tmp_path / "chunked.h5")
    st = _write_run(a)
    _write_run(b, 9)
    for name in ["states", "state_history", "energy_history", "time_step_history", "final_energies",
                 "potential_values", "noise_data"]:
        assert D.shape(a, name) == D.shape(b, name), name
        assert np.array_equal(D.read(a, name), D.read(b, name)), name
    assert np.array_equal(D.init_states(b, 40, 6, 4, 0.5)[1], st[7])
    # the layout, filter and dataspace messages say what the reference's datasets say
    lay = D.header_message(b, "energy_history", MSG_LAYOUT)
    assert lay[:3] == bytes([3, 2, 3]) and struct.unpack_from("<III", lay, 11) == (1, 1, 8)
    flt = D.header_message(b, "energy_history", 11)
    assert struct.unpack_from("<HHHH", flt, 8) == (1, 8, 0, 1) and struct.unpack_from("<I", flt, 24)[0] == 9
    spc = D.header_message(b, "energy_history", MSG_SPACE)
    assert spc[2] & 1 and struct.unpack_from("<QQ", spc, 24) == (2 ** 64 - 1, 2 ** 64 - 1)
    assert D.header_message(b, "potential_values", MSG_LAYOUT)[:2] == bytes([3, 1])  # scalar stays contiguous


def _inflate_chunks(b, tree, nd, out, es, dims):
    """Chunk B-tree (type 1) walked from the specification, chunks inflated
    with Python's zlib and placed by their offsets."""
    import zlib
    assert b[tree:tree + 4] == b"TREE" and b[tree + 4] == 1
    level, n = b[tree + 5], struct.unpack_from("<H", b, tree + 6)[0]
    ks = 8 + 8 * nd
    for i in range(n):
        key = tree + 24 + i * (ks + 8)
        size, mask = struct.unpack_from("<II", b, key)
        off = struct.unpack_from(f"<{nd}Q", b, key + 8)
        child = struct.unpack_from("<Q", b, key + ks)[0]
        if level:
            _inflate_chunks(b, child, nd, out, es, dims)
            continue
        raw = zlib.decompress(b[child:child + size])
        assert len(raw) == es and mask == 0
        lin = 0
        for d, o in zip(dims, off[:-1]):
            lin = lin * d + o
        out[lin * es:(lin + 1) * es] = raw


def test_chunk_index_decoded_independently(tmp_path):
    p = str(tmp_path / "chunked.h5")
    _write_run(p, 6)
    b = open(p, "rb").read()
    lay = D.header_message(p, "energy_history", MSG_LAYOUT)
    tree = struct.unpack_from("<Q", lay, 3)[0]
    dims, _ = D.shape(p, "energy_history")
    out = bytearray(8 * int(np.prod(dims)))
    _inflate_chunks(b, tree, 3, out, 8, dims)
    assert np.array_equal(np.frombuffer(bytes(out), dtype="<f8").reshape(dims), D.read(p, "energy_history"))
    assert b[tree + 5] == 1  # 1200 chunks: leaves under one internal node
