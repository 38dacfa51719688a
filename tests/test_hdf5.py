"""HDF5 mesh I/O, file-format level (include/op_hdf5.h's op2b_h5_* helpers:
host code, no GPU): the reader against a file written by the HDF5 library
(scipy's MATLAB 7.3 test file, when installed), against a file built here
field by field from the HDF5 File Format Specification with the layouts the
writer never produces (superblock v2, v2 object headers, link messages,
chunked storage with shuffle + deflate, big-endian integers, v3 attributes),
and round trips through the writer (every type, nested groups, large groups,
replacement, additions to a library-written file)."""
import os
import struct
import zlib

import numpy as np
import pytest

from op2b import lib as L

UNDEF = 0xFFFFFFFFFFFFFFFF


def _matlab_file():
    try:
        import scipy.io.matlab as m
    except ImportError:
        return None
    p = os.path.join(os.path.dirname(m.__file__), "tests", "data", "testhdf5_7.4_GLNX86.mat")
    return p if os.path.exists(p) else None


MAT = _matlab_file()


@pytest.mark.skipif(MAT is None, reason="scipy's HDF5-based MATLAB test file is not installed")
def test_reads_a_file_written_by_the_hdf5_library():
    # MATLAB 7.4 wrote it through the HDF5 library: a 512-byte user block,
    # superblock v0, symbol-table root group, a contiguous double dataset
    # (0:pi/4:2*pi, stored 9 x 1) with a string attribute
    assert L.h5_list(MAT) == ["/testdouble"]
    assert L.h5_info(MAT, "testdouble") == ((9, 1), "double")
    v = L.h5_read(MAT, "/testdouble").ravel()
    np.testing.assert_allclose(v, np.arange(9) * np.pi / 4, rtol=2e-16, atol=0)
    assert L.h5_get_attr(MAT, "testdouble", "MATLAB_class") == "double"
    assert L.h5_info(MAT, "nothing") is None


@pytest.mark.skipif(MAT is None, reason="scipy's HDF5-based MATLAB test file is not installed")
def test_adding_to_a_library_written_file_keeps_what_was_there(tmp_path):
    f = str(tmp_path / "m.h5")
    with open(MAT, "rb") as src, open(f, "wb") as dst:
        dst.write(src.read())
    L.h5_write(f, "/extra/q", np.ones((3, 4)))
    assert L.h5_list(f) == ["/extra/", "/extra/q", "/testdouble"]
    np.testing.assert_array_equal(L.h5_read(f, "testdouble").ravel(),
                                  L.h5_read(MAT, "testdouble").ravel())
    assert L.h5_get_attr(f, "testdouble", "MATLAB_class") == "double"


@pytest.mark.parametrize("dtype", [np.int32, np.int64, np.float32, np.float64])
def test_round_trip_of_every_type(tmp_path, dtype):
    f = str(tmp_path / "t.h5")
    rng = np.random.default_rng(3)
    a = (rng.standard_normal((17, 3)) * 1000).astype(dtype)
    L.h5_write(f, "/a/b/c", a)
    shape, t = L.h5_info(f, "/a/b/c")
    assert shape == (17, 3) and t == {np.int32: "int", np.int64: "long",
                                      np.float32: "float", np.float64: "double"}[dtype]
    np.testing.assert_array_equal(L.h5_read(f, "a/b/c"), a)
    # and converted on reading, as the library converts to a native type
    if np.issubdtype(dtype, np.integer):
        np.testing.assert_array_equal(L.h5_read(f, "a/b/c", "double"), a.astype(np.float64))
    else:
        np.testing.assert_array_equal(L.h5_read(f, "a/b/c", "int"),
                                      np.trunc(a.astype(np.float64)).astype(np.int32))


def test_scalars_empty_datasets_and_replacement(tmp_path):
    f = str(tmp_path / "s.h5")
    L.h5_write(f, "scalar", np.array(7, dtype=np.int32))
    L.h5_write(f, "empty", np.zeros((0, 4)))
    L.h5_write(f, "x", np.arange(4.0))
    assert L.h5_info(f, "scalar") == ((), "int")
    assert int(L.h5_read(f, "scalar")) == 7
    assert L.h5_read(f, "empty").shape == (0, 4)
    L.h5_write(f, "x", np.arange(6, dtype=np.int32).reshape(2, 3))   # replaced
    np.testing.assert_array_equal(L.h5_read(f, "x"), np.arange(6).reshape(2, 3))
    assert L.h5_list(f) == ["/empty", "/scalar", "/x"]
    with pytest.raises(L.Op2Error):
        L.h5_write(f, "/x/y", np.zeros(2))     # x is a dataset, not a group


def test_large_groups_and_attributes(tmp_path):
    f = str(tmp_path / "g.h5")
    for i in range(300):
        L.h5_write(f, f"/many/d{i:03d}", np.array([i, -i], dtype=np.int64))
    names = L.h5_list(f)
    assert len(names) == 301 and names[0] == "/many/" and names[-1] == "/many/d299"
    for i in (0, 7, 8, 150, 299):
        np.testing.assert_array_equal(L.h5_read(f, f"many/d{i:03d}"), [i, -i])
    L.h5_set_attr(f, "/many/d005", "dim", [2])
    L.h5_set_attr(f, "/many/d005", "type", "long", "string")
    L.h5_set_attr(f, "/many", "note", [1.5, 2.5], "double")
    assert L.h5_get_attr(f, "/many/d005", "dim") == "2"
    assert L.h5_get_attr(f, "/many/d005", "type") == "long"
    assert L.h5_get_attr(f, "/many", "note") == "1.5 2.5"
    assert L.h5_get_attr(f, "/many/d005", "absent") is None


def test_errors_are_reported(tmp_path):
    bad = tmp_path / "not.h5"
    bad.write_bytes(b"plain text, no signature" * 40)
    with pytest.raises(L.Op2Error, match="not an HDF5 file"):
        L.h5_list(str(bad))
    with pytest.raises(L.Op2Error, match="cannot open"):
        L.h5_list(str(tmp_path / "missing.h5"))
    f = str(tmp_path / "e.h5")
    L.h5_write(f, "x", np.arange(3.0))
    out = np.empty(5)
    assert L.load().op2b_h5_read(f.encode(), b"x", b"double", out.ctypes.data, 5) == -1
    assert "3 elements" in L.last_error()
    with pytest.raises(L.Op2Error):
        L.h5_read(f, "y")


# ---------------------------------------------------------------------------
# A file built field by field from the format specification, in the layouts
# the writer never produces.


def _ohdr_v2(messages):
    """Version-2 object header: messages as (type, bytes); 4-byte chunk size."""
    body = b"".join(struct.pack("<BHB", t, len(d), 0) + d for t, d in messages)
    return b"OHDR" + bytes([2, 0x02]) + struct.pack("<I", len(body)) + body + b"\0\0\0\0"


def _link(name, addr):
    n = name.encode()
    return 6, bytes([1, 0, len(n)]) + n + struct.pack("<Q", addr)


def _space_v2(dims):
    return 1, bytes([2, len(dims), 0, 1]) + b"".join(struct.pack("<Q", d) for d in dims)


def _int32_be():
    # class 0 version 1, big endian, signed; offset 0, precision 32
    return 3, bytes([0x10, 0x09, 0, 0]) + struct.pack("<IHH", 4, 0, 32)


def _f64_le():
    return 3, bytes([0x11, 0x20, 63, 0]) + struct.pack("<IHHBBBBI", 8, 0, 64, 52, 11, 0, 52, 1023)


def _string(n):
    return bytes([0x13, 0x00, 0, 0]) + struct.pack("<I", n)


def _attr_v3(name, text):
    dt = _string(len(text))
    ds = bytes([2, 0, 0, 0])                      # version 2, scalar
    nm = name.encode() + b"\0"
    return 0x0C, (bytes([3, 0]) + struct.pack("<HHH", len(nm), len(dt), len(ds)) + b"\0" +
                  nm + dt + ds + text.encode())


def _build_spec_file(path, a, chunk, b):
    """Superblock v2; root group of link messages holding a chunked
    big-endian int dataset /grid/a (shuffle + deflate, one chunk stored with
    deflate skipped by its filter mask) and a compact double dataset /b."""
    out = bytearray(48)                           # superblock, patched below

    def put(blob):
        while len(out) % 8:
            out.append(0)
        at = len(out)
        out.extend(blob)
        return at

    rows, cols = a.shape
    cr, cc = chunk
    keys, kids = [], []
    n = 0
    for r0 in range(0, rows, cr):
        for c0 in range(0, cols, cc):
            blk = np.zeros((cr, cc), dtype=">i4")
            sub = a[r0:r0 + cr, c0:c0 + cc]
            blk[:sub.shape[0], :sub.shape[1]] = sub
            raw = blk.tobytes()
            shuffled = bytes(np.frombuffer(raw, np.uint8).reshape(-1, 4).T.ravel())
            mask = 2 if n == 1 else 0             # the second chunk skips deflate
            data = shuffled if mask else zlib.compress(shuffled, 6)
            kids.append(put(data))
            keys.append(struct.pack("<II3Q", len(data), mask, r0, c0, 0))
            n += 1
    final = struct.pack("<II3Q", 0, 0, rows, cols, 0)
    tree = b"TREE" + bytes([1, 0]) + struct.pack("<HQQ", n, UNDEF, UNDEF)
    for k, c in zip(keys, kids):
        tree += k + struct.pack("<Q", c)
    tree += final
    bt = put(tree)
    layout = 8, bytes([3, 2, 3]) + struct.pack("<Q", bt) + struct.pack("<III", cr, cc, 4)
    pline = 0x0B, (bytes([2, 2]) + struct.pack("<HHHI", 2, 0, 1, 4) +
                   struct.pack("<HHHI", 1, 0, 1, 6))
    a_oh = put(_ohdr_v2([_space_v2([rows, cols]), _int32_be(), layout, pline,
                         _attr_v3("type", "int")]))
    bvals = np.asarray(b, dtype="<f8")
    compact = 8, bytes([3, 0]) + struct.pack("<H", bvals.nbytes) + bvals.tobytes()
    b_oh = put(_ohdr_v2([_space_v2([len(bvals)]), _f64_le(), compact]))
    linfo = 2, bytes([0, 0]) + struct.pack("<QQ", UNDEF, UNDEF)
    grid = put(_ohdr_v2([linfo, _link("a", a_oh)]))
    root = put(_ohdr_v2([linfo, _link("grid", grid), _link("b", b_oh)]))
    sb = (bytes([0x89, 0x48, 0x44, 0x46, 0x0D, 0x0A, 0x1A, 0x0A, 2, 8, 8, 0]) +
          struct.pack("<QQQQ", 0, UNDEF, len(out), root) + b"\0\0\0\0")
    out[:48] = sb
    with open(path, "wb") as fh:
        fh.write(bytes(out))


def test_reader_paths_the_writer_does_not_produce(tmp_path):
    f = str(tmp_path / "spec.h5")
    a = np.arange(7 * 5, dtype=np.int32).reshape(7, 5) * 37 - 500
    b = [0.25, -1.0, 3.5]
    _build_spec_file(f, a, (3, 2), b)
    assert L.h5_list(f) == ["/grid/", "/grid/a", "/b"]
    assert L.h5_info(f, "/grid/a") == ((7, 5), "UNRECOGNISED")     # big-endian
    np.testing.assert_array_equal(L.h5_read(f, "/grid/a", "int"), a)
    np.testing.assert_array_equal(L.h5_read(f, "/grid/a", "double"), a.astype(np.float64))
    assert L.h5_get_attr(f, "/grid/a", "type") == "int"
    np.testing.assert_array_equal(L.h5_read(f, "b"), b)
    # rewritten by the writer: same values, now in its own layout
    L.h5_write(f, "/c", np.array([1, 2], dtype=np.int32))
    np.testing.assert_array_equal(L.h5_read(f, "/grid/a", "int"), a)
    assert L.h5_info(f, "/grid/a") == ((7, 5), "UNRECOGNISED")
    np.testing.assert_array_equal(L.h5_read(f, "b"), b)


def test_corrupt_sizes_are_errors_not_allocations(tmp_path):
    """A file whose structures claim more bytes than it holds (here the root
    object header's size, and a truncated copy) is refused with a message;
    the reader never allocates what the file merely claims."""
    f = str(tmp_path / "ok.h5")
    L.h5_write(f, "x", np.arange(10.0))
    raw = bytearray(open(f, "rb").read())
    root_oh = struct.unpack_from("<Q", raw, 64)[0]      # root symbol table entry
    bad = bytearray(raw)
    struct.pack_into("<I", bad, root_oh + 8, 0xFFFFFFF0)   # object header size
    g = str(tmp_path / "bad.h5")
    open(g, "wb").write(bytes(bad))
    with pytest.raises(L.Op2Error, match="beyond its end"):
        L.h5_list(g)
    t = str(tmp_path / "short.h5")
    open(t, "wb").write(bytes(raw[:len(raw) - 40]))          # the data cut short
    with pytest.raises(L.Op2Error):
        L.h5_read(t, "x")
