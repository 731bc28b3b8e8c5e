"""HDF5 container files written and read without libhdf5 (cn_h5_write /
cn_h5_query / cn_h5_read, host code, no GPU).

The reader is pinned to a file that libhdf5 wrote: scipy ships a MATLAB 7.3
test file (an HDF5 file after a 512-byte user block) whose dataset
"testdouble" holds k * pi / 4, k = 0..8.  The writer's files are walked here
by a checker of the structures libhdf5 decodes (superblock version 0, the
root group's symbol table, local heap and its free list, group and chunk
B-tree node sizes, version 1 object headers), and its datatype and
dataspace messages are compared byte for byte with those libhdf5 wrote into
that file.  Round trips cover both layouts, all three types, hyperslab reads,
conversions and the error paths."""
import ctypes as C
import math
import os
import struct

import numpy as np
import pytest

from cubismnova_b200 import _lib
from cubismnova_b200 import io as IO

CN_ERR_INVALID_ARGUMENT, CN_ERR_SIZE_MISMATCH, CN_ERR_UNSUPPORTED, CN_ERR_FILE = 1, 7, 12, 14
UNDEF = 2**64 - 1


def _libhdf5_file():
    import scipy.io.matlab as M
    p = os.path.join(os.path.dirname(M.__file__), "tests", "data", "testhdf5_7.4_GLNX86.mat")
    if not os.path.exists(p):
        pytest.skip("scipy's libhdf5-written test file is not installed")
    return p


# ------------------------------------------------------------ file walker

def _u(b, off, n):
    return int.from_bytes(b[off:off + n], "little")


def _ohdr_v1(b, base, addr):
    """Messages (type, flags, body) of a version 1 object header; checks the
    prefix, the 8-byte alignment of message sizes and the message count."""
    p = base + addr
    assert b[p] == 1 and b[p + 1] == 0
    nmsgs, refc, size = _u(b, p + 2, 2), _u(b, p + 4, 4), _u(b, p + 8, 4)
    assert refc >= 1
    out, blocks = [], [(p + 16, size)]
    while blocks:
        q, n = blocks.pop(0)
        end = q + n
        while q < end:
            t, s, fl = _u(b, q, 2), _u(b, q + 2, 2), b[q + 4]
            assert s % 8 == 0 and q + 8 + s <= end
            body = b[q + 8:q + 8 + s]
            if t == 0x10:
                blocks.append((base + _u(body, 0, 8), _u(body, 8, 8)))
            out.append((t, fl, body))
            q += 8 + s
    assert len(out) == nmsgs
    return out


def walk(path):
    """The structure of a one-dataset file as libhdf5 decodes it; returns
    the dataset's messages {type: body} and the node extents found."""
    b = open(path, "rb").read()
    base = b.find(b"\x89HDF\r\n\x1a\n")
    assert base in (0, 512, 1024, 2048)
    assert b[base + 8] == 0 and b[base + 13] == 8 and b[base + 14] == 8  # superblock 0, 8-byte offsets/lengths
    leaf_k, int_k = _u(b, base + 16, 2), _u(b, base + 18, 2)
    sb_base, fs, eof, drv = struct.unpack_from("<QQQQ", b, base + 24)
    assert sb_base == base and fs == UNDEF and drv == UNDEF
    # the stored end of file counts from the file's first byte (user block included)
    assert eof <= len(b), "libhdf5 refuses a file shorter than its stored end-of-file address"
    name_off, root_oh, cache = struct.unpack_from("<QQI", b, base + 56)
    c_tree, c_heap = struct.unpack_from("<QQ", b, base + 56 + 24)
    stab = [m for m in _ohdr_v1(b, base, root_oh) if m[0] == 0x11]
    assert len(stab) == 1
    tree, heap = struct.unpack_from("<QQ", stab[0][2], 0)
    if cache == 1:
        assert (c_tree, c_heap) == (tree, heap)
    # local heap: header, data segment, free list ending in 1 (libhdf5's end mark)
    h = base + heap
    assert b[h:h + 4] == b"HEAP" and b[h + 4] == 0
    dsize, free, daddr = struct.unpack_from("<QQQ", b, h + 8)
    seg = b[base + daddr:base + daddr + dsize]
    assert len(seg) == dsize and seg[0] == 0  # "" at offset 0
    while free != 1:
        assert free < dsize
        nxt, fsz = struct.unpack_from("<QQ", seg, free)
        assert fsz >= 16 and free + fsz <= dsize
        free = nxt
    # group B-tree leaf: allocated for 2K children and 2K + 1 keys
    t = base + tree
    assert b[t:t + 4] == b"TREE" and b[t + 4] == 0 and b[t + 5] == 0
    used = _u(b, t + 6, 2)
    assert used == 1
    k0, child, k1 = struct.unpack_from("<QQQ", b, t + 24)
    node_bytes = 24 + 2 * int_k * 8 + (2 * int_k + 1) * 8
    s = base + child
    assert b[s:s + 4] == b"SNOD" and b[s + 4] == 1
    nsym = _u(b, s + 6, 2)
    snod_bytes = 8 + 2 * leaf_k * 40
    assert not (t < s < t + node_bytes), "the symbol-table node overlaps the B-tree node's allocation"
    entries = {}
    for i in range(nsym):
        lno, oh = struct.unpack_from("<QQ", b, s + 8 + 40 * i)
        nm = seg[lno:seg.index(b"\0", lno)].decode()
        entries[nm] = oh
    assert seg[k1:seg.index(b"\0", k1)].decode() == max(entries)
    return b, base, entries, dict(node_bytes=node_bytes, snod_bytes=snod_bytes, tree=tree, snod=child)


def _messages(path, name):
    b, base, entries, _ = walk(path)
    return {t: body for t, fl, body in _ohdr_v1(b, base, entries[name])}


# ------------------------------------------------------------------ tests

def test_reader_pinned_to_a_libhdf5_file():
    p = _libhdf5_file()
    shape, dt = IO.h5_query(p, "testdouble")
    assert shape == (9, 1) and dt == np.float64
    a = IO.h5_read(p, "testdouble")
    assert np.array_equal(a.ravel(), np.arange(9) * (math.pi / 4))
    assert np.array_equal(IO.h5_read(p, "/testdouble", count=(4, 1), dtype=np.float32).ravel(),
                          (np.arange(4) * (math.pi / 4)).astype(np.float32))
    walk(p)  # the walker accepts libhdf5's own structure


def test_datatype_and_dataspace_messages_match_libhdf5(tmp_path):
    ref = _messages(_libhdf5_file(), "testdouble")
    x = np.arange(9, dtype=np.float64).reshape(9, 1)
    IO.h5_write(str(tmp_path / "d.h5"), x, dataset="testdouble")
    ours = _messages(str(tmp_path / "d.h5"), "testdouble")
    # H5T_IEEE_F64LE as libhdf5 encodes it (version 1, 20 bytes + padding)
    assert ours[0x0003][:20] == ref[0x0003][:20]
    # simple dataspace, version 1, no maximum dims
    assert ours[0x0001] == ref[0x0001]


@pytest.mark.parametrize("chunked", [False, True])
@pytest.mark.parametrize("dtype", [np.float64, np.float32, np.int32])
def test_round_trip_and_structure(tmp_path, chunked, dtype):
    rng = np.random.default_rng(int(chunked) * 3 + [np.float64, np.float32, np.int32].index(dtype))
    for rank in (1, 2, 4, 5):
        shape = tuple(int(v) for v in rng.integers(1, 7, size=rank))
        x = (rng.standard_normal(shape) * 1e4).astype(dtype)
        p = str(tmp_path / f"f{rank}.h5")
        IO.h5_write(p, x, chunked=chunked)
        assert os.path.getsize(p) == struct.unpack_from("<Q", open(p, "rb").read(), 40)[0]
        msgs = _messages(p, "data")
        layout = msgs[0x0008]
        assert layout[0] == 3 and layout[1] == (2 if chunked else 1)
        if chunked:
            # chunk dims = dataset dims, then the element size; one leaf entry
            nd = layout[2]
            assert nd == rank + 1
            dims = struct.unpack_from(f"<{nd}I", layout, 11)
            assert dims == shape + (x.itemsize,)
            b = open(p, "rb").read()
            t = _u(layout, 3, 8)
            assert b[t:t + 4] == b"TREE" and b[t + 4] == 1 and _u(b, t + 6, 2) == 1
            key = 8 + 8 * nd
            assert _u(b, t + 24, 4) == x.nbytes and _u(b, t + 28, 4) == 0
            right = struct.unpack_from(f"<{nd}Q", b, t + 24 + key + 8 + 8)
            assert right == shape + (0,)
            assert t + 24 + 64 * 8 + 65 * key <= _u(b, t + 24 + key, 8)  # chunk after the node's allocation
        else:
            assert _u(layout, 10, 8) == x.nbytes
        y = IO.h5_read(p)
        assert y.dtype == x.dtype and np.array_equal(y, x)
        cnt = tuple(int(rng.integers(1, s + 1)) for s in shape)
        assert np.array_equal(IO.h5_read(p, count=cnt), x[tuple(slice(0, c) for c in cnt)])
        if dtype != np.int32:
            other = np.float32 if dtype == np.float64 else np.float64
            assert np.array_equal(IO.h5_read(p, dtype=other), x.astype(other))
        else:
            assert np.array_equal(IO.h5_read(p, dtype=np.float64), x.astype(np.float64))


def test_names_and_empty_dataset(tmp_path):
    p = str(tmp_path / "e.h5")
    IO.h5_write(p, np.zeros((0, 3), np.float64), dataset="a_long_dataset_name_of_40_characters_xyz")
    assert IO.h5_query(p, "a_long_dataset_name_of_40_characters_xyz") == ((0, 3), np.float64)
    assert IO.h5_read(p, "a_long_dataset_name_of_40_characters_xyz").shape == (0, 3)
    walk(p)


def test_errors(tmp_path):
    lib = _lib.lib()
    p = str(tmp_path / "x.h5")
    IO.h5_write(p, np.ones((4, 4), np.float32))
    with pytest.raises(_lib.CnError) as e:
        IO.h5_read(str(tmp_path / "missing.h5"))
    assert e.value.status == CN_ERR_FILE
    with pytest.raises(_lib.CnError) as e:
        IO.h5_read(p, "other")
    assert e.value.status == CN_ERR_FILE and "no dataset 'other'" in str(e.value)
    with pytest.raises(_lib.CnError) as e:
        IO.h5_read(p, count=(5, 4))
    assert e.value.status == CN_ERR_SIZE_MISMATCH
    with pytest.raises(_lib.CnError) as e:  # floats are not converted to integers
        IO.h5_read(p, dtype=np.int32)
    assert e.value.status == CN_ERR_UNSUPPORTED
    junk = str(tmp_path / "junk.h5")
    open(junk, "wb").write(b"\0" * 4096)
    with pytest.raises(_lib.CnError) as e:
        IO.h5_query(junk)
    assert e.value.status == CN_ERR_FILE and "no HDF5 superblock" in str(e.value)
    dims = (C.c_longlong * 2)(2, 2)
    assert lib.cn_h5_write(p.encode(), b"a/b", 2, dims, 0, None, 0) == CN_ERR_INVALID_ARGUMENT
    assert lib.cn_h5_write(p.encode(), b"d", 2, dims, 0, None, 0) == CN_ERR_INVALID_ARGUMENT  # data NULL
    # one chunk must stay under 4 GiB (the writer says so before touching data)
    big = (C.c_longlong * 2)(2**20, 2**10)
    assert lib.cn_h5_write(p.encode(), b"d", 2, big, 1, C.c_void_p(1), 1) == CN_ERR_UNSUPPORTED
    # a truncated file: the data beyond the end
    b = open(p, "rb").read()
    t = str(tmp_path / "t.h5")
    open(t, "wb").write(b[:-8])
    with pytest.raises(_lib.CnError) as e:
        IO.h5_read(t)
    assert e.value.status == CN_ERR_FILE
