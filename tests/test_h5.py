"""The HDF5 subset of the data I/O (no GPU): the metadata checksum against the
published lookup3 vectors, the C++ writer read back by an independently
written Python reader, and the C++ reader on files built here with the
optional header fields an HDF5 library may write.
"""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np
import pytest

from h5read import SIGNATURE, H5File, lookup3


def _lib():
    from powerllel_channel_sycl_b200._lib import lib
    return lib()


# lookup3.c's driver prints these for hashlittle (Jenkins, 2006)
LOOKUP3_VECTORS = [
    (b"", 0, 0xDEADBEEF),
    (b"Four score and seven years ago", 0, 0x17770551),
    (b"Four score and seven years ago", 1, 0xCD628161),
]


@pytest.mark.parametrize("data,init,expect", LOOKUP3_VECTORS)
def test_lookup3_vectors(data, init, expect):
    assert lookup3(data, init) == expect
    buf = C.create_string_buffer(data, len(data))
    assert _lib().plc_h5_lookup3(buf, len(data), init) == expect


def test_lookup3_c_matches_python_all_tails():
    rng = np.random.default_rng(3)
    for n in list(range(0, 40)) + [255, 1000]:
        d = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        buf = C.create_string_buffer(d, len(d))
        assert _lib().plc_h5_lookup3(buf, n, 7) == lookup3(d, 7), n


def write(path, sets):
    """sets: list of (name, ndarray f64 or i32)."""
    L = _lib()
    n = len(sets)
    names = (C.c_char_p * n)(*[s[0].encode() for s in sets])
    types = (C.c_int * n)(*[0 if s[1].dtype == np.float64 else 1 for s in sets])
    ndims = (C.c_int * n)(*[s[1].ndim for s in sets])
    dims = [d for s in sets for d in s[1].shape]
    dims_c = (C.c_longlong * len(dims))(*dims)
    arrs = [np.ascontiguousarray(s[1]) for s in sets]
    data = (C.c_void_p * n)(*[a.ctypes.data for a in arrs])
    rc = L.plc_h5_write(str(path).encode(), n, names, types, ndims, dims_c, data)
    assert rc == 0, L.plc_last_error(None)


def read(path, name):
    L = _lib()
    nd = C.c_int(8)
    dims = (C.c_longlong * 8)()
    rc = L.plc_h5_read(str(path).encode(), name.encode(), None, 0, dims, C.byref(nd))
    if rc != 0:
        return rc, L.plc_last_error(None).decode()
    shape = tuple(dims[:nd.value])
    out = np.empty(shape)
    rc = L.plc_h5_read(str(path).encode(), name.encode(), out.ctypes.data, out.size, dims,
                       C.byref(C.c_int(8)))
    assert rc == 0
    return 0, out


def test_field_file_layout(tmp_path):
    """outputField's file: [nz][ny][nx] f64 dataset plus the 1-element int "nt"."""
    rng = np.random.default_rng(0)
    u = rng.standard_normal((6, 5, 4))
    p = tmp_path / "inst_00000010_u.h5"
    write(p, [("nt", np.array([10], np.int32)), ("u", u)])
    f = H5File(p)
    assert f.superblock_version == 2
    assert f.names() == ["nt", "u"]
    got = f.dataset("u")
    assert got.dtype == np.float64 and got.shape == (6, 5, 4)
    assert np.array_equal(got, u)
    nt = f.dataset("nt")
    assert nt.dtype == np.int32 and nt.shape == (1,) and nt[0] == 10
    # the C reader gives the same
    rc, back = read(p, "u")
    assert rc == 0 and np.array_equal(back, u)
    rc, back = read(p, "nt")
    assert rc == 0 and back.tolist() == [10.0]


def test_special_values_and_sizes(tmp_path):
    vals = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, 1.7976931348623157e308, 1.0 / 3])
    big = np.arange(70000, dtype=np.float64).reshape(7, 100, 100)  # chunk-size field of 4 bytes
    empty = np.zeros((0, 3))
    many = [(f"s{q:03d}", np.array([q], np.int32)) for q in range(300)]  # a root header over 255 B
    p = tmp_path / "a.h5"
    write(p, [("vals", vals), ("big", big), ("empty", empty)] + many)
    f = H5File(p)
    assert np.array_equal(f.dataset("vals").view(np.uint64), vals.view(np.uint64))
    assert np.array_equal(f.dataset("big"), big)
    assert f.dataset("empty").shape == (0, 3)
    assert all(f.dataset(n)[0] == v[0] for n, v in many)
    rc, back = read(p, "vals")
    assert rc == 0 and np.array_equal(back.view(np.uint64), vals.view(np.uint64))
    rc, back = read(p, "s299")
    assert rc == 0 and back[0] == 299


def test_reader_errors(tmp_path):
    p = tmp_path / "b.h5"
    write(p, [("x", np.ones(3))])
    rc, msg = read(p, "y")
    assert rc == -6 and "no dataset 'y'" in msg
    rc, msg = read(tmp_path / "missing.h5", "x")
    assert rc == -6 and "doesn't exist" in msg
    raw = bytearray(p.read_bytes())
    raw[60] ^= 0x01  # inside the root group's object header
    q = tmp_path / "c.h5"
    q.write_bytes(bytes(raw))
    rc, msg = read(q, "x")
    assert rc == -6 and "checksum" in msg
    raw = bytearray(p.read_bytes())
    raw[20] ^= 0x01  # superblock
    q.write_bytes(bytes(raw))
    rc, msg = read(q, "x")
    assert rc == -6 and "superblock checksum" in msg
    q.write_bytes(b"not hdf5" * 10)
    rc, msg = read(q, "x")
    assert rc == -6 and "not an HDF5 file" in msg


# ---- files with the optional fields another writer may use --------------------
def _ohdr(msgs, times=False, width_flag=None, creation_order_tracked=False):
    body = b""
    for mtype, payload, order in msgs:
        body += struct.pack("<BHB", mtype, len(payload), 0)
        if creation_order_tracked:
            body += struct.pack("<H", order)
        body += payload
    if width_flag is None:
        width_flag = 0 if len(body) < 256 else 1
    flags = width_flag | (0x20 if times else 0) | (0x04 if creation_order_tracked else 0)
    h = b"OHDR" + bytes([2, flags])
    if times:
        h += struct.pack("<IIII", 1, 2, 3, 4)
    h += len(body).to_bytes(1 << width_flag, "little") + body
    return h + struct.pack("<I", lookup3(h))


def _build_file(path, arr, name="u", times=True, link_creation_order=True, dataspace_v1=True):
    """A root group with one f64 dataset, laid out by hand: superblock 3,
    object headers with times, tracked message creation order and a 2-byte
    chunk size, a link message carrying a creation order and a 2-byte name
    length, a version-1 dataspace with maximum dimensions."""
    shape = arr.shape
    if dataspace_v1:
        ds = bytes([1, len(shape), 1, 0]) + b"\0" * 4 + b"".join(struct.pack("<Q", d) for d in shape)
        ds += b"".join(struct.pack("<Q", d) for d in shape)  # maximum dimensions
    else:
        ds = bytes([2, len(shape), 0, 1]) + b"".join(struct.pack("<Q", d) for d in shape)
    dt = bytes([0x11, 0x20, 63, 0]) + struct.pack("<I", 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
    fill = bytes([3, 0x09])
    data_addr_placeholder = 0

    def dset_header(addr):
        lay = bytes([3, 1]) + struct.pack("<QQ", addr, arr.nbytes)
        return _ohdr([(0x01, ds, 0), (0x03, dt, 1), (0x05, fill, 2), (0x08, lay, 3)],
                     times=times, width_flag=1, creation_order_tracked=True)

    def root_header(dset_addr):
        nm = name.encode()
        if link_creation_order:
            link = bytes([1, 0x04 | 0x01]) + struct.pack("<Q", 0) + struct.pack("<H", len(nm)) + nm
        else:
            link = bytes([1, 0]) + bytes([len(nm)]) + nm
        link += struct.pack("<Q", dset_addr)
        linfo = bytes([0, 0]) + b"\xff" * 16
        ginfo = bytes([0, 0])
        return _ohdr([(0x02, linfo, 0), (0x0A, ginfo, 1), (0x06, link, 2)], times=times,
                     width_flag=1, creation_order_tracked=True)

    root_len = len(root_header(0))
    dset_addr = 48 + root_len
    dset_len = len(dset_header(data_addr_placeholder))
    data_addr = dset_addr + dset_len
    eof = data_addr + arr.nbytes
    sb = SIGNATURE + bytes([3, 8, 8, 0]) + struct.pack("<QQQQ", 0, 0xFFFFFFFFFFFFFFFF, eof, 48)
    sb += struct.pack("<I", lookup3(sb))
    out = sb + root_header(dset_addr) + dset_header(data_addr) + arr.astype("<f8").tobytes()
    assert len(out) == eof
    path.write_bytes(out)


@pytest.mark.parametrize("times,order,v1", [(True, True, True), (False, False, False),
                                            (True, False, True)])
def test_c_reader_optional_fields(tmp_path, times, order, v1):
    arr = np.random.default_rng(1).standard_normal((3, 4, 5))
    p = tmp_path / "x.h5"
    _build_file(p, arr, times=times, link_creation_order=order, dataspace_v1=v1)
    assert np.array_equal(H5File(p).dataset("u"), arr)  # the hand-built file is well formed
    rc, back = read(p, "u")
    assert rc == 0, back
    assert np.array_equal(back, arr)


# ---- the library's default format: superblock 0, symbol-table groups ---------
UNDEF = 0xFFFFFFFFFFFFFFFF


def _pad8(b):
    return b + b"\0" * (-len(b) % 8)


def _v1_msg(mtype, payload):
    payload = _pad8(payload)
    return struct.pack("<HHB3x", mtype, len(payload), 0) + payload


def _v1_header(msgs_bytes, nmsgs):
    return struct.pack("<BBHII4x", 1, 0, nmsgs, 1, len(msgs_bytes)) + msgs_bytes


def _entry(name_off, addr, cache=0, scratch=b"\0" * 16):
    return struct.pack("<QQI4x", name_off, addr, cache) + scratch


def build_v0_file(path, sets, superblock=0, two_level=False):
    """A file in the layout an HDF5 library writes with default properties:
    superblock 0 (or 1), version-1 object headers, the root group as a symbol
    table (local heap, version-1 B-tree, symbol nodes), dataspace version 1,
    fill value version 2, and the layout message in a continuation block."""
    buf = bytearray()

    def alloc(n):
        a = len(buf)
        buf.extend(b"\0" * n)
        return a

    sb_len = (56 if superblock == 0 else 60) + 40
    alloc(sb_len)
    names = sorted(s[0] for s in sets)
    # local heap: "" at 0, then each name, 8-byte aligned
    heap_data = bytearray(b"\0" * 8)
    offs = {}
    for n in names:
        offs[n] = len(heap_data)
        heap_data += _pad8(n.encode() + b"\0")
    heap_seg = alloc(len(heap_data))
    buf[heap_seg:heap_seg + len(heap_data)] = heap_data
    heap = alloc(32)
    buf[heap:heap + 32] = b"HEAP" + bytes([0, 0, 0, 0]) + struct.pack("<QQQ", len(heap_data), UNDEF, heap_seg)
    # datasets
    hdr_addr = {}
    for name, arr in sets:
        arr = np.ascontiguousarray(arr)
        data = alloc(arr.nbytes)
        buf[data:data + arr.nbytes] = arr.tobytes()
        ds = bytes([1, arr.ndim, 0, 0, 0, 0, 0, 0]) + b"".join(struct.pack("<Q", d) for d in arr.shape)
        if arr.dtype == np.float64:
            dt = bytes([0x11, 0x20, 63, 0]) + struct.pack("<I", 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
        else:
            dt = bytes([0x10, 0x08, 0, 0]) + struct.pack("<I", 4) + struct.pack("<HH", 0, 32)
        fill = bytes([2, 1, 2, 0])
        lay = bytes([3, 1]) + struct.pack("<QQ", data, arr.nbytes)
        cont_block = _v1_msg(0x08, lay)
        cont = alloc(len(cont_block))
        buf[cont:cont + len(cont_block)] = cont_block
        msgs = (_v1_msg(0x01, ds) + _v1_msg(0x03, dt) + _v1_msg(0x05, fill)
                + _v1_msg(0x10, struct.pack("<QQ", cont, len(cont_block))))
        h = _v1_header(msgs, 5)
        a = alloc(len(h))
        buf[a:a + len(h)] = h
        hdr_addr[name] = a
    # symbol nodes (one per name in the two-level case) and B-tree nodes
    def snod(group):
        body = b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(group))
        body += b"".join(_entry(offs[n], hdr_addr[n]) for n in group)
        body += b"\0" * (40 * (8 - len(group)))  # unused entries of a node of 2K = 8
        a = alloc(len(body))
        buf[a:a + len(body)] = body
        return a

    def tree(level, keys, children):
        body = b"TREE" + bytes([0, level]) + struct.pack("<HQQ", len(children), UNDEF, UNDEF)
        for k, c in zip(keys, children):
            body += struct.pack("<QQ", k, c)
        body += struct.pack("<Q", keys[-1])
        a = alloc(len(body))
        buf[a:a + len(body)] = body
        return a

    if two_level:
        leaves = [tree(0, [0, offs[n]], [snod([n])]) for n in names]
        root_tree = tree(1, [0] + [offs[n] for n in names], leaves)
    else:
        root_tree = tree(0, [0, offs[names[-1]]], [snod(names)])
    rh = _v1_header(_v1_msg(0x11, struct.pack("<QQ", root_tree, heap)), 1)
    root = alloc(len(rh))
    buf[root:root + len(rh)] = rh
    sb = SIGNATURE + bytes([superblock, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", 4, 16, 0)
    if superblock == 1:
        sb += struct.pack("<HH", 32, 0)
    sb += struct.pack("<QQQQ", 0, UNDEF, len(buf), UNDEF)
    sb += _entry(0, root, 1, struct.pack("<QQ", root_tree, heap))
    assert len(sb) == sb_len
    buf[0:sb_len] = sb
    path.write_bytes(bytes(buf))


@pytest.mark.parametrize("superblock,two_level", [(0, False), (1, False), (0, True)])
def test_c_reader_default_library_format(tmp_path, superblock, two_level):
    """A checkpoint in the format the reference's libhdf5 writes by default."""
    u = np.random.default_rng(2).standard_normal((4, 3, 5))
    p = tmp_path / "save_u.h5"
    build_v0_file(p, [("nt", np.array([1234], np.int32)), ("u", u)], superblock, two_level)
    rc, back = read(p, "u")
    assert rc == 0, back
    assert np.array_equal(back, u)
    rc, back = read(p, "nt")
    assert rc == 0 and back.tolist() == [1234.0]
    rc, msg = read(p, "v")
    assert rc == -6 and "no dataset 'v'" in msg


@pytest.mark.parametrize("fmt", ["latest", "default"])
def test_c_reader_survives_damaged_files(tmp_path, fmt):
    """Truncated or corrupted files give PLC_ERR_IO (or, where the damage is
    harmless, the data), never a crash or an out-of-file read."""
    u = np.arange(24, dtype=np.float64).reshape(2, 3, 4)
    p = tmp_path / "ok.h5"
    if fmt == "latest":
        write(p, [("nt", np.array([7], np.int32)), ("u", u)])
    else:
        build_v0_file(p, [("nt", np.array([7], np.int32)), ("u", u)])
    good = p.read_bytes()
    rng = np.random.default_rng(11)
    q = tmp_path / "bad.h5"
    cases = [good[:n] for n in rng.integers(0, len(good), 40)]
    for _ in range(300):
        b = bytearray(good)
        for pos in rng.integers(0, len(good), rng.integers(1, 4)):
            b[pos] = int(rng.integers(0, 256))
        cases.append(bytes(b))
    for data in cases:
        q.write_bytes(data)
        for name in ("u", "nt"):
            rc, _ = read(q, name)
            assert rc in (0, -6)
