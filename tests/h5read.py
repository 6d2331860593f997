"""A small HDF5 reader for the tests, written separately from the library's C++
reader from the HDF5 File Format Specification 3.0: superblock version 2/3,
version-2 object headers, a compact root group of Link messages, version-1/2
dataspaces, fixed-point and IEEE floating-point datatypes, contiguous layout.
Every metadata checksum (Jenkins lookup3) is verified.
"""
from __future__ import annotations

import struct

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"


def _rot(x, k):
    return ((x << k) | (x >> (32 - k))) & 0xFFFFFFFF


def lookup3(data: bytes, initval: int = 0) -> int:
    """Bob Jenkins' hashlittle (lookup3.c, 2006), the HDF5 metadata checksum."""
    m = 0xFFFFFFFF
    n = len(data)
    a = b = c = (0xDEADBEEF + n + initval) & m
    k = 0
    while n > 12:
        a = (a + int.from_bytes(data[k:k + 4], "little")) & m
        b = (b + int.from_bytes(data[k + 4:k + 8], "little")) & m
        c = (c + int.from_bytes(data[k + 8:k + 12], "little")) & m
        a = (a - c) & m; a ^= _rot(c, 4); c = (c + b) & m
        b = (b - a) & m; b ^= _rot(a, 6); a = (a + c) & m
        c = (c - b) & m; c ^= _rot(b, 8); b = (b + a) & m
        a = (a - c) & m; a ^= _rot(c, 16); c = (c + b) & m
        b = (b - a) & m; b ^= _rot(a, 19); a = (a + c) & m
        c = (c - b) & m; c ^= _rot(b, 4); b = (b + a) & m
        n -= 12
        k += 12
    if n == 0:
        return c
    tail = data[k:k + n] + b"\x00" * (12 - n)
    a = (a + int.from_bytes(tail[0:4], "little")) & m
    b = (b + int.from_bytes(tail[4:8], "little")) & m
    c = (c + int.from_bytes(tail[8:12], "little")) & m
    c ^= b; c = (c - _rot(b, 14)) & m
    a ^= c; a = (a - _rot(c, 11)) & m
    b ^= a; b = (b - _rot(a, 25)) & m
    c ^= b; c = (c - _rot(b, 16)) & m
    a ^= c; a = (a - _rot(c, 4)) & m
    b ^= a; b = (b - _rot(a, 14)) & m
    c ^= b; c = (c - _rot(b, 24)) & m
    return c


class H5File:
    """Root-group datasets of a file in the subset above."""

    def __init__(self, path):
        with open(path, "rb") as f:
            self.buf = f.read()
        b = self.buf
        if b[:8] != SIGNATURE:
            raise ValueError("not an HDF5 file")
        self.superblock_version = b[8]
        if b[8] not in (2, 3):
            raise ValueError(f"superblock version {b[8]}")
        if b[9] != 8 or b[10] != 8:
            raise ValueError("offset/length size")
        (chk,) = struct.unpack_from("<I", b, 44)
        if lookup3(b[:44]) != chk:
            raise ValueError("superblock checksum")
        base, ext, self.eof, root = struct.unpack_from("<QQQQ", b, 12)
        if base != 0 or ext != 0xFFFFFFFFFFFFFFFF:
            raise ValueError("base address / superblock extension")
        if self.eof != len(b):
            raise ValueError(f"end-of-file address {self.eof} != file size {len(b)}")
        self.links = {}
        for mtype, off, size in self._messages(root):
            if mtype == 0x06:
                name, addr = self._link(off)
                self.links[name] = addr

    def _messages(self, addr):
        b = self.buf
        if b[addr:addr + 4] != b"OHDR" or b[addr + 4] != 2:
            raise ValueError("object header")
        flags = b[addr + 5]
        p = addr + 6
        if flags & 0x20:
            p += 16
        if flags & 0x10:
            p += 4
        width = 1 << (flags & 3)
        chunk = int.from_bytes(b[p:p + width], "little")
        p += width
        end = p + chunk
        (chk,) = struct.unpack_from("<I", b, end)
        if lookup3(b[addr:end]) != chk:
            raise ValueError("object header checksum")
        out = []
        hdr = 6 if flags & 0x04 else 4
        while p + hdr <= end:
            mtype = b[p]
            (size,) = struct.unpack_from("<H", b, p + 1)
            p += hdr
            out.append((mtype, p, size))
            p += size
        if p != end:
            raise ValueError("messages do not fill the chunk")
        return out

    def _link(self, off):
        b = self.buf
        if b[off] != 1:
            raise ValueError("link message version")
        flags = b[off + 1]
        p = off + 2
        ltype = 0
        if flags & 0x08:
            ltype = b[p]
            p += 1
        if flags & 0x04:
            p += 8
        if flags & 0x10:
            p += 1
        w = 1 << (flags & 3)
        n = int.from_bytes(b[p:p + w], "little")
        p += w
        name = b[p:p + n].decode()
        p += n
        if ltype != 0:
            raise ValueError("only hard links")
        (addr,) = struct.unpack_from("<Q", b, p)
        return name, addr

    def names(self):
        return sorted(self.links)

    def dataset(self, name) -> np.ndarray:
        b = self.buf
        shape = dtype = data = None
        for mtype, off, size in self._messages(self.links[name]):
            if mtype == 0x01:
                ver, nd = b[off], b[off + 1]
                d0 = off + (8 if ver == 1 else 4)
                shape = struct.unpack_from("<" + "Q" * nd, b, d0)
            elif mtype == 0x03:
                cls, ver = b[off] & 0x0F, b[off] >> 4
                if ver != 1:
                    raise ValueError("datatype version")
                bits0 = b[off + 1]
                (esize,) = struct.unpack_from("<I", b, off + 4)
                if bits0 & 1:
                    raise ValueError("big endian")
                if cls == 1:
                    (boff, prec) = struct.unpack_from("<HH", b, off + 8)
                    eloc, esz, mloc, msz = b[off + 12:off + 16]
                    (bias,) = struct.unpack_from("<I", b, off + 16)
                    if esize == 8:
                        assert (prec, eloc, esz, mloc, msz, bias) == (64, 52, 11, 0, 52, 1023)
                        assert b[off + 2] == 63  # sign bit location
                    dtype = {8: "<f8", 4: "<f4"}[esize]
                elif cls == 0:
                    signed = bool(bits0 & 0x08)
                    dtype = ("<i" if signed else "<u") + str(esize)
                else:
                    raise ValueError(f"datatype class {cls}")
            elif mtype == 0x08:
                if b[off] != 3 or b[off + 1] != 1:
                    raise ValueError("layout")
                addr, nbytes = struct.unpack_from("<QQ", b, off + 2)
                data = (addr, nbytes)
        n = int(np.prod(shape)) if shape else 1
        addr, nbytes = data
        item = np.dtype(dtype).itemsize
        if nbytes != n * item or addr + nbytes > len(b):
            raise ValueError("data extent")
        return np.frombuffer(b, dtype=dtype, count=n, offset=addr).reshape(shape).copy()
