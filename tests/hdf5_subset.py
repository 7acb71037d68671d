"""A reader of the HDF5 subset that kpolaris_b200/host/kp_hdf5.hpp writes --
test infrastructure, written independently of the writer from the HDF5 file
format specification: superblock version 2, version-2 object headers with
their Jenkins lookup3 checksums, compact new-style groups (Link Info, Group
Info and Link messages), contiguous datasets and scalar attributes of
fixed-point, IEEE floating-point and fixed-length string types.  Anything
outside the subset raises, so a test cannot pass on a structure the reader
does not understand.

    f = read(path)                 # the root Group
    f.attrs["schema"]              # str, int or float
    f["frame_0/freq_0/I"]          # numpy array shaped like the dataset
"""
from __future__ import annotations

import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"


def lookup3(data: bytes, initval: int = 0) -> int:
    """Bob Jenkins' hashlittle (lookup3.c, 2006), byte-at-a-time form."""
    M = 0xFFFFFFFF

    def rot(x, k):
        return ((x << k) | (x >> (32 - k))) & M

    n = len(data)
    a = b = c = (0xDEADBEEF + n + initval) & M
    i = 0
    while n > 12:
        a = (a + int.from_bytes(data[i:i + 4], "little")) & M
        b = (b + int.from_bytes(data[i + 4:i + 8], "little")) & M
        c = (c + int.from_bytes(data[i + 8:i + 12], "little")) & M
        a = (a - c) & M; a ^= rot(c, 4); c = (c + b) & M
        b = (b - a) & M; b ^= rot(a, 6); a = (a + c) & M
        c = (c - b) & M; c ^= rot(b, 8); b = (b + a) & M
        a = (a - c) & M; a ^= rot(c, 16); c = (c + b) & M
        b = (b - a) & M; b ^= rot(a, 19); a = (a + c) & M
        c = (c - b) & M; c ^= rot(b, 4); b = (b + a) & M
        n -= 12
        i += 12
    if n == 0:
        return c
    tail = data[i:i + n] + bytes(12 - n)
    a = (a + int.from_bytes(tail[0:4], "little")) & M
    b = (b + int.from_bytes(tail[4:8], "little")) & M
    c = (c + int.from_bytes(tail[8:12], "little")) & M
    c ^= b; c = (c - rot(b, 14)) & M
    a ^= c; a = (a - rot(c, 11)) & M
    b ^= a; b = (b - rot(a, 25)) & M
    c ^= b; c = (c - rot(b, 16)) & M
    a ^= c; a = (a - rot(c, 4)) & M
    b ^= a; b = (b - rot(a, 14)) & M
    c ^= b; c = (c - rot(b, 24)) & M
    return c


class FormatError(ValueError):
    pass


class Dataset:
    def __init__(self, name, value, attrs):
        self.name, self.value, self.attrs = name, value, attrs

    @property
    def shape(self):
        return self.value.shape

    def __getitem__(self, key):
        return self.value[key]


class Group:
    def __init__(self, name, attrs, links):
        self.name, self.attrs, self.links = name, attrs, links

    def __getitem__(self, path):
        node = self
        for part in path.strip("/").split("/"):
            if not isinstance(node, Group) or part not in node.links:
                raise KeyError(path)
            node = node.links[part]
        return node

    def __contains__(self, path):
        try:
            self[path]
            return True
        except KeyError:
            return False

    def keys(self):
        return list(self.links)


def _datatype(buf, p):
    """(numpy dtype or ('str', size), bytes consumed)."""
    cv = buf[p]
    cls, ver = cv & 0x0F, cv >> 4
    if ver != 1:
        raise FormatError(f"datatype version {ver}")
    bits = buf[p + 1:p + 4]
    size = struct.unpack_from("<I", buf, p + 4)[0]
    if cls == 0:  # fixed point
        if bits[0] & 0x01:
            raise FormatError("big-endian integer")
        off, prec = struct.unpack_from("<HH", buf, p + 8)
        if off != 0 or prec != 8 * size:
            raise FormatError("padded integer")
        signed = bool(bits[0] & 0x08)
        return np.dtype(("<i" if signed else "<u") + str(size)), 12
    if cls == 1:  # floating point
        if bits[0] & 0x01 or bits[0] & 0x40:
            raise FormatError("non little-endian float")
        off, prec, eloc, esz, mloc, msz = struct.unpack_from("<HHBBBB", buf, p + 8)
        bias = struct.unpack_from("<I", buf, p + 16)[0]
        norm = (bits[0] >> 4) & 0x03
        if (size, off, prec, eloc, esz, mloc, msz, bias, norm, bits[1]) == (8, 0, 64, 52, 11, 0, 52, 1023, 2, 63):
            return np.dtype("<f8"), 20
        if (size, off, prec, eloc, esz, mloc, msz, bias, norm, bits[1]) == (4, 0, 32, 23, 8, 0, 23, 127, 2, 31):
            return np.dtype("<f4"), 20
        raise FormatError("non-IEEE float")
    if cls == 3:  # fixed-length string
        pad, cset = bits[0] & 0x0F, bits[0] >> 4
        if pad != 0 or cset not in (0, 1):
            raise FormatError("string padding/charset")
        return ("str", size), 8
    raise FormatError(f"datatype class {cls}")


def _dataspace(buf, p):
    ver, rank, flags, kind = buf[p], buf[p + 1], buf[p + 2], buf[p + 3]
    if ver != 2:
        raise FormatError(f"dataspace version {ver}")
    if kind == 0:
        if rank != 0:
            raise FormatError("scalar with rank")
        return ()
    if kind != 1:
        raise FormatError(f"dataspace type {kind}")
    dims = struct.unpack_from(f"<{rank}Q", buf, p + 4)
    return tuple(int(d) for d in dims)


def _value(dt, raw, shape):
    if isinstance(dt, tuple):
        size = dt[1]
        if shape != ():
            raise FormatError("string arrays")
        s = bytes(raw[:size])
        if b"\0" not in s:
            raise FormatError("string without terminator")
        return s.split(b"\0", 1)[0].decode("ascii")
    n = int(np.prod(shape)) if shape else 1
    arr = np.frombuffer(bytes(raw[:n * dt.itemsize]), dtype=dt).copy()
    if shape == ():
        return arr[0].item()
    return arr.reshape(shape)


def _object(buf, addr, name):
    if buf[addr:addr + 4] != b"OHDR":
        raise FormatError(f"no object header at {addr}")
    ver, flags = buf[addr + 4], buf[addr + 5]
    if ver != 2:
        raise FormatError(f"object header version {ver}")
    if flags & 0xFC:
        raise FormatError(f"object header flags {flags:#x}")
    width = 1 << (flags & 0x03)
    p = addr + 6
    chunk = int.from_bytes(buf[p:p + width], "little")
    p += width
    end = p + chunk
    stored = struct.unpack_from("<I", buf, end)[0]
    if lookup3(bytes(buf[addr:end])) != stored:
        raise FormatError(f"object header checksum at {addr}")
    attrs, links, space, dtype, layout, linfo, ginfo, fill = {}, {}, None, None, None, False, False, False
    while p + 4 <= end:
        mtype, msize, mflags = buf[p], struct.unpack_from("<H", buf, p + 1)[0], buf[p + 3]
        q = p + 4
        if mtype == 0x00:
            pass
        elif mtype == 0x01:
            space = _dataspace(buf, q)
        elif mtype == 0x02:
            if buf[q] != 0 or buf[q + 1] != 0:
                raise FormatError("link info with creation order")
            heap, index = struct.unpack_from("<QQ", buf, q + 2)
            if heap != UNDEF or index != UNDEF:
                raise FormatError("dense link storage")
            linfo = True
        elif mtype == 0x03:
            dtype, _ = _datatype(buf, q)
        elif mtype == 0x05:
            if buf[q] != 3 or buf[q + 1] & 0x20:
                raise FormatError("fill value message")
            fill = True
        elif mtype == 0x06:
            if buf[q] != 1 or buf[q + 1] & 0xFC:
                raise FormatError("link message form")
            lw = 1 << (buf[q + 1] & 0x03)
            nlen = int.from_bytes(buf[q + 2:q + 2 + lw], "little")
            lname = bytes(buf[q + 2 + lw:q + 2 + lw + nlen]).decode("ascii")
            target = struct.unpack_from("<Q", buf, q + 2 + lw + nlen)[0]
            if lname in links:
                raise FormatError(f"duplicate link {lname}")
            links[lname] = target
        elif mtype == 0x08:
            if buf[q] != 3 or buf[q + 1] != 1:
                raise FormatError("non-contiguous layout")
            layout = struct.unpack_from("<QQ", buf, q + 2)
        elif mtype == 0x0A:
            if buf[q] != 0 or buf[q + 1] != 0:
                raise FormatError("group info form")
            ginfo = True
        elif mtype == 0x0C:
            if buf[q] != 3 or buf[q + 1] != 0:
                raise FormatError("attribute message form")
            nsz, tsz, ssz = struct.unpack_from("<HHH", buf, q + 2)
            r = q + 9
            aname = bytes(buf[r:r + nsz])
            if not aname.endswith(b"\0"):
                raise FormatError("attribute name terminator")
            aname = aname[:-1].decode("ascii")
            r += nsz
            adt, used = _datatype(buf, r)
            if used != tsz:
                raise FormatError("attribute datatype size")
            r += tsz
            ashape = _dataspace(buf, r)
            r += ssz
            if aname in attrs:
                raise FormatError(f"duplicate attribute {aname}")
            attrs[aname] = _value(adt, buf[r:q + msize], ashape)
        else:
            raise FormatError(f"header message type {mtype:#x}")
        p = q + msize
    if p != end:
        raise FormatError("object header messages overrun")
    if linfo or links:
        if not (linfo and ginfo) or space is not None:
            raise FormatError("group header form")
        return Group(name, attrs, {k: _object(buf, v, k) for k, v in links.items()})
    if space is None or dtype is None or layout is None or not fill:
        raise FormatError("dataset header form")
    addr_data, size = layout
    n = int(np.prod(space)) if space else 1
    if size != n * dtype.itemsize or (size and addr_data + size > len(buf)):
        raise FormatError("dataset extent")
    return Dataset(name, _value(dtype, buf[addr_data:addr_data + size], space), attrs)


def read(path):
    buf = memoryview(open(path, "rb").read())
    if bytes(buf[:8]) != SIGNATURE:
        raise FormatError("signature")
    if buf[8] != 2 or buf[9] != 8 or buf[10] != 8:
        raise FormatError("superblock version/sizes")
    base, ext, eof, root = struct.unpack_from("<QQQQ", buf, 12)
    if lookup3(bytes(buf[:44])) != struct.unpack_from("<I", buf, 44)[0]:
        raise FormatError("superblock checksum")
    if base != 0 or ext != UNDEF or eof != len(buf):
        raise FormatError("superblock addresses")
    return _object(buf, root, "/")
