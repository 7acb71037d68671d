"""Writes HDF5 files with the structures the HDF5 library itself writes --
test infrastructure for kpolaris_b200/host/kp_hdf5_read.hpp, written from
the HDF5 file format specification independently of the reader (no HDF5
library exists on these machines to make such files).

Two profiles:
  * "earliest" -- the library's default format (h5py's File(path, "w")):
    superblock version 0, version-1 object headers (8-byte aligned messages,
    optional continuation block), groups with a symbol table (version-1
    B-tree of group nodes, SNOD symbol nodes of at most 8 entries, a local
    heap of names), version-1 dataspaces, version-3 layouts (compact,
    contiguous, chunked with a version-1 B-tree of raw data chunks, filters
    deflate and shuffle in a version-1 filter pipeline).
  * "latest" -- superblock version 2, version-2 object headers ("OHDR" with
    an optional "OCHK" continuation chunk, lookup3 checksums), compact link
    storage (Link Info, Group Info and Link messages), version-2 dataspaces
    and version-4 layouts for chunked data (single-chunk index, filtered or
    not, and the implicit index).

    root = Group()
    g = root.group("header")
    g.dataset("n1", np.int32(8))
    root.dataset("prims", arr, layout="chunked", chunks=(4, 4, 4, 8), filters=("shuffle", "deflate"))
    write(path, root, profile="earliest", userblock=512)
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

from hdf5_subset import lookup3

UNDEF = 0xFFFFFFFFFFFFFFFF
SIG = b"\x89HDF\r\n\x1a\n"


def _pad8(b: bytes) -> bytes:
    return b + bytes((-len(b)) % 8)


class _Attrs:
    def attr(self, name, value):
        """A numeric scalar or array, a str (variable-length UTF-8 string, as
        h5py stores a Python str) or bytes (fixed-length string)."""
        self.attrs[name] = value
        return self


class Dataset(_Attrs):
    def __init__(self, value, layout="contiguous", chunks=None, filters=(), index="btree", continuation=False):
        self.value = np.asarray(value)
        self.layout, self.chunks, self.filters = layout, chunks, tuple(filters)
        self.index, self.continuation = index, continuation
        self.attrs = {}


class Group(_Attrs):
    def __init__(self, fanout: int = 32, continuation: bool = False):
        self.children: dict[str, object] = {}
        self.fanout, self.continuation = fanout, continuation
        self.attrs = {}

    def group(self, name, **kw) -> "Group":
        g = Group(**kw)
        self.children[name] = g
        return g

    def dataset(self, name, value, **kw) -> Dataset:
        d = Dataset(value, **kw)
        self.children[name] = d
        return d


class _Image:
    """The file being laid out: addresses are relative to the superblock."""

    def __init__(self, start: int):
        self.buf = bytearray(start)
        self.base = 0

    def alloc(self, data: bytes, align: int = 8) -> int:
        while len(self.buf) % align:
            self.buf.append(0)
        addr = len(self.buf) - self.base
        self.buf += data
        return addr

    def reserve(self, n: int, align: int = 8) -> int:
        return self.alloc(bytes(n), align)

    def put(self, addr: int, data: bytes) -> None:
        a = addr + self.base
        self.buf[a:a + len(data)] = data


def _datatype(dt: np.dtype) -> bytes:
    if dt.kind == "f":
        if dt.itemsize == 8:
            return struct.pack("<BBBBI", 0x11, 0x20, 63, 0, 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
        return struct.pack("<BBBBI", 0x11, 0x20, 31, 0, 4) + struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
    if dt.kind in "iu":
        bits0 = 0x08 if dt.kind == "i" else 0x00
        return struct.pack("<BBBBI", 0x10, bits0, 0, 0, dt.itemsize) + struct.pack("<HH", 0, 8 * dt.itemsize)
    raise ValueError(dt)


def _dataspace(shape, version) -> bytes:
    if version == 1:
        head = struct.pack("<BBBB4x", 1, len(shape), 1, 0)
        return head + b"".join(struct.pack("<Q", d) for d in shape) * 2
    kind = 0 if len(shape) == 0 else 1
    head = struct.pack("<BBBB", 2, len(shape), 1, kind)
    return head + b"".join(struct.pack("<Q", d) for d in shape) * 2


def _filter_pipeline(filters, elem) -> bytes:
    body = b""
    for name in filters:
        if name == "deflate":
            fid, nm, cv = 1, b"deflate\0", [6]
        else:
            fid, nm, cv = 2, b"shuffle\0", [elem]
        body += struct.pack("<HHHH", fid, len(nm), 0, len(cv)) + _pad8(nm)
        body += b"".join(struct.pack("<I", v) for v in cv) + (bytes(4) if len(cv) % 2 else b"")
    return struct.pack("<BB6x", 1, len(filters)) + body


def _encode_chunk(raw: bytes, filters, elem) -> bytes:
    for name in filters:
        if name == "shuffle" and elem > 1:
            n = len(raw) // elem
            a = np.frombuffer(raw[:n * elem], dtype=np.uint8).reshape(n, elem)
            raw = a.T.tobytes() + raw[n * elem:]
        elif name == "deflate":
            raw = zlib.compress(raw, 6)
    return raw


def _chunks_of(value: np.ndarray, chunks):
    """(origin, raw chunk bytes padded with zeros) in row-major chunk order."""
    grid = [range(0, d, c) for d, c in zip(value.shape, chunks)]
    for origin in np.ndindex(*[len(g) for g in grid]):
        o = tuple(i * c for i, c in zip(origin, chunks))
        block = np.zeros(chunks, dtype=value.dtype)
        sl = tuple(slice(a, min(a + c, d)) for a, c, d in zip(o, chunks, value.shape))
        part = value[sl]
        block[tuple(slice(0, s) for s in part.shape)] = part
        yield o, block.tobytes()


def _vlen_string_type(so: int = 8) -> bytes:
    # class 9 version 1, string, null-terminated, UTF-8; base type one byte
    base = struct.pack("<BBBBI", 0x10, 0, 0, 0, 1) + struct.pack("<HH", 0, 8)
    return struct.pack("<BBBBI", 0x19, 0x01, 0x01, 0, 4 + so + 4) + base


def _fixed_string_type(n: int) -> bytes:
    return struct.pack("<BBBBI", 0x13, 0x00, 0, 0, n)


class _Writer:
    def __init__(self, profile: str, userblock: int):
        self.profile = profile
        self.img = _Image(userblock)
        self.img.base = userblock

    # -- object headers --------------------------------------------------------
    def header(self, messages, continuation=False) -> int:
        """messages: [(type, body)]; returns the header address."""
        if self.profile == "earliest":
            return self._header_v1(messages, continuation)
        return self._header_v2(messages, continuation)

    def _msgs_v1(self, messages) -> bytes:
        return b"".join(struct.pack("<HHB3x", t, len(_pad8(b)), 0) + _pad8(b) for t, b in messages)

    def _header_v1(self, messages, continuation) -> int:
        if continuation and len(messages) > 1:
            first, rest = messages[:1], messages[1:]
            blk = self._msgs_v1(rest)
            caddr = self.img.alloc(blk)
            first = first + [(0x10, struct.pack("<QQ", caddr, len(blk)))]
            body = self._msgs_v1(first)
            n = len(first) + len(rest)
        else:
            body = self._msgs_v1(messages)
            n = len(messages)
        return self.img.alloc(struct.pack("<BBHII4x", 1, 0, n, 1, len(body)) + body)

    @staticmethod
    def _msgs_v2(messages) -> bytes:
        return b"".join(struct.pack("<BHB", t, len(b), 0) + b for t, b in messages)

    def _header_v2(self, messages, continuation) -> int:
        if continuation and len(messages) > 1:
            first, rest = messages[:1], messages[1:]
            blk = b"OCHK" + self._msgs_v2(rest)
            blk += struct.pack("<I", lookup3(blk))
            caddr = self.img.alloc(blk)
            messages = first + [(0x10, struct.pack("<QQ", caddr, len(blk)))]
        body = self._msgs_v2(messages)
        head = b"OHDR" + struct.pack("<BB", 2, 0x02) + struct.pack("<I", len(body))
        whole = head + body
        return self.img.alloc(whole + struct.pack("<I", lookup3(whole)))

    # -- attributes ------------------------------------------------------------
    def _global_heap(self, data: bytes):
        """(collection address, object index) of `data` in a new 4096-byte
        global heap collection; the rest of it is the free-space object."""
        obj = struct.pack("<HHIQ", 1, 0, 0, len(data)) + _pad8(data)
        size = max(4096, 16 + len(obj) + 16)
        free = size - 16 - len(obj)
        body = b"GCOL" + struct.pack("<B3xQ", 1, size) + obj + struct.pack("<HHIQ", 0, 0, 0, free)
        body += bytes(size - len(body))
        return self.img.alloc(body), 1

    def attr_messages(self, attrs):
        msgs = []
        for name, value in attrs.items():
            if isinstance(value, str):
                raw = value.encode()
                addr, idx = self._global_heap(raw)
                dtype, space, data = _vlen_string_type(), (), struct.pack("<IQI", len(raw), addr, idx)
            elif isinstance(value, bytes):
                dtype, space, data = _fixed_string_type(len(value) + 1), (), value + b"\0"
            else:
                v = np.asarray(value)
                v = v.astype(v.dtype.newbyteorder("<"))
                dtype, space, data = _datatype(v.dtype), v.shape, v.tobytes()
            ds = _dataspace(space, 1 if self.profile == "earliest" else 2)
            nm = name.encode() + b"\0"
            if self.profile == "earliest":
                body = struct.pack("<BBHHH", 1, 0, len(nm), len(dtype), len(ds)) + _pad8(nm) + _pad8(dtype) + _pad8(ds)
            else:
                body = struct.pack("<BBHHHB", 3, 0, len(nm), len(dtype), len(ds), 0) + nm + dtype + ds
            msgs.append((0x0C, body + data))
        return msgs

    # -- groups ----------------------------------------------------------------
    def group(self, g: Group) -> int:
        addrs = {name: (self.group(c) if isinstance(c, Group) else self.dataset(c))
                 for name, c in g.children.items()}
        if self.profile == "latest":
            msgs = [(0x02, struct.pack("<BBQQ", 0, 0, UNDEF, UNDEF)), (0x0A, struct.pack("<BB", 0, 0))]
            for name, a in addrs.items():
                nm = name.encode()
                msgs.append((0x06, struct.pack("<BBB", 1, 0, len(nm)) + nm + struct.pack("<Q", a)))
            return self.header(msgs + self.attr_messages(g.attrs), g.continuation)
        # local heap of names: offset 0 is the empty string
        names = sorted(addrs)
        heap = bytearray(8)
        offsets = {}
        for name in names:
            offsets[name] = len(heap)
            heap += _pad8(name.encode() + b"\0")
        heap_data = self.img.alloc(bytes(heap))
        heap_addr = self.img.alloc(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap), UNDEF, heap_data))
        # symbol nodes of up to 8 entries (2 x leaf K = 4)
        snods = []
        for i in range(0, max(len(names), 1), 8):
            part = names[i:i + 8]
            ent = b"".join(struct.pack("<QQII16x", offsets[n], addrs[n], 0, 0) for n in part)
            ent += bytes(40 * (8 - len(part)))
            snods.append((self.img.alloc(b"SNOD" + struct.pack("<BBH", 1, 0, len(part)) + ent),
                          offsets[part[-1]] if part else 0))
        # level-0 B-tree nodes of up to `fanout` SNODs, and a level-1 root above them when needed
        def node(level, kids):
            body = struct.pack("<Q", 0)
            for addr, last in kids:
                body += struct.pack("<QQ", addr, last)
            return self.img.alloc(b"TREE" + struct.pack("<BBHQQ", 0, level, len(kids), UNDEF, UNDEF) + body)

        leaves = [snods[i:i + g.fanout] for i in range(0, len(snods), g.fanout)]
        level0 = [(node(0, kids), kids[-1][1]) for kids in leaves]
        root = level0[0][0] if len(level0) == 1 else node(1, level0)
        return self.header([(0x11, struct.pack("<QQ", root, heap_addr))] + self.attr_messages(g.attrs),
                           g.continuation)

    # -- datasets --------------------------------------------------------------
    def dataset(self, d: Dataset) -> int:
        v = np.array(d.value, order="C")  # keeps a scalar 0-d
        v = v.astype(v.dtype.newbyteorder("<"))
        elem = v.dtype.itemsize
        space = _dataspace(v.shape, 1 if self.profile == "earliest" else 2)
        msgs = [(0x01, space), (0x03, _datatype(v.dtype)), (0x05, struct.pack("<BBBB", 2, 2, 2, 0))]
        if d.layout == "compact":
            raw = v.tobytes()
            msgs.append((0x08, struct.pack("<BBH", 3, 0, len(raw)) + raw))
        elif d.layout == "contiguous":
            addr = self.img.alloc(v.tobytes())
            msgs.append((0x08, struct.pack("<BBQQ", 3, 1, addr, v.nbytes)))
        else:
            chunks = tuple(d.chunks)
            if d.filters:
                msgs.append((0x0B, _filter_pipeline(d.filters, elem)))
            if d.index == "btree":
                entries = []
                for o, raw in _chunks_of(v, chunks):
                    stored = _encode_chunk(raw, d.filters, elem)
                    entries.append((o, len(stored), self.img.alloc(stored)))
                btree = self._chunk_btree(entries, v.shape)
                dims = b"".join(struct.pack("<I", c) for c in chunks) + struct.pack("<I", elem)
                msgs.append((0x08, struct.pack("<BBBQ", 3, 2, len(chunks) + 1, btree) + dims))
            else:
                data = [(o, _encode_chunk(raw, d.filters, elem)) for o, raw in _chunks_of(v, chunks)]
                dims = b"".join(struct.pack("<Q", c) for c in chunks) + struct.pack("<Q", elem)
                head = struct.pack("<BBBBB", 4, 2, 0x02 if (d.index == "single" and d.filters) else 0,
                                   len(chunks) + 1, 8) + dims
                if d.index == "single":
                    assert len(data) == 1
                    addr = self.img.alloc(data[0][1])
                    extra = struct.pack("<QI", len(data[0][1]), 0) if d.filters else b""
                    msgs.append((0x08, head + struct.pack("<B", 1) + extra + struct.pack("<Q", addr)))
                else:
                    assert not d.filters
                    addr = self.img.alloc(b"".join(raw for _, raw in data))
                    msgs.append((0x08, head + struct.pack("<BQ", 2, addr)))
        msgs.append((0x12, struct.pack("<B3xI", 1, 1700000000)))  # modification time (skipped by readers)
        return self.header(msgs + self.attr_messages(d.attrs), d.continuation)

    def _chunk_btree(self, entries, shape, fanout: int = 3) -> int:
        rank = len(shape)

        def key(o, size):
            return struct.pack("<II", size, 0) + b"".join(struct.pack("<Q", x) for x in o) + struct.pack("<Q", 0)

        end = key(tuple(shape), 0)

        def node(level, kids):
            body = b"".join(k + struct.pack("<Q", a) for k, a in kids) + end
            return self.img.alloc(b"TREE" + struct.pack("<BBHQQ", 1, level, len(kids), UNDEF, UNDEF) + body)

        leaves = [entries[i:i + fanout] for i in range(0, len(entries), fanout)]
        level0 = [(key(part[0][0], part[0][1]), node(0, [(key(o, n), a) for o, n, a in part])) for part in leaves]
        assert rank >= 0
        return level0[0][1] if len(level0) == 1 else node(1, level0)

    # -- file ------------------------------------------------------------------
    def finish(self, root: Group) -> bytes:
        sb_size = 96 if self.profile == "earliest" else 48
        sb = self.img.reserve(sb_size)
        assert sb == 0
        root_addr = self.group(root)
        eof = len(self.img.buf) - self.img.base
        if self.profile == "earliest":
            head = SIG + struct.pack("<BBBBBBBB", 0, 0, 0, 0, 0, 8, 8, 0) + struct.pack("<HHI", 4, 16, 0)
            head += struct.pack("<QQQQ", self.img.base, UNDEF, eof, UNDEF)
            head += struct.pack("<QQII16x", 0, root_addr, 0, 0)
            assert len(head) == 96
        else:
            head = SIG + struct.pack("<BBBB", 2, 8, 8, 0) + struct.pack("<QQQQ", self.img.base, UNDEF, eof, root_addr)
            head += struct.pack("<I", lookup3(head))
            assert len(head) == 48
        self.img.put(0, head)
        return bytes(self.img.buf)


def write(path, root: Group, *, profile: str = "earliest", userblock: int = 0) -> None:
    if profile not in ("earliest", "latest"):
        raise ValueError(profile)
    w = _Writer(profile, userblock)
    data = w.finish(root)
    with open(path, "wb") as f:
        f.write(data)
