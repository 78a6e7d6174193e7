"""A small HDF5 writer and reader, enough for the reference's instance files.

The reference writes solved model instances with the HDF5 C++ library
(model_instance::write_hdf5, src_ed/model_instance.hpp:1339-1421, with the
helpers of src_util/hdf5_io.cpp): nested groups whose attributes are scalar
doubles, 32-bit integers and strings, and 1-D double datasets. The HDF5 library
is not part of this package's dependencies, so this module writes and reads that
subset of the file format itself, following the published HDF5 file format
specification (version 0 superblock, version 1 object headers, groups stored as
symbol tables: a version 1 B-tree of symbol-table nodes plus a local heap of link
names), which is what the HDF5 library writes by default.

Written: strings as fixed-length, null-terminated ASCII (readers take either
kind). Read: also variable-length strings (global heap collections), header
continuation blocks and multi-level group B-trees, as the library writes them.
Not covered: chunked or compressed datasets, compact/dense ("new-style") groups,
version 2 object headers, attributes of other types than the three above.

API: File(path, mode) with .root; Group.create_group / group / attrs (dict) /
create_dataset / dataset / keys(); everything is written when the file closes.
"""
from __future__ import annotations

import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIG = b"\x89HDF\r\n\x1a\n"
LEAF_K = 8        # symbol-table node capacity: 2 * LEAF_K links
INTERNAL_K = 64   # B-tree node capacity: 2 * INTERNAL_K children


def _pad8(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 8)


# ------------------------------------------------------------------ datatypes --

def _dt_double() -> bytes:
    # class 1 (floating point), version 1; little endian, implied msb, sign at bit 63
    return struct.pack("<BBBBI", 0x11, 0x20, 0x3F, 0x00, 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)


def _dt_int32() -> bytes:
    # class 0 (fixed point), version 1; little endian, signed
    return struct.pack("<BBBBI", 0x10, 0x08, 0x00, 0x00, 4) + struct.pack("<HH", 0, 32)


def _dt_string(n: int) -> bytes:
    # class 3 (string), version 1; null-terminated ASCII of n bytes
    return struct.pack("<BBBBI", 0x13, 0x00, 0x00, 0x00, n)


def _dataspace(dims) -> bytes:
    # version 1: rank, no maximum dimensions; rank 0 is a scalar
    out = struct.pack("<BBBB4x", 1, len(dims), 0, 0)
    for d in dims:
        out += struct.pack("<Q", d)
    return out


# ------------------------------------------------------------------- writing --

class Dataset:
    def __init__(self, data):
        self.data = np.ascontiguousarray(data, dtype="<f8").ravel()
        self.attrs: dict = {}


class Group:
    def __init__(self):
        self.children: dict = {}
        self.attrs: dict = {}

    def create_group(self, name: str) -> "Group":
        if name in self.children:
            raise ValueError(f"an object named {name} exists already")
        g = Group()
        self.children[name] = g
        return g

    def create_dataset(self, name: str, data) -> Dataset:
        if name in self.children:
            raise ValueError(f"an object named {name} exists already")
        d = Dataset(data)
        self.children[name] = d
        return d

    def unlink(self, name: str):
        self.children.pop(name, None)

    def __contains__(self, name):
        return name in self.children

    def group(self, name: str) -> "Group":
        g = self.children[name]
        if not isinstance(g, Group):
            raise KeyError(f"{name} is not a group")
        return g

    def dataset(self, name: str) -> np.ndarray:
        d = self.children[name]
        if not isinstance(d, Dataset):
            raise KeyError(f"{name} is not a dataset")
        return d.data

    def keys(self):
        return list(self.children)


def _attr_message(name: str, value) -> bytes:
    if isinstance(value, str):
        raw = value.encode("ascii") + b"\0"
        dt, data = _dt_string(len(raw)), raw
    elif isinstance(value, (bool, int, np.integer)) and not isinstance(value, float):
        dt, data = _dt_int32(), struct.pack("<i", int(value))
    else:
        dt, data = _dt_double(), struct.pack("<d", float(value))
    nm = name.encode("ascii") + b"\0"
    ds = _dataspace([])
    # attribute message version 1: sizes of name, datatype and dataspace, each part padded to 8
    return struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(ds)) + _pad8(nm) + _pad8(dt) + _pad8(ds) + data


class _Writer:
    def __init__(self):
        self.buf = bytearray()

    def alloc(self, n: int) -> int:
        a = len(self.buf)
        self.buf += b"\0" * ((n + 7) // 8 * 8)
        return a

    def put(self, addr: int, b: bytes):
        self.buf[addr:addr + len(b)] = b

    def object_header(self, messages) -> int:
        body = b""
        for mtype, data in messages:
            data = _pad8(data)
            body += struct.pack("<HHB3x", mtype, len(data), 0) + data
        hdr = struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(body)) + body
        a = self.alloc(len(hdr))
        self.put(a, hdr)
        return a

    def write_dataset(self, d: Dataset) -> int:
        raw = d.data.tobytes()
        addr = self.alloc(len(raw)) if raw else UNDEF
        if raw:
            self.put(addr, raw)
        msgs = [(0x0001, _dataspace([len(d.data)])), (0x0003, _dt_double()),
                (0x0005, struct.pack("<BBBB", 2, 2, 2, 0)),  # fill value: late allocation, never written, undefined
                (0x0008, struct.pack("<BBQQ", 3, 1, addr, len(raw)))]  # contiguous layout
        msgs += [(0x000C, _attr_message(k, v)) for k, v in d.attrs.items()]
        return self.object_header(msgs)

    def write_group(self, g: Group) -> tuple[int, int, int]:
        """Returns (object header, B-tree, local heap) addresses."""
        names = sorted(g.children)
        entries = []
        for n in names:
            c = g.children[n]
            if isinstance(c, Group):
                oh, bt, lh = self.write_group(c)
                entries.append((n, oh, 1, bt, lh))
            else:
                entries.append((n, self.write_dataset(c), 0, 0, 0))
        # local heap: "" at offset 0, then the names, each null-terminated and padded to 8
        heap = bytearray(b"\0" * 8)
        offs = []
        for n in names:
            offs.append(len(heap))
            heap += _pad8(n.encode("ascii") + b"\0")
        heap += b"\0" * 8
        heap_data = self.alloc(len(heap))
        self.put(heap_data, bytes(heap))
        lh = self.alloc(32)
        # no free block: the HDF5 library's "null free list" offset is 1
        self.put(lh, b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap), 1, heap_data))
        # symbol-table nodes of up to 2 * LEAF_K entries, names in order
        cap = 2 * LEAF_K
        snods = []
        for i in range(0, max(len(entries), 1), cap):
            chunk = entries[i:i + cap]
            b = b"SNOD" + struct.pack("<BBH", 1, 0, len(chunk))
            for (n, oh, cache, bt, lhc), off in zip(chunk, offs[i:i + cap]):
                scratch = struct.pack("<QQ", bt, lhc) if cache else b"\0" * 16
                b += struct.pack("<QQI4x", off, oh, cache) + scratch
            b += b"\0" * (40 * (cap - len(chunk)))
            a = self.alloc(len(b))
            self.put(a, b)
            last = offs[min(i + cap, len(entries)) - 1] if entries else 0
            snods.append((a, last))
        if len(snods) > 2 * INTERNAL_K:
            raise ValueError(f"a group of more than {2 * INTERNAL_K * cap} objects")
        # one leaf-level B-tree node over the symbol-table nodes
        b = b"TREE" + struct.pack("<BBHQQ", 0, 0, len(snods) if entries else 0, UNDEF, UNDEF)
        b += struct.pack("<Q", 0)
        for a, last in snods if entries else []:
            b += struct.pack("<QQ", a, last)
        b += b"\0" * (16 * (2 * INTERNAL_K - (len(snods) if entries else 0)))
        bt = self.alloc(len(b))
        self.put(bt, b)
        msgs = [(0x0011, struct.pack("<QQ", bt, lh))]
        msgs += [(0x000C, _attr_message(k, v)) for k, v in g.attrs.items()]
        return self.object_header(msgs), bt, lh


def write_file(path: str, root: Group):
    w = _Writer()
    sb = w.alloc(96)
    oh, bt, lh = w.write_group(root)
    eof = len(w.buf)
    s = SIG + struct.pack("<BBBBBBBB", 0, 0, 0, 0, 0, 8, 8, 0) + struct.pack("<HHI", LEAF_K, INTERNAL_K, 0)
    s += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
    s += struct.pack("<QQI4xQQ", 0, oh, 1, bt, lh)  # root group symbol-table entry
    w.put(sb, s)
    with open(path, "wb") as f:
        f.write(bytes(w.buf))


# ------------------------------------------------------------------- reading --

class _Reader:
    def __init__(self, data: bytes):
        self.d = data
        if data[:8] != SIG:
            raise ValueError("not an HDF5 file (signature)")
        ver = data[8]
        if ver not in (0, 1):
            raise ValueError(f"HDF5 superblock version {ver} is not supported")
        if data[13] != 8 or data[14] != 8:
            raise ValueError("HDF5 files with offsets or lengths other than 8 bytes are not supported")
        p = 16 + 8 + (4 if ver == 1 else 0) + 4 * 8  # K values, flags (+ indexed-storage K), 4 addresses
        self.root_oh = struct.unpack_from("<Q", data, p + 8)[0]

    def u(self, fmt, off):
        return struct.unpack_from(fmt, self.d, off)

    def messages(self, addr):
        if self.d[addr] != 1:
            raise ValueError(f"object header version {self.d[addr]} at {addr} is not supported")
        n, _, size = self.u("<HII", addr + 2)
        blocks = [(addr + 16, size)]
        out = []
        while blocks and len(out) < n:
            p, size = blocks.pop(0)
            end = p + size
            while p + 8 <= end and len(out) < n:
                mtype, msize, flags = self.u("<HHB", p)
                body = self.d[p + 8:p + 8 + msize]
                if mtype == 0x0010:  # continuation: the next block of messages
                    blocks.append(self.u("<QQ", p + 8))
                out.append((mtype, body, flags))
                p += 8 + msize
        return out

    def datatype(self, b):
        cls, ver = b[0] & 0x0F, b[0] >> 4
        size = struct.unpack_from("<I", b, 4)[0]
        return cls, size, b

    def dataspace(self, b):
        ver, rank = b[0], b[1]
        off = 8 if ver == 1 else 4
        return [struct.unpack_from("<Q", b, off + 8 * i)[0] for i in range(rank)]

    def global_heap_object(self, addr, index):
        if self.d[addr:addr + 4] != b"GCOL":
            raise ValueError("bad global heap collection")
        size = self.u("<Q", addr + 8)[0]
        p, end = addr + 16, addr + size
        while p + 16 <= end:
            idx, _, osize = self.u("<HH4xQ", p)
            if idx == index:
                return self.d[p + 16:p + 16 + osize]
            if idx == 0:
                break
            p += 16 + (osize + 7) // 8 * 8
        raise ValueError("global heap object not found")

    def value(self, dt, dims, raw):
        cls, size, b = dt
        n = int(np.prod(dims)) if dims else 1
        if cls == 1:
            a = np.frombuffer(raw, dtype="<f8" if size == 8 else "<f4", count=n).astype(np.float64)
        elif cls == 0:
            signed = bool(b[1] & 0x08)
            a = np.frombuffer(raw, dtype=("<i" if signed else "<u") + str(size), count=n).astype(np.int64)
        elif cls == 3:
            s = raw[:size].split(b"\0", 1)[0].decode("ascii", "replace")
            return s
        elif cls == 9:  # variable-length string: (length, global heap address, index)
            ln, gaddr, idx = struct.unpack_from("<IQI", raw, 0)
            return self.global_heap_object(gaddr, idx)[:ln].decode("ascii", "replace")
        else:
            raise ValueError(f"HDF5 datatype class {cls} is not supported")
        return a if dims else (float(a[0]) if cls == 1 else int(a[0]))

    def attribute(self, body):
        ver = body[0]
        if ver == 1:
            nsz, dsz, ssz = struct.unpack_from("<HHH", body, 2)
            p = 8
            pad = lambda x: (x + 7) // 8 * 8
            name = body[p:p + nsz].split(b"\0", 1)[0].decode("ascii")
            p += pad(nsz)
            dt = self.datatype(body[p:p + dsz])
            p += pad(dsz)
            dims = self.dataspace(body[p:p + ssz])
            p += pad(ssz)
        elif ver in (2, 3):
            nsz, dsz, ssz = struct.unpack_from("<HHH", body, 2)
            p = 8 + (1 if ver == 3 else 0)
            name = body[p:p + nsz].split(b"\0", 1)[0].decode("utf-8")
            p += nsz
            dt = self.datatype(body[p:p + dsz])
            p += dsz
            dims = self.dataspace(body[p:p + ssz])
            p += ssz
        else:
            raise ValueError(f"attribute message version {ver} is not supported")
        return name, self.value(dt, dims, body[p:])

    def links(self, btree, heap_addr):
        heap_data = self.u("<Q", heap_addr + 24)[0]
        out = []

        def node(addr):
            if self.d[addr:addr + 4] == b"TREE":
                level, used = self.d[addr + 5], self.u("<H", addr + 6)[0]
                p = addr + 24 + 8
                for _ in range(used):
                    child = self.u("<Q", p)[0]
                    node(child)
                    p += 16
            elif self.d[addr:addr + 4] == b"SNOD":
                n = self.u("<H", addr + 6)[0]
                for i in range(n):
                    off, oh = self.u("<QQ", addr + 8 + 40 * i)
                    s = heap_data + off
                    name = self.d[s:self.d.index(b"\0", s)].decode("ascii")
                    out.append((name, oh))
            else:
                raise ValueError("bad group B-tree node")

        node(btree)
        return out

    def load(self, addr):
        msgs = self.messages(addr)
        attrs, stab, dims, dt, layout = {}, None, None, None, None
        for mtype, body, _ in msgs:
            if mtype == 0x000C:
                k, v = self.attribute(body)
                attrs[k] = v
            elif mtype == 0x0011:
                stab = struct.unpack_from("<QQ", body, 0)
            elif mtype == 0x0001:
                dims = self.dataspace(body)
            elif mtype == 0x0003:
                dt = self.datatype(body)
            elif mtype == 0x0008:
                layout = body
        if stab is not None:
            g = Group()
            g.attrs = attrs
            for name, oh in self.links(*stab):
                g.children[name] = self.load(oh)
            return g
        if layout is None or dt is None:
            raise ValueError("object that is neither a group nor a dataset")
        if layout[0] != 3 or layout[1] not in (0, 1):
            raise ValueError("only contiguous or compact datasets are supported")
        n = int(np.prod(dims)) if dims else 1
        if layout[1] == 1:
            a, size = struct.unpack_from("<QQ", layout, 2)
            raw = b"" if a == UNDEF else self.d[a:a + size]
        else:
            size = struct.unpack_from("<H", layout, 2)[0]
            raw = layout[4:4 + size]
        d = Dataset(self.value(dt, dims or [n], raw) if n else np.zeros(0))
        d.attrs = attrs
        return d


def read_file(path: str) -> Group:
    with open(path, "rb") as f:
        r = _Reader(f.read())
    return r.load(r.root_oh)


class File:
    """An HDF5 file held in memory: mode 'r' reads it, 'a' reads it when it exists
    (else starts empty) and writes it back on close, 'w' starts empty."""

    def __init__(self, path: str, mode: str = "r"):
        import os
        self.path, self.mode = path, mode
        if mode == "r" or (mode == "a" and os.path.exists(path)):
            self.root = read_file(path)
        elif mode in ("w", "a"):
            self.root = Group()
        else:
            raise ValueError(f"unknown mode {mode}")

    def close(self):
        if self.mode in ("w", "a"):
            write_file(self.path, self.root)
        self.mode = "r"

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        if exc[0] is None:
            self.close()
