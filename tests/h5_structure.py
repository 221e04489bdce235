"""A second, independent reading of the HDF5 table files (test helper).

Written from the HDF5 File Format Specification separately from the library's
C++ decoder: it walks the superblock (version 0), the root group's object
header, symbol-table message, local heap, group B-tree and symbol-table node,
the dataset's object header (dataspace, datatype, fill value, layout and
attribute messages) and the chunk B-tree, checking each structure's
signature and the fields H5TBmake_table sets, and returns the table's
description and its raw records.
"""
import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF


class Reader:
    def __init__(self, path):
        with open(path, "rb") as f:
            self.d = f.read()

    def u(self, at, n):
        return int.from_bytes(self.d[at:at + n], "little")

    def cstr(self, at):
        end = self.d.index(b"\0", at)
        return self.d[at:end].decode()


def _messages(r, oh):
    assert r.u(oh, 1) == 1, "object header version 1"
    n, size = r.u(oh + 2, 2), r.u(oh + 8, 4)
    assert r.u(oh + 4, 4) >= 1, "reference count"
    out, at = [], oh + 16
    while at < oh + 16 + size and len(out) < n:
        t, s = r.u(at, 2), r.u(at + 2, 2)
        assert s % 8 == 0, "message data sizes are multiples of 8"
        out.append((t, at + 8, s))
        at += 8 + s
    assert len(out) == n, "message count"
    return out


def _member_type(r, at):
    cv = r.u(at, 1)
    cls, ver = cv & 0x0F, cv >> 4
    assert ver == 1
    bits, size = r.u(at + 1, 3), r.u(at + 4, 4)
    assert bits & 1 == 0, "little-endian"
    if cls == 0:
        assert r.u(at + 8, 2) == 0 and r.u(at + 10, 2) == 8 * size
        kind = ("i" if bits & 8 else "u") + str(8 * size)
        return kind, 12
    assert cls == 1 and size == 8
    assert (r.u(at + 8, 2), r.u(at + 10, 2), r.u(at + 12, 1), r.u(at + 13, 1), r.u(at + 14, 1),
            r.u(at + 15, 1), r.u(at + 16, 4)) == (0, 64, 52, 11, 0, 52, 1023)
    assert (bits & 0xFF) == 0x20 and ((bits >> 8) & 0xFF) == 63
    return "f64", 20


def read(path):
    r = Reader(path)
    assert r.d[:8] == b"\x89HDF\r\n\x1a\n"
    assert r.u(8, 1) == 0 and r.u(13, 1) == 8 and r.u(14, 1) == 8
    leaf_k, internal_k = r.u(16, 2), r.u(18, 2)
    assert r.u(24, 8) == 0 and r.u(40, 8) == len(r.d), "end-of-file address"
    root_oh = r.u(56 + 8, 8)
    assert r.u(56 + 16, 4) == 1
    btree, heap = r.u(56 + 24, 8), r.u(56 + 32, 8)
    (t, at, _), = _messages(r, root_oh)
    assert t == 0x0011 and (r.u(at, 8), r.u(at + 8, 8)) == (btree, heap)
    assert r.d[heap:heap + 4] == b"HEAP"
    heap_data = r.u(heap + 24, 8)
    assert r.d[btree:btree + 4] == b"TREE" and r.u(btree + 4, 1) == 0 and r.u(btree + 5, 1) == 0
    assert r.u(btree + 6, 2) == 1
    snod = r.u(btree + 32, 8)
    assert r.cstr(heap_data + r.u(btree + 24, 8)) == ""
    assert r.cstr(heap_data + r.u(btree + 40, 8)) == "table"
    assert r.d[snod:snod + 4] == b"SNOD" and r.u(snod + 4, 1) == 1 and r.u(snod + 6, 2) == 1
    assert r.cstr(heap_data + r.u(snod + 8, 8)) == "table"
    dset = r.u(snod + 16, 8)
    out = {"leaf_k": leaf_k, "internal_k": internal_k, "attributes": {}}
    for t, at, s in _messages(r, dset):
        if t == 0x0001:
            assert r.u(at, 1) == 1 and r.u(at + 1, 1) == 1 and r.u(at + 2, 1) & 1
            out["nrecords"] = r.u(at + 8, 8)
            assert r.u(at + 16, 8) == UNDEF, "extendible"
        elif t == 0x0003:
            assert r.u(at, 1) == 0x16, "compound, version 1"
            nm, size = r.u(at + 1, 2), r.u(at + 4, 4)
            out["record_size"] = size
            fields, p = [], at + 8
            for _ in range(nm):
                name = r.cstr(p)
                p += (len(name) + 1 + 7) // 8 * 8
                off = r.u(p, 4)
                assert r.u(p + 4, 1) == 0, "scalar member"
                p += 32
                kind, ln = _member_type(r, p)
                p += ln
                fields.append((name, off, kind))
            out["fields"] = fields
        elif t == 0x0005:
            assert r.u(at, 1) == 2
        elif t == 0x0008:
            assert r.u(at, 1) == 3 and r.u(at + 1, 1) == 2 and r.u(at + 2, 1) == 2
            out["chunk_tree"] = r.u(at + 3, 8)
            out["chunk_records"] = r.u(at + 11, 4)
            assert r.u(at + 15, 4) == out["record_size"]
        elif t == 0x000C:
            assert r.u(at, 1) == 1
            ln, tl, sl = r.u(at + 2, 2), r.u(at + 4, 2), r.u(at + 6, 2)
            name = r.cstr(at + 8)
            p = at + 8 + (ln + 7) // 8 * 8
            assert r.u(p, 1) == 0x13
            vlen = r.u(p + 4, 4)
            p += (tl + 7) // 8 * 8
            assert r.u(p, 1) == 1 and r.u(p + 1, 1) == 0, "scalar dataspace"
            p += (sl + 7) // 8 * 8
            out["attributes"][name] = r.d[p:p + vlen - 1].decode()
            assert r.d[p + vlen - 1] == 0
    # chunk index
    chunks = []

    def walk(node, lo, hi):
        assert r.d[node:node + 4] == b"TREE" and r.u(node + 4, 1) == 1
        level, n = r.u(node + 5, 1), r.u(node + 6, 2)
        assert 1 <= n <= 64
        keys = [node + 24 + i * 32 for i in range(n + 1)]
        offs = [r.u(k + 8, 8) for k in keys]
        assert offs == sorted(offs) and offs[0] >= lo and offs[-1] <= hi
        for i in range(n):
            child = r.u(keys[i] + 24, 8)
            assert r.u(keys[i] + 4, 4) == 0, "no filters"
            if level == 0:
                assert r.u(keys[i], 4) == out["chunk_records"] * out["record_size"]
                chunks.append((offs[i], child))
            else:
                walk(child, offs[i], offs[i + 1])

    if out["nrecords"]:
        walk(out["chunk_tree"], 0, UNDEF)
    else:
        assert out["chunk_tree"] == UNDEF
    chunks.sort()
    raw = bytearray()
    for i, (off, addr) in enumerate(chunks):
        assert off == i * out["chunk_records"]
        n = min(out["chunk_records"], out["nrecords"] - off)
        raw += r.d[addr:addr + n * out["record_size"]]
    out["raw"] = bytes(raw)
    return out


def records(info, dtype):
    """The raw records as ``dtype`` (which must match the file's layout)."""
    return np.frombuffer(info["raw"], dtype=dtype, count=info["nrecords"])


__all__ = ["read", "records", "struct"]
