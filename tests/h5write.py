"""A minimal HDF5 writer for the format subset croma_b200_h5_* reads (test
infrastructure): superblock version 0, groups as symbol tables (version-1
B-tree group nodes over symbol table nodes, a local heap for the names),
version-1 object headers, datasets of fixed-point or IEEE floating-point
elements in either byte order, contiguous or compact, with a version-1
dataspace.  Written from the HDF5 File Format Specification version 3.0 to
drive the reader through the branches the reference's snapshot files do not
use: nested groups, compact storage, object-header continuation blocks,
B-trees split over several symbol table nodes and levels, big-endian and
narrow types, rank 2 and scalars.
"""
from __future__ import annotations

import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF


class _Buf:
    def __init__(self):
        self.b = bytearray()

    def alloc(self, n: int, align: int = 8) -> int:
        pad = (-len(self.b)) % align
        self.b += b"\0" * pad
        at = len(self.b)
        self.b += b"\0" * n
        return at

    def put(self, at: int, data: bytes):
        self.b[at:at + len(data)] = data


def _msg(mtype: int, data: bytes) -> bytes:
    data = data + b"\0" * ((-len(data)) % 8)
    return struct.pack("<HHB3x", mtype, len(data), 0) + data


def _dtype_msg(dt: np.dtype) -> bytes:
    big = dt.byteorder == ">" or (dt.byteorder == "=" and np.little_endian is False)
    if dt.kind == "f":
        bits = (1 if big else 0) | (2 << 4)   # byte order; mantissa normalisation: msb implied
        sign_loc = dt.itemsize * 8 - 1
        if dt.itemsize == 8:
            props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
        else:
            props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
        head = bytes([0x10 | 1, bits & 0xFF, sign_loc, 0])
        return head + struct.pack("<I", dt.itemsize) + props
    signed = dt.kind == "i"
    bits = (1 if big else 0) | (8 if signed else 0)
    head = bytes([0x10 | 0, bits, 0, 0])
    return head + struct.pack("<I", dt.itemsize) + struct.pack("<HH", 0, dt.itemsize * 8)


def _space_msg(shape, version: int = 1, null: bool = False) -> bytes:
    if version == 2:   # version 2: no reserved bytes, an explicit scalar / simple / null type
        kind = 2 if null else (0 if len(shape) == 0 else 1)
        out = struct.pack("<BBBB", 2, 0 if null else len(shape), 0, kind)
        if null:
            return out
    else:
        out = struct.pack("<BBBB4x", 1, len(shape), 0, 0)
    for d in shape:
        out += struct.pack("<Q", d)
    return out


def _object_header(buf: _Buf, messages, split: int | None = None) -> int:
    """Version-1 object header; with split, the messages from index split on
    go to a continuation block."""
    first = messages if split is None else messages[:split]
    rest = [] if split is None else messages[split:]
    cont_at = None
    body = b"".join(first)
    if rest:
        rest_body = b"".join(rest)
        cont_at = buf.alloc(len(rest_body))
        buf.put(cont_at, rest_body)
        body += _msg(0x10, struct.pack("<QQ", cont_at, len(rest_body)))
    at = buf.alloc(16 + len(body))
    nmsg = len(messages) + (1 if rest else 0)
    buf.put(at, struct.pack("<BBHII4x", 1, 0, nmsg, 1, len(body)) + body)
    return at


def _dataset(buf: _Buf, arr: np.ndarray, compact: bool, split: bool, space_version: int = 1,
             null: bool = False) -> int:
    raw = b"" if null else arr.tobytes()
    if compact:
        layout = struct.pack("<BBH", 3, 0, len(raw)) + raw
    else:
        data_at = buf.alloc(len(raw))
        buf.put(data_at, raw)
        layout = struct.pack("<BBQQ", 3, 1, data_at, len(raw))
    msgs = [_msg(0x01, _space_msg(arr.shape, space_version, null)), _msg(0x03, _dtype_msg(arr.dtype)),
            _msg(0x08, layout)]
    return _object_header(buf, msgs, split=1 if split else None)


def _group(buf: _Buf, children: dict, leaf_k: int):
    """Write the symbol table of a group whose children are {name: header
    address}; returns (btree address, heap address)."""
    names = sorted(children)
    # local heap: offset 0 is the empty string
    heap_data = bytearray(b"\0" * 8)
    offs = {}
    for n in names:
        offs[n] = len(heap_data)
        heap_data += n.encode() + b"\0"
        heap_data += b"\0" * ((-len(heap_data)) % 8)
    data_at = buf.alloc(len(heap_data))
    buf.put(data_at, bytes(heap_data))
    heap_at = buf.alloc(32)
    buf.put(heap_at, b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap_data), UNDEF, data_at))
    # symbol table nodes of at most 2 leaf_k entries each
    cap = 2 * leaf_k
    snods = []
    for i in range(0, len(names), cap):
        part = names[i:i + cap]
        node = b"SNOD" + struct.pack("<BBH", 1, 0, len(part))
        for n in part:
            node += struct.pack("<QQII16x", offs[n], children[n], 0, 0)
        node += b"\0" * ((cap - len(part)) * 40)
        at = buf.alloc(len(node))
        buf.put(at, node)
        snods.append((offs[part[0]], at))
    if not snods:
        node = b"SNOD" + struct.pack("<BBH", 1, 0, 0) + b"\0" * (cap * 40)
        at = buf.alloc(len(node))
        buf.put(at, node)
        snods.append((0, at))

    def tree(entries, level):
        node = b"TREE" + struct.pack("<BBHQQ", 0, level, len(entries), UNDEF, UNDEF)
        for key, child in entries:
            node += struct.pack("<QQ", key, child)
        node += struct.pack("<Q", 0)
        at = buf.alloc(len(node))
        buf.put(at, node)
        return at

    # one level of internal nodes over leaves of two symbol table nodes each,
    # when there are more than two
    if len(snods) <= 2:
        return tree(snods, 0), heap_at
    leaves = [(snods[i][0], tree(snods[i:i + 2], 0)) for i in range(0, len(snods), 2)]
    return tree(leaves, 1), heap_at


def write(path: str, tree: dict, leaf_k: int = 4, compact=(), split=(), sb_version: int = 0,
          userblock: int = 0, space_version: int = 1, null=()):
    """tree: {name: ndarray | dict (a subgroup)}; names in compact are
    stored compact, those in split with a continuation block.  sb_version 0
    or 1 (version 1 adds the indexed-storage K); userblock bytes (0 or
    512 * 2^k) of filler before the superblock, whose base address then
    points at it.  space_version 1 or 2 for every dataspace; names in null
    get a null dataspace (no elements)."""
    buf = _Buf()
    buf.alloc(104)   # superblock + root entry, written last

    def build(node: dict, prefix: str) -> tuple:
        children = {}
        for name, v in node.items():
            full = prefix + name
            if isinstance(v, dict):
                bt, hp = build(v, full + "/")
                children[name] = _object_header(buf, [_msg(0x11, struct.pack("<QQ", bt, hp))])
            else:
                children[name] = _dataset(buf, np.asarray(v), full in compact, full in split, space_version,
                                          full in null)
        return _group(buf, children, leaf_k)

    bt, hp = build(tree, "")
    root_oh = _object_header(buf, [_msg(0x11, struct.pack("<QQ", bt, hp))])
    sb = b"\x89HDF\r\n\x1a\n" + struct.pack("<BBBBBBBBHHI", sb_version, 0, 0, 0, 0, 8, 8, 0, leaf_k, 16, 0)
    if sb_version == 1:
        sb += struct.pack("<HH", 32, 0)   # indexed storage internal node K, reserved
    sb += struct.pack("<QQQQ", userblock, UNDEF, len(buf.b), UNDEF)
    sb += struct.pack("<QQII", 0, root_oh, 1, 0) + struct.pack("<QQ", bt, hp)
    buf.put(0, sb)
    with open(path, "wb") as f:
        f.write(b"U" * userblock + bytes(buf.b))
