"""A writer of small HDF5 files, test infrastructure: it lays files out the
way the HDF5 library does with default property lists (the way the
reference's grid and restart files are written, and the only layout
phenlei_b200.h5lite reads), after the published HDF5 File Format
Specification:

* a version 0 (or 1) superblock whose root symbol-table entry caches the
  root group's B-tree and local heap;
* version 1 object headers;
* groups: a symbol-table message, one level-0 group B-tree node, one
  symbol-table node with the members sorted by name, a local heap of names;
* datasets: version 1 dataspace, fixed-point / IEEE float / string datatype,
  version 3 contiguous layout.

    write_h5(path, {"Information": {"nBlocks": np.array([1], np.int32)}, ...})

A dict is a group, a numpy array a dataset.
"""
from __future__ import annotations

import struct

import numpy as np

UNDEF = (1 << 64) - 1


def _pad8(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 8)


class _Writer:
    def __init__(self, sb_size=96):
        self.sb_size = sb_size
        self.buf = bytearray(sb_size)     # the superblock with the root entry, written last

    def _alloc(self, data: bytes) -> int:
        addr = len(self.buf)
        self.buf += _pad8(data)
        return addr

    @staticmethod
    def _header(msgs: list) -> bytes:
        body = b""
        for mtype, data in msgs:
            data = _pad8(data)
            body += struct.pack("<HHB3x", mtype, len(data), 0) + data
        # version 1, reserved, message count, reference count, header size, alignment padding
        return struct.pack("<BBHII4x", 1, 0, len(msgs), 1, len(body)) + body

    def _datatype(self, a: np.ndarray) -> bytes:
        dt = a.dtype
        if dt.kind in "iu":
            bits = 0x08 if dt.kind == "i" else 0
            return struct.pack("<B3BI", 0x10 | 0, bits, 0, 0, dt.itemsize) + struct.pack("<HH", 0, 8 * dt.itemsize)
        if dt.kind == "f":
            if dt.itemsize == 8:
                props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
                bits = (0x20, 63, 0)       # mantissa normalisation 2 (implied 1), sign at bit 63
            else:
                props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
                bits = (0x20, 31, 0)
            return struct.pack("<B3BI", 0x10 | 1, *bits, dt.itemsize) + props
        if dt.kind == "S":
            return struct.pack("<B3BI", 0x10 | 3, 0, 0, 0, dt.itemsize)
        raise ValueError(f"dtype {dt} is not written")

    def dataset(self, a: np.ndarray) -> int:
        a = np.ascontiguousarray(a)
        if a.dtype.byteorder == ">":
            a = a.astype(a.dtype.newbyteorder("<"))
        data = a.tobytes()
        daddr = self._alloc(data) if data else UNDEF
        shape = a.shape if a.ndim else (1,)
        space = struct.pack("<BBB5x", 1, len(shape), 0) + b"".join(struct.pack("<Q", d) for d in shape)
        layout = struct.pack("<BBQQ", 3, 1, daddr, len(data))
        return self._alloc(self._header([(0x0001, space), (0x0003, self._datatype(a)), (0x0008, layout)]))

    def group(self, members: dict):
        """Returns (object header address, B-tree address, heap address)."""
        addrs = {}
        for name in sorted(members):
            v = members[name]
            addrs[name] = self.group(v)[0] if isinstance(v, dict) else self.dataset(np.asarray(v))
        names = sorted(members)
        heap_data = b"\0"
        offs = {}
        for n in names:
            offs[n] = len(heap_data)
            heap_data += _pad8(n.encode() + b"\0")
        heap_data = _pad8(heap_data)
        hdata_addr = self._alloc(heap_data)
        heap = self._alloc(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap_data), UNDEF, hdata_addr))
        entries = b"".join(struct.pack("<QQII16x", offs[n], addrs[n], 0, 0) for n in names)
        snod = self._alloc(b"SNOD" + struct.pack("<BBH", 1, 0, len(names)) + entries)
        last = offs[names[-1]] if names else 0
        btree = self._alloc(b"TREE" + struct.pack("<BBHQQ", 0, 0, 1, UNDEF, UNDEF)
                            + struct.pack("<QQQ", 0, snod, last))
        hdr = self._alloc(self._header([(0x0011, struct.pack("<QQ", btree, heap))]))
        return hdr, btree, heap

    def finish(self, root, version=0) -> bytes:
        hdr, btree, heap = root
        # version 1 adds the indexed-storage internal node K (2 bytes) and 2 reserved bytes
        extra = struct.pack("<HH", 32, 0) if version == 1 else b""
        sb = (b"\x89HDF\r\n\x1a\n" + bytes([version, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", 4, 16, 0)
              + extra + struct.pack("<QQQQ", 0, UNDEF, len(self.buf), UNDEF)
              + struct.pack("<QQII", 0, hdr, 1, 0) + struct.pack("<QQ", btree, heap))
        assert len(sb) == self.sb_size
        self.buf[:self.sb_size] = sb
        return bytes(self.buf)


def write_h5(path: str, tree: dict, superblock_version: int = 0) -> None:
    w = _Writer(100 if superblock_version == 1 else 96)
    root = w.group(tree)
    with open(path, "wb") as f:
        f.write(w.finish(root, superblock_version))
