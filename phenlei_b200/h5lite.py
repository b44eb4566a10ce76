"""A reader for the part of the HDF5 file format that PHengLEI's grid files
use, written from the published HDF5 File Format Specification.  No HDF5
library is needed (none is installed on these machines).

The reference writes its files through the HDF5 C library with default
property lists (API/PreProcess/src/Pre_HDF5File.cpp: H5Fcreate, H5Gcreate2,
H5Dcreate2).  Such files hold:

* a version 0 (or 1) superblock;
* version 1 object headers, continued through continuation messages;
* groups indexed by a version 1 B-tree of symbol-table nodes, with their
  member names in a local heap;
* datasets with a simple dataspace, a fixed-point, floating-point or
  fixed-length string datatype, and contiguous storage.

That is what this reader covers.  Anything else (version 2 object headers,
link-message groups, chunked or filtered storage) raises H5Error rather than
being misread.

    f = H5File(path)
    f.keys("/Grid-0")                          # member names of a group
    f.read("/Grid-0/FaceTopology/face2Node")   # numpy array
"""
from __future__ import annotations

import mmap
import os

import numpy as np

_SIGNATURE = b"\x89HDF\r\n\x1a\n"
_UNDEF = (1 << 64) - 1

# object header message types used here
_MSG_DATASPACE = 0x0001
_MSG_LINK_INFO = 0x0002
_MSG_DATATYPE = 0x0003
_MSG_LINK = 0x0006
_MSG_LAYOUT = 0x0008
_MSG_FILTERS = 0x000B
_MSG_CONTINUATION = 0x0010
_MSG_SYMBOL_TABLE = 0x0011


class H5Error(ValueError):
    """The file is not HDF5, or it uses a feature outside this reader's part."""


class H5File:
    def __init__(self, path: str):
        # mapped, not read: a grid file of a large mesh is read in the parts asked for
        with open(path, "rb") as f:
            size = os.fstat(f.fileno()).st_size
            if size < 8:
                raise H5Error("no HDF5 signature")
            self.b = mmap.mmap(f.fileno(), 0, access=mmap.ACCESS_READ)
        base = self._find_superblock()
        ver = self.b[base + 8]
        if ver not in (0, 1):
            raise H5Error(f"superblock version {ver}: only versions 0 and 1 are read")
        # sizes of offsets and lengths
        self.so, self.sl = self.b[base + 13], self.b[base + 14]
        p = base + 24 + (4 if ver == 1 else 0)    # version 1 adds the indexed-storage K and a reserved pair
        self.base_addr = self._addr(p)
        p += 4 * self.so                           # base, free-space, end-of-file and driver-info addresses
        # the root group's symbol table entry: link name offset, then its object header address
        self.root = self._addr(p + self.so)
        self._headers = {}

    # --- low level ------------------------------------------------------
    def _find_superblock(self) -> int:
        """The signature sits at offset 0, 512, 1024, 2048, ..."""
        off = 0
        while off + 8 <= len(self.b):
            if self.b[off:off + 8] == _SIGNATURE:
                return off
            off = 512 if off == 0 else off * 2
        raise H5Error("no HDF5 signature")

    def _u(self, p: int, n: int) -> int:
        if p < 0 or p + n > len(self.b):
            raise H5Error(f"read past the end of the file at {p}")
        return int.from_bytes(self.b[p:p + n], "little")

    def _addr(self, p: int) -> int:
        return self._u(p, self.so)

    def _len(self, p: int) -> int:
        return self._u(p, self.sl)

    def _abs(self, a: int) -> int:
        return a + self.base_addr

    # --- object headers --------------------------------------------------
    def _messages(self, addr: int) -> list:
        """(type, data position, size) of every message of the version 1
        object header at `addr`, continuation blocks included."""
        if addr in self._headers:
            return self._headers[addr]
        p = self._abs(addr)
        if self.b[p:p + 4] == b"OHDR":
            raise H5Error("version 2 object headers are not read")
        if self._u(p, 1) != 1:
            raise H5Error(f"object header version {self.b[p]} at {addr:#x}")
        nmsg = self._u(p + 2, 2)
        # version, reserved, message count (2), reference count (4), header size (4), padding to 8
        blocks = [(p + 16, self._u(p + 8, 4))]
        out = []
        while blocks and len(out) < nmsg:
            q, n = blocks.pop(0)
            end = q + n
            while q + 8 <= end and len(out) < nmsg:
                mtype, msize = self._u(q, 2), self._u(q + 2, 2)
                d = q + 8                      # type (2), size (2), flags (1), reserved (3)
                if mtype == _MSG_CONTINUATION:
                    blocks.append((self._abs(self._addr(d)), self._len(d + self.so)))
                out.append((mtype, d, msize))
                q = d + msize
        self._headers[addr] = out
        return out

    # --- groups ------------------------------------------------------------
    def _heap_name(self, heap_addr: int, off: int) -> str:
        h = self._abs(heap_addr)
        if self.b[h:h + 4] != b"HEAP":
            raise H5Error("bad local heap")
        # signature, version, reserved (3), data segment size, free-list offset, data segment address
        data = self._abs(self._addr(h + 8 + 2 * self.sl))
        s = data + off
        e = self.b.find(b"\0", s)
        if e < 0:
            raise H5Error("unterminated name in a local heap")
        return self.b[s:e].decode()

    def _btree_group(self, node: int, heap: int, out: dict):
        p = self._abs(node)
        if self.b[p:p + 4] != b"TREE" or self.b[p + 4] != 0:
            raise H5Error("bad group B-tree node")
        level, used = self.b[p + 5], self._u(p + 6, 2)
        q = p + 8 + 2 * self.so                # after the left and right sibling addresses
        for i in range(used):
            # key i (a heap offset, size-of-lengths bytes), then child i
            child = self._addr(q + self.sl + i * (self.sl + self.so))
            if level > 0:
                self._btree_group(child, heap, out)
            else:
                self._snod(child, heap, out)

    def _snod(self, addr: int, heap: int, out: dict):
        p = self._abs(addr)
        if self.b[p:p + 4] != b"SNOD":
            raise H5Error("bad symbol table node")
        n = self._u(p + 6, 2)
        esz = 2 * self.so + 24                 # name offset, header address, cache type (4), reserved (4), scratch (16)
        for i in range(n):
            e = p + 8 + i * esz
            out[self._heap_name(heap, self._addr(e))] = self._addr(e + self.so)

    def _links(self, addr: int) -> dict:
        out = {}
        for mtype, d, _ in self._messages(addr):
            if mtype == _MSG_SYMBOL_TABLE:     # B-tree address, local heap address
                self._btree_group(self._addr(d), self._addr(d + self.so), out)
            elif mtype in (_MSG_LINK, _MSG_LINK_INFO):
                raise H5Error("link-message groups are not read")
        return out

    def _resolve(self, path: str) -> int:
        addr = self.root
        for part in [s for s in path.split("/") if s]:
            links = self._links(addr)
            if part not in links:
                raise KeyError(path)
            addr = links[part]
        return addr

    def is_group(self, path: str) -> bool:
        return any(m[0] == _MSG_SYMBOL_TABLE for m in self._messages(self._resolve(path)))

    def keys(self, path: str = "/") -> list:
        if not self.is_group(path):
            raise H5Error(f"{path} is not a group")
        return sorted(self._links(self._resolve(path)))

    def exists(self, path: str) -> bool:
        try:
            self._resolve(path)
            return True
        except KeyError:
            return False

    # --- datasets --------------------------------------------------------
    def _dataspace(self, d: int) -> tuple:
        ver, nd = self.b[d], self.b[d + 1]
        if ver != 1:
            raise H5Error(f"dataspace version {ver}")
        q = d + 8                              # version, rank, flags, reserved (5)
        return tuple(self._len(q + i * self.sl) for i in range(nd))

    def _datatype(self, d: int) -> np.dtype:
        cls = self.b[d] & 0x0F
        bits = self.b[d + 1]
        size = self._u(d + 4, 4)
        order = ">" if bits & 1 else "<"
        if cls == 0:                           # fixed point; bit 3 of the class bits: signed
            return np.dtype(f"{order}{'i' if bits & 0x08 else 'u'}{size}")
        if cls == 1:                           # IEEE floating point
            return np.dtype(f"{order}f{size}")
        if cls == 3:                           # fixed-length string
            return np.dtype(f"S{size}")
        raise H5Error(f"datatype class {cls} is not read")

    def _contiguous(self, d: int):
        ver = self.b[d]
        if ver == 3:
            if self.b[d + 1] != 1:
                raise H5Error(f"layout class {self.b[d + 1]}: only contiguous storage is read")
            return self._addr(d + 2)
        if ver in (1, 2):
            if self.b[d + 2] != 1:
                raise H5Error(f"layout class {self.b[d + 2]}: only contiguous storage is read")
            return self._addr(d + 8)
        raise H5Error(f"layout version {ver}")

    def read(self, path: str) -> np.ndarray:
        shape = dtype = addr = None
        for mtype, d, _ in self._messages(self._resolve(path)):
            if mtype == _MSG_DATASPACE:
                shape = self._dataspace(d)
            elif mtype == _MSG_DATATYPE:
                dtype = self._datatype(d)
            elif mtype == _MSG_LAYOUT:
                addr = self._contiguous(d)
            elif mtype == _MSG_FILTERS:
                raise H5Error("filtered storage is not read")
        if shape is None or dtype is None or addr is None:
            raise H5Error(f"{path} is not a dataset")
        n = int(np.prod(shape)) if shape else 1
        if addr == _UNDEF:                     # never written: the default fill value, zero
            arr = np.zeros(n, dtype)
        else:
            s = self._abs(addr)
            if s + n * dtype.itemsize > len(self.b):
                raise H5Error(f"{path}: data past the end of the file")
            arr = np.frombuffer(self.b, dtype, count=n, offset=s).copy()
        if dtype.byteorder == ">":
            arr = arr.astype(dtype.newbyteorder("<"))
        return arr.reshape(shape) if shape else arr.reshape(())
