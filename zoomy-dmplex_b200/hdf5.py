"""Minimal HDF5 reading and writing for initial-state files, without an HDF5
library.

The reference loads its initial condition from the HDF5 dataset "state"
(``IOManager.hpp:122-192``, ``VecLoad`` of a Vec named "state"), a flat
float64 array in cell-major order [cell0_var0, cell0_var1, ...] written by
its ``generate_ic.py:104-125`` with h5py: a one-dimensional contiguous
dataset in the root group with the integer attributes ``num_cells`` and
``num_components``.  This module reads that format -- and, more generally,
any contiguous or compact dataset of a fixed-point or IEEE floating-point
type, little or big endian, in a file with a version 0-3 superblock,
symbol-table or link-message groups and version 1 or 2 object headers -- and
writes the same layout (superblock version 0, the root group as a symbol
table, version 1 object headers).  Chunked, compressed and virtual datasets
are rejected with a clear message.

The format is read from the HDF5 File Format Specification (version 2/3
superblocks, object headers, B-trees, local and fractal heaps); only the
structures listed above are implemented.
"""
from __future__ import annotations

import struct
from typing import Dict, Optional, Tuple

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class HDF5Error(ValueError):
    pass


class _File:
    def __init__(self, data: bytes):
        self.b = data
        self.base = self._find_superblock()
        self._parse_superblock()

    # ---------------------------------------------------------- low level
    def _find_superblock(self) -> int:
        off = 0
        while off + 8 <= len(self.b):
            if self.b[off:off + 8] == SIGNATURE:
                return off
            off = 512 if off == 0 else off * 2     # the signature sits at 0, 512, 1024, ...
        raise HDF5Error("not an HDF5 file (no signature)")

    def u(self, pos: int, n: int) -> int:
        if pos + n > len(self.b):
            raise HDF5Error("truncated file")
        return int.from_bytes(self.b[pos:pos + n], "little")

    def addr(self, pos: int) -> int:
        return self.u(pos, self.so)

    def length(self, pos: int) -> int:
        return self.u(pos, self.sl)

    def at(self, a: int) -> int:
        """File position of a relative address."""
        return self.base_addr + a

    # ---------------------------------------------------------- superblock
    def _parse_superblock(self):
        p = self.base + 8
        self.sb_version = self.b[p]
        if self.sb_version in (0, 1):
            self.so, self.sl = self.b[p + 5], self.b[p + 6]
            q = p + 16 + (4 if self.sb_version == 1 else 0)
            self.base_addr = self.u(q, self.so)
            q += 4 * self.so                          # base, free space, end of file, driver info
            # root group symbol table entry: link name offset, object header address, cache
            self.root = self.u(q + self.so, self.so)
        elif self.sb_version in (2, 3):
            self.so, self.sl = self.b[p + 1], self.b[p + 2]
            q = p + 4
            self.base_addr = self.u(q, self.so)
            self.root = self.u(q + 3 * self.so, self.so)   # base, extension, end of file, root header
        else:
            raise HDF5Error("unsupported superblock version %d" % self.sb_version)

    # ---------------------------------------------------------- object headers
    def messages(self, a: int):
        """(type, position of the message data, size) of an object header."""
        p = self.at(a)
        out = []
        if self.b[p:p + 4] == b"OHDR":                # version 2
            flags = self.b[p + 5]
            q = p + 6
            if flags & 0x20:
                q += 16                               # times
            if flags & 0x10:
                q += 4                                # attribute phase change
            size_bytes = 1 << (flags & 3)
            chunk = self.u(q, size_bytes)
            q += size_bytes
            blocks = [(q, chunk, True)]
            track = bool(flags & 0x04)
            while blocks:
                start, n, first = blocks.pop(0)
                r, end = start, start + n
                while r + 4 <= end:
                    mt, ms = self.b[r], self.u(r + 1, 2)
                    r += 4 + (2 if track else 0)
                    if mt == 0x10:                    # continuation: "OCHK" block
                        ca, cl = self.addr(r), self.length(r + self.so)
                        cp = self.at(ca)
                        if self.b[cp:cp + 4] != b"OCHK":
                            raise HDF5Error("bad object header continuation")
                        blocks.append((cp + 4, cl - 8, False))
                    elif mt != 0:
                        out.append((mt, r, ms))
                    r += ms
            return out
        if self.b[p] != 1:
            raise HDF5Error("unsupported object header version %d" % self.b[p])
        nmsg = self.u(p + 2, 2)
        size = self.u(p + 8, 4)
        blocks = [(p + 16, size)]
        while blocks and len(out) < nmsg:
            start, n = blocks.pop(0)
            r, end = start, start + n
            while r + 8 <= end and len(out) < nmsg:
                mt, ms = self.u(r, 2), self.u(r + 2, 2)
                r += 8
                if mt == 0x10:
                    blocks.append((self.at(self.addr(r)), self.length(r + self.so)))
                out.append((mt, r, ms))
                r += ms
        return [m for m in out if m[0] not in (0, 0x10)]

    # ---------------------------------------------------------- groups
    def links(self, a: int) -> Dict[str, int]:
        """Name -> object header address of the links of group a."""
        res = {}
        for mt, r, ms in self.messages(a):
            if mt == 0x11:                            # symbol table message
                res.update(self._symbol_table(self.addr(r), self.addr(r + self.so)))
            elif mt == 0x06:                          # link message (hard links)
                name, target = self._link(r)
                if name is not None:
                    res[name] = target
            elif mt == 0x02:                          # link info: dense storage in a fractal heap
                raise HDF5Error("groups with dense link storage are not supported")
        return res

    def _link(self, r):
        flags = self.b[r + 1]
        q = r + 2
        ltype = 0
        if flags & 0x08:
            ltype = self.b[q]
            q += 1
        if flags & 0x04:
            q += 8                                    # creation order
        if flags & 0x10:
            q += 1                                    # name character set
        ln = self.u(q, 1 << (flags & 3))
        q += 1 << (flags & 3)
        name = self.b[q:q + ln].decode()
        q += ln
        if ltype != 0:
            return None, None                         # soft / external links are not followed
        return name, self.addr(q)

    def _heap_name(self, heap_data: int, off: int) -> str:
        p = self.at(heap_data) + off
        e = self.b.index(b"\0", p)
        return self.b[p:e].decode()

    def _symbol_table(self, btree: int, heap: int) -> Dict[str, int]:
        hp = self.at(heap)
        if self.b[hp:hp + 4] != b"HEAP":
            raise HDF5Error("bad local heap")
        heap_data = self.addr(hp + 8 + 2 * self.sl)
        res = {}
        stack = [btree]
        while stack:
            n = self.at(stack.pop())
            if self.b[n:n + 4] != b"TREE":
                raise HDF5Error("bad group B-tree node")
            level, used = self.b[n + 5], self.u(n + 6, 2)
            q = n + 8 + 2 * self.so                   # siblings
            q += self.sl                              # key 0
            for _ in range(used):
                child = self.addr(q)
                q += self.so + self.sl                # child, next key
                if level > 0:
                    stack.append(child)
                    continue
                s = self.at(child)
                if self.b[s:s + 4] != b"SNOD":
                    raise HDF5Error("bad symbol table node")
                count = self.u(s + 6, 2)
                e = s + 8
                for _ in range(count):
                    name = self._heap_name(heap_data, self.addr(e))
                    res[name] = self.addr(e + self.so)
                    e += 2 * self.so + 24
        return res

    def resolve(self, path: str) -> int:
        a = self.root
        for part in [x for x in path.split("/") if x]:
            ls = self.links(a)
            if part not in ls:
                raise HDF5Error("no object %r (found: %s)" % (part, ", ".join(sorted(ls)) or "none"))
            a = ls[part]
        return a

    # ---------------------------------------------------------- datasets
    def _dtype(self, r: int):
        cv = self.b[r]
        cls, bits0 = cv & 0x0F, self.b[r + 1]
        size = self.u(r + 4, 4)
        order = ">" if bits0 & 1 else "<"
        if cls == 1:                                  # floating point (IEEE)
            if size not in (4, 8):
                raise HDF5Error("unsupported floating-point size %d" % size)
            return np.dtype(order + ("f4" if size == 4 else "f8"))
        if cls == 0:                                  # fixed point
            signed = bool(bits0 & 0x08)
            return np.dtype(order + ("i" if signed else "u") + str(size))
        raise HDF5Error("unsupported datatype class %d" % cls)

    def _dataspace(self, r: int) -> Tuple[int, ...]:
        v, rank, flags = self.b[r], self.b[r + 1], self.b[r + 2]
        q = r + (8 if v == 1 else 4)
        if v == 2 and self.b[r + 3] == 2:             # null dataspace
            return (0,)
        return tuple(self.length(q + i * self.sl) for i in range(rank))

    def _attr(self, r: int):
        v = self.b[r]
        if v == 1:
            nl, dl, sl = self.u(r + 2, 2), self.u(r + 4, 2), self.u(r + 6, 2)
            pad = lambda n: (n + 7) & ~7
            q = r + 8
            name = self.b[q:q + nl].split(b"\0")[0].decode()
            q += pad(nl)
            dt = self._dtype(q)
            q += pad(dl)
            shape = self._dataspace(q)
            q += pad(sl)
        elif v in (2, 3):
            nl, dl, sl = self.u(r + 2, 2), self.u(r + 4, 2), self.u(r + 6, 2)
            q = r + 8 + (1 if v == 3 else 0)
            name = self.b[q:q + nl].split(b"\0")[0].decode()
            q += nl
            dt = self._dtype(q)
            q += dl
            shape = self._dataspace(q)
            q += sl
        else:
            raise HDF5Error("unsupported attribute message version %d" % v)
        n = int(np.prod(shape)) if shape else 1
        val = np.frombuffer(self.b, dtype=dt, count=n, offset=q).copy()
        return name, (val.reshape(shape) if shape else val[0])

    def dataset(self, path: str):
        a = self.resolve(path)
        dt = shape = layout = None
        attrs = {}
        for mt, r, ms in self.messages(a):
            if mt == 0x01:
                shape = self._dataspace(r)
            elif mt == 0x03:
                dt = self._dtype(r)
            elif mt == 0x08:
                layout = r
            elif mt == 0x0C:
                try:
                    k, v = self._attr(r)
                    attrs[k] = v
                except HDF5Error:
                    pass
            elif mt == 0x0B:
                raise HDF5Error("dataset %r is compressed (filter pipeline): not supported" % path)
        if dt is None or shape is None or layout is None:
            raise HDF5Error("%r is not a dataset" % path)
        n = int(np.prod(shape))
        v = self.b[layout]
        if v == 3:
            lc = self.b[layout + 1]
            if lc == 0:                               # compact
                size = self.u(layout + 2, 2)
                arr = np.frombuffer(self.b[layout + 4:layout + 4 + size], dtype=dt, count=n)
                da = None
            elif lc == 1:                             # contiguous
                da, size = self.addr(layout + 2), self.length(layout + 2 + self.so)
                if da != UNDEF and size < n * dt.itemsize:
                    raise HDF5Error("dataset storage smaller than its shape")
            else:
                raise HDF5Error("dataset %r is chunked or virtual (layout class %d): not supported" % (path, lc))
        elif v in (1, 2):                             # the layout of files from older libraries
            rank, lc = self.b[layout + 1], self.b[layout + 2]
            q = layout + 8
            if lc == 1:
                da = self.addr(q)
            elif lc == 0:
                q += 4 * rank
                size = self.u(q, 4)
                arr = np.frombuffer(self.b[q + 4:q + 4 + size], dtype=dt, count=n)
                da = None
            else:
                raise HDF5Error("dataset %r is chunked (layout class %d): not supported" % (path, lc))
        else:
            raise HDF5Error("unsupported data layout message version %d" % v)
        if da is not None:
            if da == UNDEF:                           # never written: the fill value (0)
                arr = np.zeros(n, dtype=dt)
            else:
                arr = np.frombuffer(self.b, dtype=dt, count=n, offset=self.at(da))
        return arr.astype(dt.newbyteorder("="), copy=True).reshape(shape), attrs


def read_dataset(path: str, name: str = "state"):
    """(array, attributes) of dataset `name` (a path inside the file)."""
    with open(path, "rb") as f:
        return _File(f.read()).dataset(name)


def list_root(path: str):
    """Names of the root group's links."""
    with open(path, "rb") as f:
        h = _File(f.read())
    return sorted(h.links(h.root))


# -------------------------------------------------------------------- writing
def write_state(path: str, q: np.ndarray, name: str = "state"):
    """Write q (n_cells x n_components, or flat) the way the reference's
    generate_ic.py does: a one-dimensional little-endian float64 dataset
    `name` in the root group, contiguous, with the int64 attributes
    num_cells and num_components.  Superblock version 0, the root group a
    symbol table (v1 B-tree + local heap), version 1 object headers."""
    q = np.asarray(q, dtype="<f8")
    if q.ndim == 2:
        nc, ncomp = q.shape
    else:
        nc, ncomp = q.size, 1
    flat = np.ascontiguousarray(q.reshape(-1))
    nm = name.encode() + b"\0"

    def pad8(x):
        return x + b"\0" * ((-len(x)) % 8)

    # layout: superblock (96) | root header | heap header | heap data | B-tree | SNOD | dataset header | data
    SB = 96
    root_hdr_at = SB
    root_msgs = struct.pack("<HHB3x", 0x11, 16, 0) + b"\0" * 16           # symbol table, patched below
    root_hdr = struct.pack("<BBHII", 1, 0, 1, 1, len(root_msgs)) + b"\0" * 4 + root_msgs
    heap_at = root_hdr_at + len(root_hdr)
    heap_data = pad8(b"\0" + nm)                                           # offset 0: the empty name
    heap_hdr_len = 32
    heap_data_at = heap_at + heap_hdr_len
    heap = b"HEAP" + bytes([0, 0, 0, 0]) + struct.pack("<QQQ", len(heap_data), UNDEF, heap_data_at) + heap_data
    btree_at = heap_at + len(heap)
    snod_at = btree_at + 8 + 16 + 8 * 3                                   # one child: key, child, key
    btree = b"TREE" + bytes([0, 0]) + struct.pack("<H", 1) + struct.pack("<QQ", UNDEF, UNDEF) + \
        struct.pack("<QQQ", 0, snod_at, 1)
    # symbol table node with 1 entry (capacity 2K = 8 entries, as the library allocates)
    ds_hdr_at_placeholder = 0
    entry = struct.pack("<QQII", 1, ds_hdr_at_placeholder, 0, 0) + b"\0" * 16
    snod = b"SNOD" + bytes([1, 0]) + struct.pack("<H", 1) + entry + b"\0" * (40 * 7)
    ds_hdr_at = snod_at + len(snod)
    entry = struct.pack("<QQII", 1, ds_hdr_at, 0, 0) + b"\0" * 16
    snod = b"SNOD" + bytes([1, 0]) + struct.pack("<H", 1) + entry + b"\0" * (40 * 7)

    def msg(mt, data, flags=0):
        data = pad8(data)
        return struct.pack("<HHB3x", mt, len(data), flags) + data

    dspace = struct.pack("<BBBB4x", 1, 1, 0, 0) + struct.pack("<Q", flat.size)
    f64 = bytes([0x11, 0x20, 0x3F, 0x00]) + struct.pack("<I", 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
    i64 = bytes([0x10, 0x08, 0x00, 0x00]) + struct.pack("<I", 8) + struct.pack("<HH", 0, 64)
    scalar = struct.pack("<BBBB4x", 1, 0, 0, 0)

    def attr(aname, value):
        an = aname.encode() + b"\0"
        body = struct.pack("<BBHHH", 1, 0, len(an), len(i64), len(scalar))
        return msg(0x0C, body + pad8(an) + pad8(i64) + pad8(scalar) + struct.pack("<q", int(value)))

    fill = struct.pack("<BBBB", 2, 2, 2, 0)                                 # fill value: default, never written
    data_at_placeholder = 0
    msgs = [msg(0x01, dspace), msg(0x03, f64, 1), msg(0x05, fill, 1), None,
            attr("num_cells", nc), attr("num_components", ncomp)]
    lay = lambda a: msg(0x08, struct.pack("<BBQQ", 3, 1, a, flat.nbytes))
    msgs[3] = lay(data_at_placeholder)
    body = b"".join(msgs)
    ds_hdr = struct.pack("<BBHII", 1, 0, len(msgs), 1, len(body)) + b"\0" * 4 + body
    data_at = ds_hdr_at + len(ds_hdr)
    msgs[3] = lay(data_at)
    body = b"".join(msgs)
    ds_hdr = struct.pack("<BBHII", 1, 0, len(msgs), 1, len(body)) + b"\0" * 4 + body
    eof = data_at + flat.nbytes
    root_msgs = struct.pack("<HHB3x", 0x11, 16, 0) + struct.pack("<QQ", btree_at, heap_at)
    root_hdr = struct.pack("<BBHII", 1, 0, 1, 1, len(root_msgs)) + b"\0" * 4 + root_msgs
    root_entry = struct.pack("<QQII", 0, root_hdr_at, 1, 0) + struct.pack("<QQ", btree_at, heap_at)
    sb = SIGNATURE + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", 4, 16, 0) + \
        struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF) + root_entry
    assert len(sb) == SB and len(root_hdr) + SB == heap_at
    out = sb + root_hdr + heap + btree + snod + ds_hdr
    assert len(out) == data_at
    with open(path, "wb") as f:
        f.write(out)
        f.write(flat.tobytes())


def read_state(path: str, n_cells: Optional[int] = None, n_dof_q: Optional[int] = None, name: str = "state"):
    """The "state" dataset as an (n_cells, n_components) array in the file's
    (natural, caller) cell order.  The component count comes from the
    num_components attribute, else from n_dof_q, else from n_cells."""
    a, attrs = read_dataset(path, name)
    a = np.asarray(a, dtype=np.float64).reshape(-1)
    ncomp = int(attrs["num_components"]) if "num_components" in attrs else None
    if ncomp is None:
        if n_dof_q:
            ncomp = n_dof_q
        elif n_cells:
            ncomp = a.size // n_cells
        else:
            raise HDF5Error("cannot tell the component count: no num_components attribute")
    if a.size % ncomp:
        raise HDF5Error("%d values are not a whole number of %d-component cells" % (a.size, ncomp))
    q = a.reshape(-1, ncomp)
    if n_cells is not None and q.shape[0] != n_cells:
        raise HDF5Error("the state holds %d cells, the mesh %d" % (q.shape[0], n_cells))
    return q
