"""The subset of HDF5 that manapy's per-rank mesh files use, without h5py.

manapy writes a partitioned mesh as ``meshes<P>PROC/mesh<r>.hdf5`` with h5py's
``create_dataset`` (``manapy/partitions/meshpartitioning.py:238-275``) and reads it back in
``read_mesh_file`` (``manapy/ddm/pure_ddm.py:13-102``).  Those files hold numeric
datasets (integer and floating-point, any rank) in the root group, stored contiguously
without filters -- h5py's defaults.  This module reads that subset from the HDF5 file
format specification:

* superblock versions 0-3 (also behind a user block at 512, 1024, ... bytes);
* object headers version 1 and 2 (``OHDR``) with their continuation blocks;
* groups stored as symbol tables (version-1 B-tree of ``SNOD`` nodes + local heap) or as
  compact link messages;
* datasets with a dataspace, a fixed-point or floating-point datatype and a contiguous or
  compact layout.

Anything else (chunked or filtered datasets, dense link storage, other datatype
classes) raises ``NotImplementedError`` naming the feature.  ``write_datasets`` writes
the same subset (superblock 0, a symbol-table root group, contiguous datasets): it is
what the tests use to make files, since h5py is not available.
"""
from __future__ import annotations

import os
import struct

import numpy as np

__all__ = ["H5File", "read_datasets", "write_datasets", "read_mesh_dir"]

_SIG = b"\x89HDF\r\n\x1a\n"
_UNDEF = 0xFFFFFFFFFFFFFFFF


class H5File:
    """Root-group datasets of an HDF5 file: ``names()``, ``shape(name)``, ``dtype(name)``,
    ``read(name)``."""

    def __init__(self, path):
        with open(path, "rb") as f:
            self.buf = f.read()
        b = self.buf
        self.base = None
        off = 0
        while off + 8 <= len(b):
            if b[off:off + 8] == _SIG:
                self.base = off
                break
            off = 512 if off == 0 else off * 2
        if self.base is None:
            raise ValueError("%s is not an HDF5 file" % path)
        v = b[self.base + 8]
        if v in (0, 1):
            self.so, self.sl = b[self.base + 13], b[self.base + 14]
            p = self.base + 24 + (4 if v == 1 else 0)
            p += 4 * self.so                       # base, free space, end of file, driver info
            _, root = self._unpack_addrs(p, 2)     # root symbol table entry: name offset, header
        elif v in (2, 3):
            self.so, self.sl = b[self.base + 9], b[self.base + 10]
            p = self.base + 12
            _, _, _, root = self._unpack_addrs(p, 4)
        else:
            raise NotImplementedError("HDF5 superblock version %d" % v)
        self.links = self._group_links(self._messages(root))

    # ---------------------------------------------------------------- primitives
    def _u(self, p, n):
        return int.from_bytes(self.buf[p:p + n], "little")

    def _unpack_addrs(self, p, count):
        return [self._u(p + k * self.so, self.so) for k in range(count)]

    def _abs(self, addr):
        return self.base + addr

    # ---------------------------------------------------------------- object headers
    def _messages(self, addr):
        """[(type, data bytes)] of the object header at ``addr`` (continuations followed)."""
        p = self._abs(addr)
        b = self.buf
        out = []
        if b[p:p + 4] == b"OHDR":
            flags = b[p + 5]
            q = p + 6
            if flags & 0x20:
                q += 16
            if flags & 0x10:
                q += 4
            w = 1 << (flags & 3)
            size = self._u(q, w)
            q += w
            blocks = [(q, q + size - 4)]            # chunk 0 ends with its checksum
            while blocks:
                s, e = blocks.pop(0)
                while s + 4 <= e:
                    mtype, msize, mflags = b[s], self._u(s + 1, 2), b[s + 3]
                    s += 4 + (2 if flags & 0x04 else 0)
                    data = b[s:s + msize]
                    if mtype == 0x10:
                        a, ln = self._u(s, self.so), self._u(s + self.so, self.sl)
                        blocks.append((self._abs(a) + 4, self._abs(a) + ln - 4))  # "OCHK" ... checksum
                    elif mtype:
                        out.append((mtype, data))
                    s += msize
            return out
        if b[p] != 1:
            raise NotImplementedError("object header version %d" % b[p])
        nmsg = self._u(p + 2, 2)
        size = self._u(p + 8, 4)
        blocks = [(p + 16, p + 16 + size)]
        while blocks and len(out) < nmsg:
            s, e = blocks.pop(0)
            while s + 8 <= e and len(out) < nmsg:
                mtype, msize = self._u(s, 2), self._u(s + 2, 2)
                data = b[s + 8:s + 8 + msize]
                if mtype == 0x10:
                    a, ln = self._u(s + 8, self.so), self._u(s + 8 + self.so, self.sl)
                    blocks.append((self._abs(a), self._abs(a) + ln))
                out.append((mtype, data))
                s += 8 + msize
        return out

    # ---------------------------------------------------------------- groups
    def _group_links(self, msgs):
        links = {}
        for mtype, data in msgs:
            if mtype == 0x11:                       # symbol table: v1 B-tree + local heap
                bt, heap = self._u_bytes(data, 0, self.so), self._u_bytes(data, self.so, self.so)
                self._btree_links(bt, self._heap(heap), links)
            elif mtype == 0x06:                     # link message (compact storage)
                name, addr = self._link(data)
                if addr is not None:
                    links[name] = addr
            elif mtype == 0x02:                     # link info
                flags = data[1]
                q = 2 + (8 if flags & 1 else 0)
                if self._u_bytes(data, q, self.so) != _UNDEF & ((1 << (8 * self.so)) - 1):
                    raise NotImplementedError("groups with dense link storage (fractal heap)")
        return links

    @staticmethod
    def _u_bytes(data, q, n):
        return int.from_bytes(data[q:q + n], "little")

    def _heap(self, addr):
        p = self._abs(addr)
        if self.buf[p:p + 4] != b"HEAP":
            raise ValueError("bad local heap")
        q = p + 8 + 2 * self.sl
        return self._abs(self._u(q, self.so))

    def _name(self, heap_data, off):
        s = heap_data + off
        e = self.buf.index(b"\x00", s)
        return self.buf[s:e].decode()

    def _btree_links(self, addr, heap_data, links):
        p = self._abs(addr)
        b = self.buf
        if b[p:p + 4] != b"TREE" or b[p + 4] != 0:
            raise ValueError("bad group B-tree node")
        level, used = b[p + 5], self._u(p + 6, 2)
        q = p + 8 + 2 * self.so + self.sl          # siblings, then key 0
        for _ in range(used):
            child = self._u(q, self.so)
            q += self.so + self.sl
            if level > 0:
                self._btree_links(child, heap_data, links)
                continue
            c = self._abs(child)
            if b[c:c + 4] != b"SNOD":
                raise ValueError("bad symbol table node")
            n = self._u(c + 6, 2)
            e = c + 8
            for _ in range(n):
                name_off, obj = self._u(e, self.so), self._u(e + self.so, self.so)
                links[self._name(heap_data, name_off)] = obj
                e += 2 * self.so + 24

    def _link(self, data):
        flags = data[1]
        q = 2
        ltype = 0
        if flags & 0x08:
            ltype = data[q]
            q += 1
        if flags & 0x04:
            q += 8
        if flags & 0x10:
            q += 1
        w = 1 << (flags & 3)
        n = self._u_bytes(data, q, w)
        q += w
        name = data[q:q + n].decode()
        q += n
        if ltype != 0:
            return name, None                       # soft / external links are not followed
        return name, self._u_bytes(data, q, self.so)

    # ---------------------------------------------------------------- datasets
    def names(self):
        return sorted(self.links)

    def _describe(self, name):
        if name not in self.links:
            raise KeyError(name)
        shape = dtype = layout = None
        for mtype, data in self._messages(self.links[name]):
            if mtype == 0x01:
                shape = self._dataspace(data)
            elif mtype == 0x03:
                dtype = self._datatype(data)
            elif mtype == 0x08:
                layout = data
            elif mtype == 0x0B and len(data) > 2 and data[1] > 0:
                raise NotImplementedError("filtered (compressed) datasets")
        if shape is None or layout is None:
            raise ValueError("%s is not a dataset" % name)
        return shape, dtype, layout

    def shape(self, name):
        return self._describe(name)[0]

    def dtype(self, name):
        return self._describe(name)[1]

    def read(self, name):
        shape, dtype, layout = self._describe(name)
        if dtype is None:
            raise NotImplementedError("%s: datatype class other than integer or floating point" % name)
        n = int(np.prod(shape)) if shape else 1
        nbytes = n * dtype.itemsize
        ver = layout[0]
        if ver in (3, 4):
            cls = layout[1]
            if cls == 0:
                size = self._u_bytes(layout, 2, 2)
                raw = layout[4:4 + size]
            elif cls == 1:
                addr = self._u_bytes(layout, 2, self.so)
                if addr == (1 << (8 * self.so)) - 1:
                    return np.zeros(shape, dtype=dtype.newbyteorder("="))      # never written
                raw = self.buf[self._abs(addr):self._abs(addr) + nbytes]
            else:
                raise NotImplementedError("%s: chunked or virtual dataset layout" % name)
        elif ver in (1, 2):
            rank, cls = layout[1], layout[2]
            if cls != 1:
                raise NotImplementedError("%s: layout class %d (version %d)" % (name, cls, ver))
            addr = self._u_bytes(layout, 8, self.so)
            raw = self.buf[self._abs(addr):self._abs(addr) + nbytes]
        else:
            raise NotImplementedError("%s: data layout message version %d" % (name, ver))
        if len(raw) < nbytes:
            raise ValueError("%s: truncated data" % name)
        return np.frombuffer(raw, dtype=dtype, count=n).reshape(shape).astype(dtype.newbyteorder("="))

    def _dataspace(self, data):
        ver, rank = data[0], data[1]
        q = 8 if ver == 1 else 4
        return tuple(self._u_bytes(data, q + k * self.sl, self.sl) for k in range(rank))

    @staticmethod
    def _datatype(data):
        cls = data[0] & 0x0F
        bits = data[1] | (data[2] << 8) | (data[3] << 16)
        size = int.from_bytes(data[4:8], "little")
        order = ">" if bits & 1 else "<"
        if cls == 0:
            return np.dtype("%s%s%d" % (order, "i" if bits & 0x08 else "u", size))
        if cls == 1:
            return np.dtype("%sf%d" % (order, size))
        return None


def read_datasets(path):
    """{name: array} of every root-group dataset."""
    f = H5File(path)
    return {k: f.read(k) for k in f.names()}


# -------------------------------------------------------------------- writer (same subset)

def _pad8(b):
    return b + b"\x00" * (-len(b) % 8)


def _dt_message(a):
    dt = a.dtype
    if dt.kind in "iu":
        cls, bits = 0, (0x08 if dt.kind == "i" else 0)
        props = struct.pack("<HH", 0, 8 * dt.itemsize)
    elif dt.kind == "f":
        cls = 1
        if dt.itemsize == 8:
            bits, props = 0x20 | (63 << 8), struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
        else:
            bits, props = 0x20 | (31 << 8), struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
    else:
        raise NotImplementedError("only integer and floating-point datasets are written")
    return bytes([cls | 0x10, bits & 0xFF, (bits >> 8) & 0xFF, (bits >> 16) & 0xFF]) + \
        struct.pack("<I", dt.itemsize) + props


def write_datasets(path, datasets):
    """Write ``{name: numpy array}`` as contiguous little-endian root-group datasets
    (superblock version 0, symbol-table root group)."""
    names = sorted(datasets)
    arrays = {k: np.ascontiguousarray(np.asarray(datasets[k]).astype(
        np.asarray(datasets[k]).dtype.newbyteorder("<"))) for k in names}
    K = 4                                             # group leaf node K: 2K entries per SNOD
    heap_data = b"\x00" * 8                           # offset 0: the empty name
    name_off = {}
    for k in names:
        name_off[k] = len(heap_data)
        heap_data += _pad8(k.encode() + b"\x00")
    heap_data = _pad8(heap_data)
    chunks = [names[i:i + 2 * K] for i in range(0, len(names), 2 * K)] or [[]]
    # layout: superblock | root header | heap header | heap data | B-tree | SNODs | dataset headers | data
    sb_size = 24 + 4 * 8 + 40
    root_hdr = 16 + 8 + 16                            # one symbol table message
    heap_hdr = 32
    p_root = sb_size
    p_heap = p_root + root_hdr
    p_heapdata = p_heap + heap_hdr
    p_btree = p_heapdata + len(heap_data)
    if len(chunks) > 32:
        raise NotImplementedError("more than %d datasets in one group" % (32 * 2 * K))
    bt_size = 24 + 8 + 16 * 32                        # a node sized for 2 x 16 children (internal K)
    p_snod = p_btree + bt_size
    snod_size = 8 + 2 * K * 40
    p_dsh = p_snod + len(chunks) * snod_size
    ds_hdr = {}
    p = p_dsh
    msgs = {}
    for k in names:
        a = arrays[k]
        space = bytes([1, a.ndim, 0, 0]) + b"\x00" * 4 + b"".join(struct.pack("<Q", d) for d in a.shape)
        dtm = _dt_message(a)
        body = b""
        for mtype, data in ((0x01, space), (0x03, dtm), (0x08, None)):
            if data is None:
                data = bytes([3, 1]) + b"\x00" * 16      # address, size filled in below
            data = _pad8(data)
            body += struct.pack("<HHB3x", mtype, len(data), 0) + data
        msgs[k] = body
        ds_hdr[k] = p
        p += 16 + len(body)
    data_addr = {}
    for k in names:
        data_addr[k] = p
        p += -(-arrays[k].nbytes // 8) * 8
    eof = p
    out = bytearray(eof)
    # superblock version 0
    sb = _SIG + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", K, 16, 0)
    sb += struct.pack("<QQQQ", 0, _UNDEF, eof, _UNDEF)
    sb += struct.pack("<QQII", 0, p_root, 1, 0) + struct.pack("<QQ", p_btree, p_heap)
    out[0:len(sb)] = sb
    # root object header (version 1) with its symbol table message
    rh = struct.pack("<BBHII", 1, 0, 1, 1, 24) + b"\x00" * 4
    rh += struct.pack("<HHB3x", 0x11, 16, 0) + struct.pack("<QQ", p_btree, p_heap)
    out[p_root:p_root + len(rh)] = rh
    # local heap
    hh = b"HEAP" + bytes([0, 0, 0, 0]) + struct.pack("<QQQ", len(heap_data), _UNDEF, p_heapdata)
    out[p_heap:p_heap + len(hh)] = hh
    out[p_heapdata:p_heapdata + len(heap_data)] = heap_data
    # B-tree (group node, level 0): key, child, key, ..., child, key
    bt = b"TREE" + bytes([0, 0]) + struct.pack("<H", len(chunks)) + struct.pack("<QQ", _UNDEF, _UNDEF)
    bt += struct.pack("<Q", 0)
    for j, ch in enumerate(chunks):
        bt += struct.pack("<Q", p_snod + j * snod_size)
        bt += struct.pack("<Q", name_off[ch[-1]] if ch else 0)
    out[p_btree:p_btree + len(bt)] = bt
    # symbol table nodes
    for j, ch in enumerate(chunks):
        sn = b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(ch))
        for k in ch:
            sn += struct.pack("<QQII", name_off[k], ds_hdr[k], 0, 0) + b"\x00" * 16
        q = p_snod + j * snod_size
        out[q:q + len(sn)] = sn
    # dataset object headers and data
    for k in names:
        a = arrays[k]
        body = bytearray(msgs[k])
        # the layout message is the last one: version 3, contiguous, address, size
        lay = len(body) - 24
        body[lay:lay + 18] = bytes([3, 1]) + struct.pack("<QQ", data_addr[k] if a.nbytes else _UNDEF, a.nbytes)
        hdr = struct.pack("<BBHII", 1, 0, 3, 1, len(body)) + b"\x00" * 4 + bytes(body)
        out[ds_hdr[k]:ds_hdr[k] + len(hdr)] = hdr
        if a.nbytes:
            out[data_addr[k]:data_addr[k] + a.nbytes] = a.tobytes()
    with open(path, "wb") as f:
        f.write(bytes(out))


# -------------------------------------------------------------------- manapy's mesh directories

def read_mesh_dir(mesh_dir):
    """The whole mesh (elements [nc, k+1] with manapy's count column, vertex [nn, 4]) from
    a ``meshes<P>PROC`` directory written by manapy's partitioner: ``mesh0.hdf5`` alone,
    or the ``P`` rank files reassembled through their ``localcelltoglobal`` /
    ``localnodetoglobal`` maps (each rank's elements hold global node ids,
    ``manapy/partitions/meshpartitioning.py:262-270``)."""
    files = sorted((f for f in os.listdir(mesh_dir) if f.startswith("mesh") and f.endswith(".hdf5")),
                   key=lambda f: int(f[4:-5]))
    if not files:
        raise FileNotFoundError("no mesh<r>.hdf5 in %s" % mesh_dir)
    parts = [read_datasets(os.path.join(mesh_dir, f)) for f in files]
    if len(parts) == 1:
        return parts[0]["elements"].astype(np.int32), parts[0]["nodes"].astype(np.float64)
    nc = sum(len(p["elements"]) for p in parts)
    nn = int(max(int(p["localnodetoglobal"].max()) for p in parts)) + 1
    width = parts[0]["elements"].shape[1]
    elements = np.full((nc, width), -1, dtype=np.int32)
    vertex = np.zeros((nn, parts[0]["nodes"].shape[1]), dtype=np.float64)
    for p in parts:
        elements[p["localcelltoglobal"]] = p["elements"]
        vertex[p["localnodetoglobal"]] = p["nodes"]
    if (elements < 0).any():
        raise ValueError("the rank files do not cover every cell once")
    return elements, vertex
