"""Locality-preserving renumbering of cells, faces and nodes for the device tables.

manapy's numbering is whatever the mesh file gives (the benchmark meshes
permute their cells at random), so neighbouring cells are scattered in memory
and every gather misses.  The device tables use their own numbering:

* cells sorted along a Morton (Z-order) curve of their centres;
* faces sorted by the smallest new index of their two cells (then by the
  other one), so a block of cells finds its faces in a contiguous range;
* nodes sorted by the smallest new index of their incident cells.

Only the storage order changes.  Every per-cell list keeps manapy's order
(ascending *original* ids), so sums are accumulated in exactly the order
manapy uses.  Fields cross the boundary through ``perm`` (new -> old) and
``inv`` (old -> new) gathers.
"""
from __future__ import annotations

import numpy as np

__all__ = ["morton_cells", "face_order", "node_order", "Renumbering"]


def _part1by1(v):
    v = v.astype(np.uint64) & np.uint64(0xFFFFFFFF)
    v = (v | (v << np.uint64(16))) & np.uint64(0x0000FFFF0000FFFF)
    v = (v | (v << np.uint64(8))) & np.uint64(0x00FF00FF00FF00FF)
    v = (v | (v << np.uint64(4))) & np.uint64(0x0F0F0F0F0F0F0F0F)
    v = (v | (v << np.uint64(2))) & np.uint64(0x3333333333333333)
    v = (v | (v << np.uint64(1))) & np.uint64(0x5555555555555555)
    return v


def _part1by2(v):
    v = v.astype(np.uint64) & np.uint64(0x1FFFFF)
    v = (v | (v << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
    v = (v | (v << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
    v = (v | (v << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
    v = (v | (v << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
    v = (v | (v << np.uint64(2))) & np.uint64(0x1249249249249249)
    return v


def morton_cells(center, dim):
    """Cell order (new -> old) along the Z-order curve of the cell centres."""
    c = np.asarray(center)[:, :dim]
    lo = c.min(axis=0)
    span = np.maximum(c.max(axis=0) - lo, 1e-300)
    bits = 20 if dim == 2 else 20
    q = np.floor((c - lo) / span * ((1 << bits) - 1)).astype(np.int64)
    if dim == 2:
        key = _part1by1(q[:, 0]) | (_part1by1(q[:, 1]) << np.uint64(1))
    else:
        key = _part1by2(q[:, 0]) | (_part1by2(q[:, 1]) << np.uint64(1)) | (_part1by2(q[:, 2]) << np.uint64(2))
    return np.argsort(key, kind="stable")


def face_order(face_cellid, cinv):
    """Face order (new -> old) by (min, max) new index of the face's cells."""
    c0 = cinv[face_cellid[:, 0]]
    c1 = np.where(face_cellid[:, 1] >= 0, cinv[np.maximum(face_cellid[:, 1], 0)], c0)
    lo = np.minimum(c0, c1)
    hi = np.maximum(c0, c1)
    return np.lexsort((hi, lo))


def node_order(n2c_ptr, n2c_idx, cinv, nnodes):
    """Node order (new -> old) by the smallest new index of the incident cells."""
    cnt = np.diff(n2c_ptr)
    node = np.repeat(np.arange(nnodes), cnt)
    first = np.full(nnodes, np.iinfo(np.int64).max, dtype=np.int64)
    np.minimum.at(first, node, cinv[n2c_idx].astype(np.int64))
    return np.argsort(first, kind="stable")


class Renumbering:
    """perm (new -> old) and inv (old -> new) of cells, faces and nodes."""

    def __init__(self, A, enabled=True, first=None):
        """``first``: optional boolean mask of cells numbered before all others (each group
        in the order it would have otherwise)."""
        nc, nf, nn = int(A["nbcells"]), int(A["nbfaces"]), int(A["nbnodes"])
        if enabled:
            self.cperm = morton_cells(A["cells_center"], int(A["dim"]))
        else:
            self.cperm = np.arange(nc)
        if first is not None:
            first = np.asarray(first, dtype=bool)
            self.cperm = np.concatenate([self.cperm[first[self.cperm]], self.cperm[~first[self.cperm]]])
        self.cinv = np.empty(nc, dtype=np.int64)
        self.cinv[self.cperm] = np.arange(nc)
        if enabled:
            self.fperm = face_order(A["faces_cellid"], self.cinv)
            self.nperm = node_order(A["n2c_ptr"], A["n2c_idx"], self.cinv, nn)
        else:
            self.fperm = np.arange(nf)
            self.nperm = np.arange(nn)
        self.finv = np.empty(nf, dtype=np.int64)
        self.finv[self.fperm] = np.arange(nf)
        self.ninv = np.empty(nn, dtype=np.int64)
        self.ninv[self.nperm] = np.arange(nn)
        self.enabled = enabled

    @staticmethod
    def relabel_csr(ptr, idx, row_perm, val_inv):
        """Rows reordered by ``row_perm`` (new -> old), values mapped by ``val_inv``;
        the order of entries within a row is kept.  Returns (ptr, idx, source entry)."""
        cnt = np.diff(ptr)[row_perm]
        nptr = np.zeros(len(row_perm) + 1, dtype=np.int64)
        np.cumsum(cnt, out=nptr[1:])
        starts = np.repeat(ptr[:-1][row_perm], cnt)
        offs = np.arange(int(nptr[-1]), dtype=np.int64) - np.repeat(nptr[:-1], cnt)
        src = starts + offs
        return nptr, val_inv[idx[src]], src
