"""Tile tables of the shared-memory-staged first phase of the fused step.

The first phase of the step (least-squares cell gradient over each cell's vertex
neighbours, ``manapy/ast/functions2d.py:5-104`` / ``functions3d.py:4-120``, the Barth
limiter and the centre-to-vertex node values, ``functions2d.py:199-276``) reads, for
every cell, the centre and value of ~12 (triangles) or ~60 (tetrahedra) neighbours.
A block of the staged kernel owns one tile of ``TILE`` consecutive cells (device
numbering): it first copies the centre and value of every cell its tile's stencils
touch -- the tile's own cells and a halo -- into shared memory, and then reads each
neighbour from there.  Each neighbour row then crosses the memory system once per
tile instead of once per cell that uses it (on the benchmark meshes 1.6 rows per cell
in 2D against ~25 gathers, 3.8 in 3D against ~120).

Tables (device numbering; ``t`` a tile, local index ``l``: own cell ``c`` of tile
``t`` -> ``c - TILE t``, halo entry ``p`` -> ``TILE + p``):

* ``tile_halo_ptr[ntiles + 1]``, ``tile_halo_idx``: each tile's halo cells, ascending;
* ``lsq_loc``: the least-squares stencils as uint16 local indices, in the SELL-32 layout
  and entry order of ``lsq_sell_idx`` (padding 0xFFFF: the cell itself);
* ``tile_node_ptr[ntiles + 1]``, ``tile_node_idx``: the nodes whose smallest incident cell
  lies in the tile (every cell incident to such a node is a vertex neighbour of that
  cell, hence in the tile's stencil union);
* ``n2c_loc``: uint16 local index (in the node's tile) of every node -> cell incidence,
  in the order of ``n2c_idx`` (manapy's order).

Sums keep manapy's order (stencils and node lists are unchanged), so the staged kernel
computes the same numbers as the unstaged one.  A mesh whose largest union would not
fit ``max_union`` entries gets no tile tables and runs the unstaged kernel.
"""
from __future__ import annotations

import numpy as np

__all__ = ["TILE", "MAX_UNION", "tile_tables"]

TILE = 256
# shared memory per block: (TILE + halo) x (dim + 1) doubles; 2048 entries = 64 KiB in 3D
MAX_UNION = 2048


def tile_tables(T, nc, max_union=MAX_UNION):
    """The tile tables (dict of numpy arrays, plus ``tile_max_halo``) from the device tables
    ``T`` (``cellnid_ptr/idx``, ``n2c_ptr/idx``, ``lsq_sell_ptr``); None if some tile's
    union exceeds ``max_union`` entries."""
    ptr = np.asarray(T["cellnid_ptr"], dtype=np.int64)
    idx = np.asarray(T["cellnid_idx"], dtype=np.int64)
    ntiles = (nc + TILE - 1) // TILE
    cnt = np.diff(ptr)
    row = np.repeat(np.arange(nc, dtype=np.int64), cnt)
    rt = row // TILE
    halo = (idx // TILE) != rt
    keys = np.unique(rt[halo] * nc + idx[halo])            # (tile, halo cell), ascending
    htile = keys // nc
    hptr = np.searchsorted(htile, np.arange(ntiles + 1, dtype=np.int64)).astype(np.int64)
    nhalo = np.diff(hptr)
    if TILE + int(nhalo.max(initial=0)) > max_union:
        return None
    loc = idx - rt * TILE
    loc[halo] = TILE + (np.searchsorted(keys, rt[halo] * nc + idx[halo]) - hptr[rt[halo]])
    # the stencils in lsq_sell's layout: same SELL-32 slots, local values, padding 0xFFFF
    gp = np.asarray(T["lsq_sell_ptr"], dtype=np.int64)
    k = np.arange(len(idx), dtype=np.int64) - np.repeat(ptr[:-1], cnt)
    dest = gp[row // 32] + k * 32 + (row % 32)
    lsq_loc = np.full(int(gp[-1]), 0xFFFF, dtype=np.uint16)
    lsq_loc[dest] = loc
    # nodes: owned by the tile of their smallest incident cell
    nptr = np.asarray(T["n2c_ptr"], dtype=np.int64)
    nidx = np.asarray(T["n2c_idx"], dtype=np.int64)
    nn = len(nptr) - 1
    ncnt = np.diff(nptr)
    owner = np.full(nn, np.iinfo(np.int64).max, dtype=np.int64)
    nrow = np.repeat(np.arange(nn, dtype=np.int64), ncnt)
    np.minimum.at(owner, nrow, nidx)
    otile = owner // TILE
    order = np.argsort(otile, kind="stable")
    tnptr = np.searchsorted(otile[order], np.arange(ntiles + 1, dtype=np.int64))
    et = otile[nrow]                                         # tile of each incidence's node
    own_e = (nidx // TILE) == et
    n2c_loc = np.where(own_e, nidx - et * TILE, 0)
    hk = et[~own_e] * nc + nidx[~own_e]
    pos = np.searchsorted(keys, hk)
    if len(hk) and not np.array_equal(keys[np.minimum(pos, len(keys) - 1)], hk):
        return None                                          # an incident cell outside the union
    n2c_loc[~own_e] = TILE + (pos - hptr[et[~own_e]])
    return {
        "tile_halo_ptr": hptr.astype(np.int32),
        "tile_halo_idx": (keys % nc).astype(np.int32),
        "lsq_loc": lsq_loc,
        "tile_node_ptr": tnptr.astype(np.int32),
        "tile_node_idx": order.astype(np.int32),
        "n2c_loc": n2c_loc.astype(np.uint16),
        "tile_max_halo": int(nhalo.max(initial=0)),
    }
