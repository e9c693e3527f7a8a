"""Tile tables of the staged first phase: every local index maps back to the same global
stencil entry and node incidence, in the same order, for 2D and 3D meshes."""
import numpy as np
import pytest

from manapy_b200 import geometry as G, tiles, workloads as W
from manapy_b200.device import DeviceMesh


def _local_to_global(tt, t, l, nc):
    c0 = t * tiles.TILE
    if l < tiles.TILE:
        return c0 + l
    return int(tt["tile_halo_idx"][tt["tile_halo_ptr"][t] + l - tiles.TILE])


@pytest.mark.parametrize("wl", [W.C2.scaled(n=24), W.C4.scaled(n=7)])
def test_tile_tables_reproduce_the_stencils_and_node_lists(wl):
    el, vx = wl.mesh()
    dm = DeviceMesh(G.build(el, vx, wl.dim), device=None)
    T = dm.t
    assert "lsq_loc" in T and "tile_halo_max" in T
    nc = dm.nbcells
    tt = {k: np.asarray(v) for k, v in T.items()}
    ptr, idx = tt["cellnid_ptr"], tt["cellnid_idx"]
    gp, loc = tt["lsq_sell_ptr"], tt["lsq_loc"]
    for i in range(nc):
        t, lane = i // tiles.TILE, i % 32
        L = (gp[i // 32 + 1] - gp[i // 32]) // 32
        got = []
        for k in range(L):
            v = int(loc[gp[i // 32] + 32 * k + lane])
            if v != 0xFFFF:
                got.append(_local_to_global(tt, t, v, nc))
        assert got == list(idx[ptr[i]:ptr[i + 1]]), i
    # halo lists: ascending, outside their tile, and no larger than the recorded maximum
    hp = tt["tile_halo_ptr"]
    for t in range(len(hp) - 1):
        h = tt["tile_halo_idx"][hp[t]:hp[t + 1]]
        assert np.all(np.diff(h) > 0) and np.all(h // tiles.TILE != t)
    assert int(tt["tile_halo_max"][0]) == int(np.diff(hp).max())
    # nodes: each in the tile of its smallest incident cell, incidences mapped in n2c order
    npt, nid = tt["n2c_ptr"], tt["n2c_idx"]
    tp, tn = tt["tile_node_ptr"], tt["tile_node_idx"]
    assert sorted(tn.tolist()) == list(range(dm.nbnodes))
    for t in range(len(tp) - 1):
        for n in tn[tp[t]:tp[t + 1]]:
            cells = nid[npt[n]:npt[n + 1]]
            assert cells.min() // tiles.TILE == t
            got = [_local_to_global(tt, t, int(tt["n2c_loc"][e]), nc) for e in range(npt[n], npt[n + 1])]
            assert got == list(cells)


def test_a_union_beyond_the_shared_memory_gives_no_tiles():
    wl = W.C2.scaled(n=16)
    el, vx = wl.mesh()
    dm = DeviceMesh(G.build(el, vx, 2), device=None, reorder=False)   # scattered numbering: large unions
    T = {k: np.asarray(v) for k, v in dm.t.items()}
    assert tiles.tile_tables(T, dm.nbcells, max_union=tiles.TILE + 8) is None
