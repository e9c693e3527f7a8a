"""The two layouts of the least-squares stencil (``device.lsq_sell``): every cell keeps
exactly its neighbours, and the slot-shared layout touches fewer distinct rows per
warp-wide gather than manapy's order."""
import numpy as np
import pytest

from manapy_b200 import geometry as G, meshgen, native, reorder as R
from manapy_b200.device import DeviceMesh, lsq_sell, sell32


def _csr(dim, n):
    el, vx = meshgen.cube_tetrahedra(n, seed=1) if dim == 3 else meshgen.square_triangles(n, seed=1)
    A = G.build(el, vx, dim)
    Rn = R.Renumbering(A)
    ptr, idx, _ = Rn.relabel_csr(A["cellnid_ptr"], A["cellnid_idx"], Rn.cperm, Rn.cinv)
    return np.asarray(ptr), np.asarray(idx)


def _rows(gp, gi, n):
    """Per row, its entries in slot order (-1 dropped), and the slot count of each warp."""
    out, slots = [], []
    for g in range(len(gp) - 1):
        blk = np.asarray(gi[gp[g]:gp[g + 1]]).reshape(-1, 32)
        slots.append(blk.shape[0])
        for lane in range(32):
            if 32 * g + lane < n:
                col = blk[:, lane]
                out.append(col[col >= 0])
            else:
                assert np.all(blk[:, lane] == -1)
    return out, slots


def _distinct_per_slot(gp, gi):
    tot = 0
    for g in range(len(gp) - 1):
        for row in np.asarray(gi[gp[g]:gp[g + 1]]).reshape(-1, 32):
            tot += len(np.unique(row[row >= 0]))
    return tot


@pytest.mark.parametrize("dim,n", [(2, 40), (3, 8)])
def test_shared_layout_keeps_every_neighbour_once(dim, n):
    ptr, idx = _csr(dim, n)
    nc = len(ptr) - 1
    gp, gi = lsq_sell(ptr, idx, "shared")
    rows, slots = _rows(gp, gi, nc)
    for i in range(nc):
        assert sorted(rows[i].tolist()) == sorted(idx[ptr[i]:ptr[i + 1]].tolist())
    # as many slots per warp as its longest row: no extra index traffic
    lens = np.diff(ptr)
    for g, L in enumerate(slots):
        assert L == lens[32 * g:32 * g + 32].max()
    # manapy's layout: each row in manapy's order, -1 after it
    mp, mi = lsq_sell(ptr, idx, "manapy")
    mrows, _ = _rows(mp, mi, nc)
    for i in range(nc):
        assert np.array_equal(mrows[i], idx[ptr[i]:ptr[i + 1]])
    # the shared layout gathers far fewer distinct rows
    assert _distinct_per_slot(gp, gi) < 0.6 * _distinct_per_slot(mp, mi)


def test_shared_layout_edge_cases():
    # empty rows, a row longer than the others, a value repeated within one row, 34 rows
    ptr = np.array([0, 0, 3, 3, 9] + [9 + 2 * k for k in range(1, 30)], dtype=np.int64)
    ptr = np.concatenate([ptr, [ptr[-1] + 1]])
    rng = np.random.default_rng(0)
    idx = rng.integers(0, 50, size=int(ptr[-1])).astype(np.int32)
    idx[3:9] = [7, 7, 8, 7, 9, 10]
    gp, gi = native.sell_aligned(ptr, idx)
    n = len(ptr) - 1
    rows, slots = _rows(gp, gi, n)
    for i in range(n):
        assert sorted(rows[i].tolist()) == sorted(idx[ptr[i]:ptr[i + 1]].tolist())
    assert slots == [6, 2]
    gp2, gi2 = native.sell_aligned(ptr, idx, slack=3)
    assert np.diff(gp2).tolist() == [32 * 9, 32 * 5]
    with pytest.raises(ValueError):
        native.sell_aligned(np.array([0, 2]), np.array([1], dtype=np.int32))
    # an all-empty table
    gp3, gi3 = native.sell_aligned(np.zeros(5, dtype=np.int64), np.zeros(0, dtype=np.int32))
    assert gp3.tolist() == [0, 0] and len(gi3) == 0


def test_layout_choice_reaches_the_device_tables():
    el, vx = meshgen.square_triangles(30, seed=2)
    A = G.build(el, vx, 2)
    a = DeviceMesh(A, device=None, stencil="manapy")
    b = DeviceMesh(A, device=None)
    c = DeviceMesh.from_native(el, vx)
    assert b.stencil == c.stencil == "shared" and a.stencil == "manapy"
    gp, gi, _ = sell32(np.asarray(a.t["cellnid_ptr"]), np.asarray(a.t["cellnid_idx"]))
    assert np.array_equal(a.t["lsq_sell_idx"], gi)
    assert np.array_equal(b.t["lsq_sell_idx"], c.t["lsq_sell_idx"])
    assert not np.array_equal(a.t["lsq_sell_idx"], b.t["lsq_sell_idx"])
    with pytest.raises(ValueError):
        DeviceMesh(A, device=None, stencil="sorted")


def test_vertex_sum_lists_keep_cells_and_weights():
    """Tetrahedra: the slot-shared vertex -> cells lists of the edge-sum step hold, per
    vertex, exactly its CSR cells with their centre->vertex weights."""
    el, vx = meshgen.cube_tetrahedra(5, seed=3)
    dm = DeviceMesh(G.build(el, vx, 3), device=None)
    ptr, idx, al = (np.asarray(dm.t[k]) for k in ("n2c_ptr", "n2c_idx", "n2c_alpha"))
    gp, gi, ga = (np.asarray(dm.t[k]) for k in ("n2c_sum_ptr", "n2c_sum_idx", "n2c_sum_alpha"))
    n = len(ptr) - 1
    for g in range(len(gp) - 1):
        bi = gi[gp[g]:gp[g + 1]].reshape(-1, 32)
        ba = ga[gp[g]:gp[g + 1]].reshape(-1, 32)
        for lane in range(32):
            r = 32 * g + lane
            col, wts = bi[:, lane], ba[:, lane]
            assert np.all(wts[col < 0] == 0)
            got = sorted(zip(col[col >= 0].tolist(), wts[col >= 0].tolist()))
            ref = sorted(zip(idx[ptr[r]:ptr[r + 1]].tolist(), al[ptr[r]:ptr[r + 1]].tolist())) if r < n else []
            assert got == ref


def test_edge_tables_of_a_tetrahedral_mesh():
    """cell_edges names the edge of each local vertex pair, edge_origin its vertex of
    smaller index, and each edge's cell list holds exactly the cells that contain it."""
    el, vx = meshgen.cube_tetrahedra(4, seed=2)
    dm = DeviceMesh(G.build(el, vx, 3), device=None)
    vt = np.asarray(dm.t["cell_vtx"]).astype(np.int64)
    ce = np.asarray(dm.t["cell_edges"]).astype(np.int64)
    org = np.asarray(dm.t["edge_origin"]).astype(np.int64)
    gp, gi = np.asarray(dm.t["edge_sell_ptr"]), np.asarray(dm.t["edge_sell_idx"])
    ne, nc = dm.nbedges, dm.nbcells
    assert np.all(ce[:, 6:] == -1) and ce[:, :6].min() == 0 and ce[:, :6].max() == ne - 1
    ends = {}
    for i in range(nc):
        for k, (a, b) in enumerate(DeviceMesh.TET_EDGES):
            e, pair = ce[i, k], tuple(sorted((vt[i, a], vt[i, b])))
            assert ends.setdefault(e, pair) == pair          # one pair per edge id
            assert org[e] == pair[0]
    assert len(ends) == ne and len(set(ends.values())) == ne
    rows, _ = _rows(gp, gi, ne)
    for e in range(ne):
        a, b = ends[e]
        holders = sorted(np.nonzero(np.any(vt == a, axis=1) & np.any(vt == b, axis=1))[0].tolist())
        assert sorted(rows[e].tolist()) == holders
