"""Device renumbering: tables stay consistent and per-cell lists keep manapy's order."""
import numpy as np
import pytest

from manapy_b200 import geometry as G, meshgen
from manapy_b200.device import DeviceBC, DeviceMesh, cell_order_codes
from manapy_b200.reorder import Renumbering
from manapy_b200 import boundary as B


@pytest.mark.parametrize("dim,n", [(2, 12), (3, 3)])
def test_relabelled_tables_are_consistent(dim, n):
    el, vx = meshgen.square_triangles(n, seed=3) if dim == 2 else meshgen.cube_tetrahedra(n, seed=3)
    A = G.build(el, vx, dim)
    dm = DeviceMesh(A, "cpu", reorder=True)
    R = dm.R
    t = {k: v.numpy() for k, v in dm.t.items()}
    nlf = 3 if dim == 2 else 4
    # permutations are bijections
    for p, inv in ((R.cperm, R.cinv), (R.fperm, R.finv), (R.nperm, R.ninv)):
        assert np.array_equal(np.sort(p), np.arange(len(p)))
        assert np.array_equal(inv[p], np.arange(len(p)))
    # cell -> faces and face -> cells agree with the host tables
    old_faces = A["cells_faceid"][:, :nlf]
    assert np.array_equal(t["cell_faces"][:, :nlf], R.finv[old_faces[R.cperm]])
    fc = A["faces_cellid"]
    new_fc = t["face_cellid"]
    assert np.array_equal(new_fc[R.finv, 0], R.cinv[fc[:, 0]])
    b = fc[:, 1] < 0
    assert np.all(new_fc[R.finv[b], 1] == -1)
    assert np.array_equal(new_fc[R.finv[~b], 1], R.cinv[fc[~b, 1]])
    # cell-neighbour lists keep manapy's order (ascending old id)
    ptr, idx = t["cellnid_ptr"], t["cellnid_idx"]
    for k in range(0, A["nbcells"], max(1, A["nbcells"] // 50)):
        old = R.cperm[k]
        mine = R.cperm[idx[ptr[k]:ptr[k + 1]]]
        ref = A["cellnid_idx"][A["cellnid_ptr"][old]:A["cellnid_ptr"][old + 1]]
        assert np.array_equal(mine, ref)
    # accumulation order codes refer to ascending *manapy* face ids
    assert np.array_equal(t["cell_order"], cell_order_codes(old_faces[R.cperm]))
    # geometry moved with its entity
    assert np.array_equal(t["cell_center"], A["cells_center"][R.cperm])
    assert np.array_equal(t["face_normal"], A["faces_normal"][R.fperm])
    # neighbours are closer in memory after renumbering (locality)
    c0, c1 = new_fc[:, 0], new_fc[:, 1]
    inner = c1 >= 0
    assert np.median(np.abs(c0[inner] - c1[inner])) < np.median(np.abs(fc[~b, 0] - fc[~b, 1]))


def test_cell_at_face_ghost_index_follows_renumbering():
    el, vx = meshgen.square_triangles(10, seed=1)
    A = G.build(el, vx, 2)
    # a dirichlet side listed after a neumann side (bottom faces have small ids)
    bc = B.resolve(A, {"in": "neumann", "bottom": "dirichlet", "upper": "neumann", "out": "neumann"},
                   {"bottom": 1.0})
    caf = np.nonzero(bc.kind == B.G_CELL_AT_FACE)[0]
    assert len(caf) == 10
    dm = DeviceMesh(A, "cpu", reorder=True)
    db = DeviceBC(A, bc, "cpu", mesh=dm)
    v = db.value.numpy()
    assert np.array_equal(v[dm.R.finv[caf]], dm.R.cinv[caf])


def test_sell32_layout_round_trips():
    from manapy_b200.device import sell32
    rng = np.random.default_rng(0)
    cnt = rng.integers(0, 20, size=77)
    ptr = np.zeros(78, dtype=np.int64)
    np.cumsum(cnt, out=ptr[1:])
    idx = rng.integers(0, 1000, size=int(ptr[-1]))
    vals = rng.standard_normal(int(ptr[-1]))
    for fill in (-1, "first"):
        gp, gi, gv = sell32(ptr, idx, vals, fill=fill)
        for r in range(77):
            g, l = divmod(r, 32)
            length = (gp[g + 1] - gp[g]) // 32
            row = gi[gp[g] + 32 * np.arange(length) + l]
            rv = gv[gp[g] + 32 * np.arange(length) + l]
            assert np.array_equal(row[:cnt[r]], idx[ptr[r]:ptr[r + 1]])
            assert np.array_equal(rv[:cnt[r]], vals[ptr[r]:ptr[r + 1]])
            assert np.all(rv[cnt[r]:] == 0)
            if fill == -1:
                assert np.all(row[cnt[r]:] == -1)
            elif cnt[r]:
                assert np.all(row[cnt[r]:] == idx[ptr[r]])


def test_first_cells_are_numbered_first():
    el, vx = meshgen.square_triangles(20, seed=4)
    A = G.build(el, vx, 2)
    base = Renumbering(A)
    first = np.random.default_rng(0).random(A["nbcells"]) < 0.3
    R = Renumbering(A, first=first)
    k = int(first.sum())
    assert np.all(first[R.cperm[:k]]) and not np.any(first[R.cperm[k:]])
    # each group keeps the locality order
    assert np.array_equal(R.cperm[:k], base.cperm[first[base.cperm]])
    assert np.array_equal(R.cperm[k:], base.cperm[~first[base.cperm]])
    assert np.array_equal(R.cinv[R.cperm], np.arange(A["nbcells"]))


@pytest.mark.parametrize("dim,n", [(2, 12), (3, 3)])
def test_cell_scratch_sizes_follow_the_edge_tables(dim, n):
    """Scratch the fused steps need: FP64 4 nbcells (2D) or 8 nbcells (3D), FP32c 4 / 5 nbcells;
    once a tetrahedral struct carries the edge tables, FP64 adds 4 (nbnodes + nbedges) doubles
    and FP32c rounds its records up to 8 floats (32 bytes, where the FP64 sums start) and adds
    8 (nbnodes + nbedges) floats."""
    el, vx = meshgen.square_triangles(n, seed=3) if dim == 2 else meshgen.cube_tetrahedra(n, seed=3)
    dm = DeviceMesh(G.build(el, vx, dim), "cpu", reorder=True)
    nc, nn = dm.nbcells, dm.nbnodes
    assert dm.cell_scratch_size() == (4 if dim == 2 else 8) * nc
    assert dm.cell_scratch_size_f32c() == (4 if dim == 2 else 5) * nc
    assert dm.use_edge_sums() == (dim == 3)
    if dim == 3:
        ne = dm.nbedges
        assert ne > 0 and dm.struct.nbedges == ne
        rec = dm.cell_scratch_size_f32c() - 8 * (nn + ne)
        assert rec >= 5 * nc and rec % 8 == 0 and rec - 5 * nc < 8
        assert dm.cell_scratch_size() == 8 * nc + 4 * (nn + ne)
    else:
        assert dm.cell_scratch_size_f32c() == 4 * nc
