"""Host mesh builder against the reference Domain arrays (golden vectors)."""
import numpy as np
import pytest

from conftest import golden, rel_max
from manapy_b200 import geometry as G, meshgen

TABLES = {"cells_cellnid": ("cellnid_ptr", "cellnid_idx"), "cells_ghostnid": ("ghostnid_ptr", "ghostnid_idx"),
          "nodes_cellid": ("n2c_ptr", "n2c_idx"), "nodes_ghostid": ("n2g_ptr", "n2g_idx")}


@pytest.mark.parametrize("name,dim", [("dom2d", 2), ("dom3d", 3)])
def test_domain_arrays_match_reference(name, dim):
    g = golden(name)
    A = G.build(g["in_elements"], g["in_vertex"], dim)
    for key in g.files:
        if key.startswith("in_"):
            continue
        mine = G.padded_from_csr(A[TABLES[key][0]], A[TABLES[key][1]]) if key in TABLES else np.asarray(A[key])
        ref = g[key]
        assert mine.shape == ref.shape, key
        if ref.dtype.kind in "iu":
            assert np.array_equal(mine, ref), key          # connectivity: bit-exact
        else:
            tol = 1e-13 if key == "faces_dist_ortho" else 1e-15
            assert rel_max(mine, ref) <= tol, key          # FP64 geometry: rounding only


def test_mesh_sizes():
    for n in (1, 3, 10):
        el, vx = meshgen.square_triangles(n, seed=n)
        A = G.build(el, vx, 2)
        s = meshgen.mesh_sizes_2d(n)
        assert (A["nbcells"], A["nbfaces"], A["nbnodes"]) == (s["cells"], s["faces"], s["nodes"])
        assert np.all(A["cells_volume"] > 0)
        assert abs(A["cells_volume"].sum() - 1.0) < 1e-12
    for n in (1, 2, 4):
        el, vx = meshgen.cube_tetrahedra(n, seed=n)
        A = G.build(el, vx, 3)
        assert A["nbcells"] == 6 * n ** 3
        # conforming split: Nf = 2 Nc + (boundary faces) / 2
        nb = int(np.sum(A["faces_cellid"][:, 1] == -1))
        assert A["nbfaces"] == 2 * A["nbcells"] + nb // 2
        # a single hex has faces whose vertex tags match no side (manapy names them 100)
        assert (len(A["unmatched_boundary_faces"]) > 0) == (n == 1)
        assert abs(A["cells_volume"].sum() - 1.0) < 1e-12


def test_meshgen_is_seeded():
    a = meshgen.square_triangles(5, seed=3)
    b = meshgen.square_triangles(5, seed=3)
    c = meshgen.square_triangles(5, seed=4)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[1], c[1])


def test_face_names_and_lists():
    el, vx = meshgen.square_triangles(7, seed=2)
    A = G.build(el, vx, 2)
    for lst, tag in (("infaces", 1), ("outfaces", 2), ("upperfaces", 3), ("bottomfaces", 4)):
        assert len(A[lst]) == 7 and np.all(A["faces_name"][A[lst]] == tag)
    assert len(A["unmatched_boundary_faces"]) == 0
    # every cell's outward normals close (divergence theorem on a constant)
    cf = A["cells_faceid"][:, :3]
    s = A["cells_nf"].sum(axis=1)
    assert np.max(np.abs(s)) < 1e-15


def test_rejects_mixed_elements():
    el, vx = meshgen.square_triangles(2, seed=0)
    el = el.copy()
    el[0, -1] = 4
    with pytest.raises(ValueError):
        G.build(el, vx, 2)
