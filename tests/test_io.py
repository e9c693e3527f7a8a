"""gmsh reader (vertex tags by manapy's rules) and VTU writer, on the CPU."""
import os

import numpy as np
import pytest

import manapy_b200 as M
from manapy_b200 import geometry as G, gmsh, meshgen, vtu


def _boundary(A):
    """Boundary faces with their names (manapy's face names 1-6) as physical tags."""
    b = A["faces_cellid"][:, 1] < 0
    k = A["faces_nodeid"].shape[1] - 1
    nodes = A["faces_nodeid"][b, :k]
    names = A["faces_name"][b]
    return [(int(t), nodes[names == t]) for t in np.unique(names)]


@pytest.mark.parametrize("dim,n", [(2, 9), (3, 3)])
def test_roundtrip_reproduces_elements_and_vertex_tags(tmp_path, dim, n):
    el, vx = meshgen.square_triangles(n, seed=4) if dim == 2 else meshgen.cube_tetrahedra(n, seed=4)
    A = G.build(el, vx, dim)
    path = str(tmp_path / "m.msh")
    gmsh.write_msh(path, el, vx, _boundary(A))
    el2, vx2 = gmsh.read_msh(path, dim)
    assert np.array_equal(el2, el)
    assert np.array_equal(vx2[:, :3], vx[:, :3])
    # vertex tags recomputed from the boundary elements' physical groups
    assert np.array_equal(vx2[:, 3], vx[:, 3])
    dom = M.Domain.from_msh(path, dim)
    assert int(dom.nbcells) == len(el)


def test_tag_precedence():
    # vertex 0 on a tag-3 line and a tag-1 line -> 1; vertex 2 on tags 4 and 5 -> 4;
    # vertex 3 only on tag 6 -> 6; later tag-1/2 writes win over earlier ones
    bnd = [(np.array([[0, 1]]), np.array([3])), (np.array([[0, 4]]), np.array([1])),
           (np.array([[2, 3]]), np.array([5])), (np.array([[2, 5]]), np.array([4])),
           (np.array([[4, 6]]), np.array([2])), (np.array([[3, 7]]), np.array([6]))]
    g = gmsh.vertex_tags(8, bnd)
    assert list(g) == [1, 3, 4, 5, 2, 4, 2, 6]


def test_reads_a_gmsh_41_file_of_the_reference_if_present():
    root = os.environ.get("MANAPY_REFERENCE")
    if not root:
        pytest.skip("MANAPY_REFERENCE (the reference source tree) is not set")
    path = os.path.join(root, "mesh", "carre.msh")
    if not os.path.exists(path):
        pytest.skip("reference mesh not available")
    el, vx = gmsh.read_msh(path, 2)
    A = G.build(el, vx, 2)
    assert len(A["unmatched_boundary_faces"]) == 0
    assert set(np.unique(A["faces_name"])) == {0, 1, 2, 3, 4}
    assert np.isclose(A["cells_volume"].sum(), 1.0)


def test_vtu_cell_and_node_files(tmp_path):
    el, vx = meshgen.square_triangles(6, seed=1)
    dom = M.Domain(dim=2, mesh=(el, vx))
    w = np.arange(int(dom.nbcells), dtype=np.float64)
    dom.save_on_cell_multi(dt=0.1, time=1.0, niter=3, miter=2, variables=["w"], values=[w],
                           path=str(tmp_path))
    arrs = vtu.read_vtu_arrays(str(tmp_path / "visu0-2.vtu"))
    assert np.array_equal(arrs["w"], w)
    assert np.array_equal(arrs["connectivity"].reshape(-1, 3), dom.cells.nodeid[:, :3])
    assert np.array_equal(arrs["Points"], dom.nodes.vertex[:, :3])
    assert set(arrs["types"]) == {5}
    assert (tmp_path / "visu2.pvtu").exists()
    wn = np.linspace(0, 1, int(dom.nbnodes))
    dom.save_on_node_multi(variables=["wn"], values=[wn], miter=3, path=str(tmp_path))
    assert np.array_equal(vtu.read_vtu_arrays(str(tmp_path / "visu0-3.vtu"))["wn"], wn)
