"""CUDABackend.compile: manapy's own kernel argument lists, run on the GPU, against the oracle."""
import numpy as np
import pytest

from conftest import golden, rel_max
import manapy_b200 as M
from manapy_b200 import boundary as B
import oracle as O

pytestmark = pytest.mark.gpu


def _fn(name):
    def f():
        pass
    f.__name__ = name
    return f


@pytest.mark.parametrize("name,dim", [("k2d", 2), ("k3d", 3)])
def test_compiled_kernels_take_manapy_arguments(name, dim, cuda):
    g = golden(name)
    dom = M.Domain(dim=dim, mesh=(g["in_elements"], g["in_vertex"]))
    A = dom.host_arrays
    m = O.Mesh(A)
    be = dom.backend
    bcs = {"in": "dirichlet", "out": "dirichlet", "upper": "neumann", "bottom": "neumann"}
    if dim == 3:
        bcs.update({"front": "nonslip", "back": "neumann"})
    bc = B.resolve(A, bcs, {"in": 0.25, "out": -0.5})
    d = dom
    c, f, n = d.cells, d.faces, d.nodes
    w = g["w_cell"].copy()
    z = np.zeros(0)
    zi = np.zeros((0, 2), np.int32)
    # facetocell
    uc = np.zeros(m.nc)
    be.compile(_fn("facetocell"))(g["u_face"], uc, c.faceid, dim)
    assert rel_max(uc, g["u_cell"]) <= 1e-15
    # ghost values, as Variable.update_ghost_value calls them
    ghost = np.zeros(m.nf)
    be.compile(_fn("ghost_value_dirichlet"))(bc.value, ghost, f.cellid, bc.dirichletfaces, z, f.dist_ortho)
    be.compile(_fn("ghost_value_neumann"))(w, ghost, f.cellid, A["upperfaces"], z, f.dist_ortho)
    be.compile(_fn("ghost_value_neumann"))(w, ghost, f.cellid, A["bottomfaces"], z, f.dist_ortho)
    if dim == 3:
        be.compile(_fn("ghost_value_nonslip"))(w, ghost, f.cellid, A["frontfaces"], z, f.dist_ortho)
        be.compile(_fn("ghost_value_neumann"))(w, ghost, f.cellid, A["backfaces"], z, f.dist_ortho)
    assert rel_max(ghost, g["w_ghost"]) == 0
    # gradient + limiter
    gx, gy, gz, psi = (np.zeros(m.nc) for _ in range(4))
    sfx = "_%dd" % dim
    be.compile(_fn("cell_gradient" + sfx))(w, ghost, z, z, c.center, c.cellnid, c.ghostnid, c.haloghostnid,
                                           c.halonid, c.nodeid, c.periodicnid, n.periodicid, f.ghostcenter,
                                           c.haloghostcenter, n.vertex, d.halos.centvol, c.shift, gx, gy, gz)
    assert rel_max(gx, g["gradx"]) < 1e-13 and rel_max(gy, g["grady"]) < 1e-13
    be.compile(_fn("barthlimiter" + sfx))(w, ghost, z, gx, gy, gz, psi, f.cellid, c.faceid, f.name, f.halofid,
                                          c.center, f.center)
    assert rel_max(psi, g["psi"]) < 1e-13
    node = np.zeros(m.nn)
    be.compile(_fn("centertovertex" + sfx))(w, ghost, z, z, c.center, d.halos.centvol, n.cellid, n.ghostid,
                                            n.haloghostid, n.periodicid, n.halonid, n.vertex, f.ghostcenter,
                                            c.haloghostcenter, n.R_x, n.R_y, n.R_z, n.lambda_x, n.lambda_y,
                                            n.lambda_z, n.number, c.shift, node)
    assert rel_max(node, g["w_node"]) < 1e-13
    gfx, gfy, gfz = (np.zeros(m.nf) for _ in range(3))
    be.compile(_fn("face_gradient" + sfx))(w, ghost, z, g["w_node"], f.cellid, f.nodeid, f.ghostcenter, f.halofid,
                                           c.center, d.halos.centvol, n.vertex, f.airDiamond, f.normal, f.f_1,
                                           f.f_2, f.f_3, f.f_4, c.shift, gfx, gfy, gfz, A["innerfaces"],
                                           d.halofaces, bc.dirichletfaces, bc.neumannfaces,
                                           d.periodicboundaryfaces)
    assert rel_max(gfx, g["gfx"]) < 1e-13 and rel_max(gfy, g["gfy"]) < 1e-13
    for order in (1, 2):
        rez = np.zeros(m.nc)
        be.compile(_fn("explicitscheme_convective" + sfx))(
            rez, w, ghost, z, g["u_face"], g["v_face"], g["wz_face"], g["gradx"], g["grady"], g["gradz"], z, z, z,
            g["psi"], z, c.center, f.center, d.halos.centvol, f.ghostcenter, f.cellid, f.normal, f.halofid, f.name,
            A["innerfaces"], d.halofaces, A["boundaryfaces"], d.periodicboundaryfaces, c.shift, order)
        assert rel_max(rez, g["rez_o%d" % order]) < 1e-13
    D = (1e-3, 2e-3, 3e-3 if dim == 3 else 0.0)
    dis = np.zeros(m.nc)
    be.compile(_fn("explicitscheme_dissipative"))(g["gfx"], g["gfy"], g["gfz"], f.cellid, f.normal, f.name, dis, *D)
    assert rel_max(dis, g["dissip"]) < 1e-13
    dt = be.compile(_fn("time_step"))(g["u_cell"], O.facetocell(m, g["v_face"]), O.facetocell(m, g["wz_face"]),
                                      0.8, f.normal, f.mesure, c.volume, c.faceid, dim, *D)
    assert abs(dt - float(g["dt"])) <= 1e-15 * float(g["dt"])
    w2 = w.copy()
    be.compile(_fn("update_new_value"))(w2, g["rez_o1"], g["dissip"], g["source"], float(g["dt"]), c.volume)
    assert rel_max(w2, g["w_updated"]) < 1e-14


def test_compile_rejects_unknown_kernels_and_foreign_tables(cuda):
    g = golden("k2d")
    dom = M.Domain(dim=2, mesh=(g["in_elements"], g["in_vertex"]))
    with pytest.raises(NotImplementedError):
        dom.backend.compile(_fn("get_triplet_2d"))
    f = dom.backend.compile(_fn("facetocell"))
    with pytest.raises(ValueError):
        f(np.zeros(dom.nbfaces), np.zeros(dom.nbcells), np.zeros((3, 4), np.int32), 2)
    with pytest.raises(TypeError):
        f(np.zeros(dom.nbfaces))


def test_maintainer_path_with_a_reference_built_domain(cuda):
    """CUDABackend.for_manapy_domain on the Domain arrays manapy itself built (dom2d.npz):
    the kernels take manapy's argument lists with the mesh tables of that Domain and give
    the oracle's results (the oracle runs on this package's host tables, which
    tests/test_backend_maintainer.py shows equal manapy's)."""
    import types
    from manapy_b200.backend import CUDABackend
    g = golden("dom2d")
    md = types.SimpleNamespace(dim=2, cells=types.SimpleNamespace(nodeid=g["cells_nodeid"]),
                               nodes=types.SimpleNamespace(vertex=g["nodes_vertex"]))
    be = CUDABackend.for_manapy_domain(md)
    A = be.domain.host_arrays
    m = O.Mesh(A)
    rng = np.random.default_rng(3)
    w = rng.standard_normal(m.nc)
    ghost = rng.standard_normal(m.nf)
    z = np.zeros(0)
    zi = np.zeros((0, 2), np.int32)
    gx, gy, gz = (np.zeros(m.nc) for _ in range(3))
    # arguments as manapy's Variable.compute_cell_gradient passes them, from manapy's Domain
    be.compile(_fn("cell_gradient_2d"))(w, ghost, z, z, g["cells_center"], g["cells_cellnid"], g["cells_ghostnid"],
                                         zi, zi, g["cells_nodeid"], zi, zi, g["faces_ghostcenter"], z,
                                         g["nodes_vertex"], z, z, gx, gy, gz)
    ox, oy, oz = (np.zeros(m.nc) for _ in range(3))
    O.cell_gradient(m, w, ghost, ox, oy, oz)
    assert rel_max(gx, ox) < 1e-13 and rel_max(gy, oy) < 1e-13
    uc = np.zeros(m.nc)
    uf = rng.standard_normal(m.nf)
    be.compile(_fn("facetocell"))(uf, uc, g["cells_faceid"], 2)
    assert rel_max(uc, O.facetocell(m, uf)) <= 1e-15
