"""Debug check of a mesh's index tables (mb_check_tables): valid meshes pass, and a table
with one planted bad entry is named with the entry's position.  Only the check kernel
reads the corrupted copies; no step runs on them."""
import numpy as np
import pytest
import torch

import manapy_b200 as M
from manapy_b200 import geometry as G, meshgen, workloads as W

pytestmark = pytest.mark.gpu


def _mesh(dim):
    from manapy_b200.device import DeviceMesh
    el, vx = meshgen.square_triangles(24, seed=5) if dim == 2 else meshgen.cube_tetrahedra(5, seed=5)
    return DeviceMesh(G.build(el, vx, dim), "cuda")


def _plant(dm, name, pos, value):
    t = dm.t[name].clone()
    t.view(-1)[pos] = value
    dm.t[name + ".bad"] = t           # keeps the copy alive
    setattr(dm.struct, name, t.data_ptr())


@pytest.mark.parametrize("dim", [2, 3])
def test_valid_meshes_pass(dim, cuda):
    _mesh(dim).check_tables()
    wl = W.C2.scaled(n=20) if dim == 2 else W.C4.scaled(n=4)
    el, vx = wl.mesh()
    dom = M.Domain(dim=dim, mesh=(el, vx), check_tables=True)
    assert dom.device_mesh.nbcells == len(el)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("name,where,value,msg", [
    ("lsq_sell_idx", 37, "nc+7", "lsq_sell_idx: entry 37"),
    ("cell_nbr", 4 * 9 + 1, "-nf-3", "cell_nbr: entry 37"),
    ("face_cellid", 2 * 11 + 1, "nc", "face_cellid: entry 23"),
    ("cell_vtx", 4 * 5, "nn", "cell_vtx: entry 20"),
    ("n2c_sell_idx", 3, "-1", "n2c_sell_idx: entry 3"),
])
def test_a_planted_bad_entry_is_named(dim, name, where, value, msg, cuda):
    dm = _mesh(dim)
    nc, nf, nn = dm.nbcells, dm.nbfaces, dm.nbnodes
    v = {"nc+7": nc + 7, "-nf-3": -nf - 3, "nc": nc, "nn": nn, "-1": -1}[value]
    _plant(dm, name, where, v)
    with pytest.raises(ValueError, match=msg):
        dm.check_tables()


def test_edge_tables_are_checked_when_in_use(cuda):
    dm = _mesh(3)
    assert dm.use_edge_sums()
    dm.check_tables()
    _plant(dm, "edge_sell_idx", 5, dm.nbcells)
    with pytest.raises(ValueError, match="edge_sell_idx: entry 5"):
        dm.check_tables()


def test_offsets_out_of_order_are_named(cuda):
    dm = _mesh(2)
    ptr = dm.t["cellnid_ptr"]
    _plant(dm, "cellnid_ptr", 5, int(ptr[4].item()) - 1)    # the last offset is kept
    with pytest.raises(ValueError, match="cellnid_ptr: entry 5 .* out of order"):
        dm.check_tables()
