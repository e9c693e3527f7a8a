"""VTU output straight from device buffers, written while the solver keeps stepping.

``Domain.save_on_cell_multi`` / ``save_on_node_multi`` (``manapy/ddm/domain.py:735-849``)
take the field values; manapy passes host arrays (``w.cell``) and meshio writes them.
Here the values may be the ``Variable`` itself: its device array is gathered into
manapy's numbering on the compute stream, copied to pinned host memory on a side stream
and written by a background thread.  The files must hold exactly the values the
variable had when the save was issued, in manapy's cell and node numbering.
"""
import numpy as np
import pytest

import manapy_b200 as M
from manapy_b200 import vtu, workloads as W

pytestmark = pytest.mark.gpu


def _solver(wl):
    el, vx = wl.mesh()
    dom = M.Domain(dim=wl.dim, mesh=(el, vx))
    w = M.Variable(domain=dom, BC=wl.bc, values=wl.bc_values)
    vel = [M.Variable(domain=dom) for _ in range(3)]
    for var, a in zip(vel, wl.velocity(dom.faces.center)):
        var.face = a
        var.interpolate_facetocell()
    w.cell = wl.init(dom.cells.center)
    S = M.AdvectionDiffusionSolver(w, vel=tuple(vel), conf=M.Struct(
        Dxx=wl.diffusion[0], Dyy=wl.diffusion[1], Dzz=wl.diffusion[2], order=wl.order, cfl=wl.cfl))
    return dom, w, S


@pytest.mark.parametrize("wl", [W.C2.scaled(n=80), W.C4.scaled(n=8)])
def test_asynchronous_save_from_device_while_stepping(wl, tmp_path, cuda):
    dom, w, S = _solver(wl)
    S.advance(5, graph=True)
    w.interpolate_celltonode()
    fut = dom.save_on_cell_multi(dt=S.dt, time=1.0, niter=5, miter=1, variables=["w"], values=[w],
                                 path=str(tmp_path), asynchronous=True)
    fut_n = dom.save_on_node_multi(niter=5, miter=2, variables=["wn"], values=[w], path=str(tmp_path),
                                   asynchronous=True)
    S.advance(7, graph=True)          # the state moves on while the files are written
    dom.wait_saves()
    assert fut.done() and fut_n.done()
    # what the state was at the save: replay the same steps on a fresh solver
    dom2, w2, S2 = _solver(wl)
    S2.advance(5, graph=True)
    w2.interpolate_celltonode()
    ref_cell, ref_node = w2.cell, w2.node
    k = 3 if wl.dim == 2 else 4
    got = vtu.read_vtu_arrays(str(tmp_path / "visu0-1.vtu"))
    assert np.array_equal(got["w"], ref_cell)
    assert np.array_equal(got["connectivity"].reshape(-1, k), dom.cells.nodeid[:, :k])
    assert np.array_equal(got["Points"], dom.nodes.vertex[:, :3])
    assert np.array_equal(vtu.read_vtu_arrays(str(tmp_path / "visu0-2.vtu"))["wn"], ref_node)
    assert (tmp_path / "visu1.pvtu").exists() and (tmp_path / "visu2.pvtu").exists()
    assert not np.array_equal(w.cell, ref_cell)   # the solver did advance meanwhile


def test_synchronous_save_of_a_device_tensor_matches_the_host_path(tmp_path, cuda):
    import torch
    dom, w, S = _solver(W.C2.scaled(n=30))
    S.advance(3, graph=False)
    host = w.cell
    dom.save_on_cell_multi(miter=1, variables=["w"], values=[torch.from_numpy(host).cuda()], path=str(tmp_path))
    dom.save_on_cell_multi(miter=2, variables=["w"], values=[host], path=str(tmp_path))
    a = vtu.read_vtu_arrays(str(tmp_path / "visu0-1.vtu"))["w"]
    b = vtu.read_vtu_arrays(str(tmp_path / "visu0-2.vtu"))["w"]
    assert np.array_equal(a, b) and np.array_equal(a, host)
