"""Checkpoint and resume (``manapy_b200.checkpoint``): a run stopped, saved, and resumed
in a fresh solver continues bit for bit, in FP64 and FP32-compensated precision, for
advection-diffusion (2D, 3D) and shallow water."""
import numpy as np
import pytest

import manapy_b200 as M
from manapy_b200 import checkpoint, workloads as W

pytestmark = pytest.mark.gpu


def _advdiff(dom, wl, precision):
    w = M.Variable(domain=dom, BC=wl.bc, values=wl.bc_values)
    vel = [M.Variable(domain=dom) for _ in range(3)]
    for var, a in zip(vel, wl.velocity(dom.faces.center)):
        var.face = a
        var.interpolate_facetocell()
    w.cell = wl.init(dom.cells.center)
    S = M.AdvectionDiffusionSolver(w, vel=tuple(vel), conf=M.Struct(
        Dxx=wl.diffusion[0], Dyy=wl.diffusion[1], Dzz=wl.diffusion[2], order=wl.order, cfl=wl.cfl,
        precision=precision))
    return [w], S


def _sw(dom, wl, precision):
    vs = [M.Variable(domain=dom) for _ in range(5)]
    for var, a in zip(vs, wl.init_sw(dom.cells.center)):
        var.cell = a
    S = M.ShallowWaterSolver(vs[0], hvel=(vs[1], vs[2]), hc=vs[3], Z=vs[4],
                             conf=M.Struct(order=1, cfl=wl.cfl, grav=wl.grav, precision=precision))
    return vs[:3], S


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
@pytest.mark.parametrize("wl,make", [(W.C2.scaled(n=40), _advdiff), (W.C4.scaled(n=6), _advdiff),
                                     (W.C3.scaled(n=40), _sw)])
def test_resume_continues_bit_for_bit(tmp_path, wl, make, precision, cuda):
    el, vx = wl.mesh()
    dom = M.Domain(dim=wl.dim, mesh=(el, vx))
    fields, S = make(dom, wl, precision)
    S.advance(9)
    path = str(tmp_path / "ck.npz")
    checkpoint.save(path, S, step=9, time=1.5)
    S.advance(8)
    ref = [f.cell for f in fields]
    fields2, S2 = make(dom, wl, precision)
    step, t = checkpoint.load(path, S2)
    assert (step, t) == (9, 1.5)
    S2.advance(8)
    for a, b in zip(ref, [f.cell for f in fields2]):
        assert np.array_equal(a, b)


def test_a_checkpoint_of_another_mesh_is_refused(tmp_path, cuda):
    wl = W.C2.scaled(n=20)
    el, vx = wl.mesh()
    _, S = _advdiff(M.Domain(dim=2, mesh=(el, vx)), wl, "fp64")
    path = str(tmp_path / "ck.npz")
    checkpoint.save(path, S)
    wl2 = W.C2.scaled(n=22)
    el2, vx2 = wl2.mesh()
    _, S2 = _advdiff(M.Domain(dim=2, mesh=(el2, vx2)), wl2, "fp64")
    with pytest.raises(ValueError):
        checkpoint.load(path, S2)
