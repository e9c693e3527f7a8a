"""Mass conservation of the shallow-water step (dam break over a bump, C3's set-up).

The FP64 mass is sum(volume * h).  A finite-volume step changes it only through the
boundary faces: every inner face flux leaves one cell and enters the other, so

    M(t + dt) - M(t) = -dt * sum over boundary faces of the h flux

(``ShallowWaterSolver.boundary_mass_flux``).  With manapy's Neumann-copy walls (what its
``slip`` condition degrades to, ``manapy/boundary/bc.py:59-76``) that boundary flux is the
interior cell's own h u.n and mass leaves or enters; with reflective walls (mirrored
momentum, an addition without a manapy counterpart) the SRNH mass flux through a wall is
zero up to rounding and the mass is conserved.

Tolerances (relative to the initial mass): FP64 1e-12.  FP32-compensated: 1e-7 -- its
per-cell increments are FP32 products, so the inner-face cancellation holds only to FP32
rounding of each cell's increment (about 1e-10 of the mass per step; measured below 1e-8
after the runs here).
"""
import numpy as np
import pytest

import manapy_b200 as M
from manapy_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32c": 1e-7}


def _solver(wl, walls, precision):
    el, vx = wl.mesh()
    dom = M.Domain(dim=2, mesh=(el, vx))
    vs = [M.Variable(domain=dom) for _ in range(5)]
    for var, a in zip(vs, wl.init_sw(dom.cells.center)):
        var.cell = a
    S = M.ShallowWaterSolver(vs[0], hvel=(vs[1], vs[2]), hc=vs[3], Z=vs[4],
                             conf=M.Struct(order=1, cfl=wl.cfl, grav=wl.grav, walls=walls, precision=precision))
    return dom, vs, S


def _run(S, steps):
    m0 = S.mass()
    outflow = 0.0
    for _ in range(steps):
        dt = S.stepper()
        S.compute_fluxes()
        S.compute_new_val()
        outflow += dt * S.boundary_mass_flux()
    return m0, S.mass(), outflow


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_mass_identity_with_neumann_walls(precision, cuda):
    wl = W.C3.scaled(n=200, steps=150)
    _, _, S = _solver(wl, "neumann", precision)
    m0, m1, outflow = _run(S, wl.steps)
    # the walls do pass mass (the copied state has a normal velocity) ...
    assert abs(outflow) > 1e3 * TOL[precision] * m0
    # ... and the mass changes by exactly what they pass
    assert abs((m1 - m0) + outflow) / m0 <= TOL[precision]


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_mass_conserved_with_reflective_walls(precision, cuda):
    wl = W.C3.scaled(n=200, steps=150)
    _, vs, S = _solver(wl, "reflective", precision)
    m0, m1, outflow = _run(S, wl.steps)
    assert abs(outflow) <= TOL[precision] * m0
    assert abs(m1 - m0) / m0 <= TOL[precision]
    assert np.all(np.isfinite(vs[0].cell)) and np.min(vs[0].cell) > 0


def test_reflective_walls_change_only_the_boundary_treatment(cuda):
    """From a state with momentum, one first-order step of the two wall modes differs only in
    the cells that touch a boundary face."""
    wl = W.C3.scaled(n=60, steps=1)
    dom, va, Sa = _solver(wl, "neumann", "fp64")
    _, vb, Sb = _solver(wl, "reflective", "fp64")
    for vs in (va, vb):
        vs[1].cell = np.full(int(dom.nbcells), 0.3)
        vs[2].cell = np.full(int(dom.nbcells), -0.2)
    for S in (Sa, Sb):
        S.stepper()
        S.compute_fluxes()
        S.compute_new_val()
    A = dom.host_arrays
    cid = A["faces_cellid"]
    touching = np.zeros(int(dom.nbcells), bool)
    touching[cid[cid[:, 1] < 0, 0]] = True
    for a, b in zip(va[:3], vb[:3]):
        assert np.array_equal(a.cell[~touching], b.cell[~touching])
    assert not np.array_equal(va[1].cell[touching], vb[1].cell[touching])


def test_unknown_wall_mode_is_rejected(cuda):
    wl = W.C3.scaled(n=4, steps=1)
    el, vx = wl.mesh()
    dom = M.Domain(dim=2, mesh=(el, vx))
    vs = [M.Variable(domain=dom) for _ in range(5)]
    with pytest.raises(ValueError):
        M.ShallowWaterSolver(vs[0], hvel=(vs[1], vs[2]), hc=vs[3], Z=vs[4], conf=M.Struct(walls="slip"))
