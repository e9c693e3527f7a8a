"""Edge cases through the public API against the oracle: the smallest meshes (every
cell a boundary cell), zero velocity, zero diffusion at order 2, every boundary kind,
a source term, and shallow water at rest (the well-balanced lake)."""
import numpy as np
import pytest

from conftest import rel_max
import manapy_b200 as M
from manapy_b200 import boundary as B, geometry as G, meshgen, workloads as W
import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _run(el, vx, dim, bc, vals, D, order, vel, steps, src=None, init=None):
    dom = M.Domain(dim=dim, mesh=(el, vx))
    w = M.Variable(domain=dom, BC=bc, values=vals)
    vs = [M.Variable(domain=dom) for _ in range(3)]
    for var, a in zip(vs, vel(dom.faces.center)):
        var.face = a
        var.interpolate_facetocell()
    cc = dom.cells.center
    w.cell = init(cc) if init else np.exp(-((cc[:, 0] - 0.4) ** 2 + (cc[:, 1] - 0.6) ** 2) / 0.05)
    S = M.AdvectionDiffusionSolver(w, vel=tuple(vs), conf=M.Struct(Dxx=D, Dyy=D, Dzz=D if dim == 3 else 0.,
                                                                    order=order, cfl=0.5))
    if src is not None:
        w.source = src(cc)  # after the solver: constructing it resets the source term, as in manapy
    A = G.build(el, vx, dim)
    o = O.AdvDiffOracle(A, B.resolve(A, bc, vals), D, D, D if dim == 3 else 0., order=order, cfl=0.5)
    o.set_velocity(*vel(A["faces_center"]))
    o.w[:] = init(A["cells_center"]) if init else np.exp(-((A["cells_center"][:, 0] - 0.4) ** 2 +
                                                           (A["cells_center"][:, 1] - 0.6) ** 2) / 0.05)
    if src is not None:
        o.src[:] = src(A["cells_center"])
    for _ in range(steps):
        S.stepper(); S.compute_fluxes(); S.compute_new_val()
        o.step()
    return w.cell, o.w


def _vel(fc):
    return 0.8 + 0 * fc[:, 0], -0.3 + 0 * fc[:, 0], 0 * fc[:, 0]


SIDES2 = ("in", "out", "upper", "bottom")


@pytest.mark.parametrize("n", [2, 3, 4])  # n = 1: the bottom edge joins tags 1 and 2, which
                                          # name no side (manapy rejects that mesh too)
@pytest.mark.parametrize("order", [1, 2])
def test_smallest_meshes(n, order, cuda):
    el, vx = meshgen.square_triangles(n, seed=n)
    bc = {s: "dirichlet" for s in SIDES2}
    vals = {s: 0.25 for s in SIDES2}
    got, ref = _run(el, vx, 2, bc, vals, 1e-3, order, _vel, 5)
    assert rel_max(got, ref) < TOL


@pytest.mark.parametrize("kinds", [("neumann",) * 4, ("nonslip",) * 4, ("dirichlet", "neumannNH", "neumann", "slip")])
def test_boundary_kinds(kinds, cuda):
    el, vx = meshgen.square_triangles(12, seed=7)
    bc = dict(zip(SIDES2, kinds))
    vals = {s: (0.5 if k in ("dirichlet", "neumannNH") else 0.0) for s, k in bc.items()}
    got, ref = _run(el, vx, 2, bc, vals, 2e-3, 2, _vel, 8)
    assert rel_max(got, ref) < TOL


def test_zero_velocity_pure_diffusion(cuda):
    el, vx = meshgen.square_triangles(14, seed=2)
    bc = {s: "dirichlet" for s in SIDES2}
    vals = {s: 0.0 for s in SIDES2}
    zero = lambda fc: (0 * fc[:, 0], 0 * fc[:, 0], 0 * fc[:, 0])  # noqa: E731
    got, ref = _run(el, vx, 2, bc, vals, 5e-3, 2, zero, 6)
    assert rel_max(got, ref) < TOL


def test_zero_diffusion_order2_with_source(cuda):
    el, vx = meshgen.square_triangles(14, seed=3)
    bc = {s: "neumann" for s in SIDES2}
    vals = {}
    src = lambda cc: np.sin(3 * cc[:, 0]) * np.cos(2 * cc[:, 1])  # noqa: E731
    got, ref = _run(el, vx, 2, bc, vals, 0.0, 2, _vel, 7, src=src)
    assert rel_max(got, ref) < TOL


def test_tetrahedra_smallest_conforming(cuda):
    el, vx = meshgen.cube_tetrahedra(2, seed=1)
    sides = ("in", "out", "upper", "bottom", "front", "back")
    bc = {s: "dirichlet" for s in sides}
    vals = {s: 0.1 for s in sides}
    vel3 = lambda fc: (0.5 + 0 * fc[:, 0], 0.2 + 0 * fc[:, 0], -0.4 + 0 * fc[:, 0])  # noqa: E731
    got, ref = _run(el, vx, 3, bc, vals, 1e-3, 2, vel3, 4)
    assert rel_max(got, ref) < TOL


def test_lake_at_rest_initial_state(cuda):
    """h + Z constant, no velocity, a bump in the bed: FP64 against the oracle, and the
    FP32-compensated step within its stated tolerance (manapy's source term reads the
    last cell for boundary cells, so the lake is not exactly at rest near the walls)."""
    el, vx = meshgen.square_triangles(16, seed=5)
    A = G.build(el, vx, 2)

    def state(cc):
        Z = 0.1 * np.exp(-((cc[:, 0] - 0.5) ** 2 + (cc[:, 1] - 0.5) ** 2) / 0.02)
        return [1.0 - Z, 0 * Z, 0 * Z, 0 * Z, Z]

    so = O.ShallowWaterOracle(A, order=1, cfl=0.5, grav=9.81)
    for k, a in zip(("h", "hu", "hv", "hc", "Z"), state(A["cells_center"])):
        so.state()[k][:] = a
    for _ in range(20):
        so.step()
    for precision, tol in (("fp64", TOL), ("fp32c", 1e-5)):
        dom = M.Domain(dim=2, mesh=(el, vx))
        vs = [M.Variable(domain=dom) for _ in range(5)]
        for var, a in zip(vs, state(dom.cells.center)):
            var.cell = a
        S = M.ShallowWaterSolver(vs[0], hvel=(vs[1], vs[2]), hc=vs[3], Z=vs[4],
                                 conf=M.Struct(order=1, cfl=0.5, precision=precision))
        S.advance(20)
        assert rel_max(vs[0].cell, so.h) < tol, precision
        # near rest the momenta are rounding-level: compare them on the scale of h
        for k, var in zip(("hu", "hv"), vs[1:3]):
            ref = so.state()[k]
            assert np.max(np.abs(var.cell - ref)) / np.abs(so.h).max() < tol, (precision, k)
