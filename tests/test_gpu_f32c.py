"""FP32-compensated advection-diffusion step (``precision="fp32c"``) against the FP64 oracle.

Stated tolerances (relative, over all cells, after the whole run):
L2 = ||w - w_ref||_2 / ||w_ref||_2 <= 1e-7 and Linf = max|w - w_ref| / max|w_ref| <= 2e-7.
The state is FP32 plus its FP32 rounding error (the update is an exact two-sum), so no
increment is lost from step to step; what remains is FP32 rounding of each step's
residual, evaluated on differences from the cell's own value with compensated face
sums (measured: 5e-9 L2 after 1,003 steps of the 2,000,000-cell C2 run).
"""
import numpy as np
import pytest

from conftest import rel_max
import manapy_b200 as M
from manapy_b200 import boundary as B, geometry as G, workloads as W
import oracle as O

pytestmark = pytest.mark.gpu
L2_TOL = 1e-7
LINF_TOL = 2e-7


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def _api(el, vx, wl, precision, **conf):
    dom = M.Domain(dim=wl.dim, mesh=(el, vx))
    w = M.Variable(domain=dom, BC=wl.bc, values=wl.bc_values)
    vel = [M.Variable(domain=dom) for _ in range(3)]
    for var, a in zip(vel, wl.velocity(dom.faces.center)):
        var.face = a
        var.interpolate_facetocell()
    w.cell = wl.init(dom.cells.center)
    S = M.AdvectionDiffusionSolver(w, vel=tuple(vel), conf=M.Struct(
        Dxx=wl.diffusion[0], Dyy=wl.diffusion[1], Dzz=wl.diffusion[2], order=wl.order, cfl=wl.cfl,
        precision=precision, **conf))
    return dom, w, S


def _oracle(el, vx, wl):
    A = G.build(el, vx, wl.dim)
    o = O.AdvDiffOracle(A, B.resolve(A, wl.bc, wl.bc_values), *wl.diffusion, order=wl.order, cfl=wl.cfl)
    o.set_velocity(*wl.velocity(A["faces_center"]))
    o.w[:] = wl.init(A["cells_center"])
    return o


CASES = [W.C1.scaled(n=60, steps=100), W.C2.scaled(n=120, steps=200), W.C4.scaled(n=10, steps=40),
         W.C4.scaled(n=8, steps=20, order=1)]


@pytest.mark.parametrize("wl", CASES, ids=lambda wl: "%s-n%d-o%d" % (wl.name[:2], wl.n, wl.order))
def test_fp32c_error_vs_fp64_oracle(wl, cuda):
    el, vx = wl.mesh()
    dom, w, S = _api(el, vx, wl, "fp32c")
    o = _oracle(el, vx, wl)
    S.advance(wl.steps, graph=True)
    for _ in range(wl.steps):
        o.step()
    l2, linf = rel_l2(w.cell, o.w), rel_max(w.cell, o.w)
    print("%s fp32c after %d steps: L2 %.2e Linf %.2e" % (wl.name, wl.steps, l2, linf))
    assert l2 <= L2_TOL and linf <= LINF_TOL, (l2, linf)


def test_fp32c_tetrahedra_edge_sums_match_stencil_gather(cuda):
    """Second-order FP32c on tetrahedra: the least-squares sums by inclusion-exclusion over
    vertex and edge sums (FP64 sums of the FP32 state, the default) and the gather of each
    cell's whole stencil (lsq_sums=False) agree to FP32 rounding, and both meet the oracle
    tolerance."""
    wl = W.C4.scaled(n=10, steps=30)
    el, vx = wl.mesh()
    o = _oracle(el, vx, wl)
    for _ in range(wl.steps):
        o.step()
    res = {}
    for sums in (True, False):
        dom, w, S = _api(el, vx, wl, "fp32c", lsq_sums=sums)
        S.advance(wl.steps, graph=True)
        assert bool(S._dm.struct.cell_edges) == sums
        res[sums] = np.array(w.cell)
        l2, linf = rel_l2(res[sums], o.w), rel_max(res[sums], o.w)
        print("C4 n=10 fp32c lsq_sums=%s after %d steps: L2 %.2e Linf %.2e" % (sums, wl.steps, l2, linf))
        assert l2 <= L2_TOL and linf <= LINF_TOL, (sums, l2, linf)
    assert rel_l2(res[True], res[False]) <= L2_TOL


def test_fp32c_manapy_loop_and_graph_agree_bitwise(cuda):
    wl = W.C2.scaled(n=40, steps=9)
    el, vx = wl.mesh()
    _, w1, S1 = _api(el, vx, wl, "fp32c")
    _, w2, S2 = _api(el, vx, wl, "fp32c")
    _, w3, S3 = _api(el, vx, wl, "fp32c")
    S1.advance(wl.steps, graph=True)
    S2.advance(wl.steps, graph=False)
    for _ in range(wl.steps):
        S3.stepper(); S3.compute_fluxes(); S3.compute_new_val()
    assert np.array_equal(w1.cell, w2.cell)
    assert np.array_equal(w1.cell, w3.cell)


def test_fp32c_reads_and_writes_between_steps(cuda):
    """Reading w.cell between steps changes nothing; writing it restarts from the new values."""
    wl = W.C2.scaled(n=30, steps=6)
    el, vx = wl.mesh()
    _, w1, S1 = _api(el, vx, wl, "fp32c")
    _, w2, S2 = _api(el, vx, wl, "fp32c")
    for k in range(wl.steps):
        S1.stepper(); S1.compute_fluxes(); S1.compute_new_val()
        _ = w1.cell  # read: FP32 state converted once, exactly
        S2.stepper(); S2.compute_fluxes(); S2.compute_new_val()
    assert np.array_equal(w1.cell, w2.cell)
    x = w1.cell * 0.5
    w1.cell = x
    w2.cell = x
    S1.advance(3)
    S2.advance(3, graph=True)
    assert np.array_equal(w1.cell, w2.cell)
    assert np.all(np.isfinite(w1.cell))


def test_fp32c_intermediates_follow_the_fp32_state(cuda):
    """manapy's intermediate arrays stay readable in fp32c mode (evaluated in FP64 from the FP32 input)."""
    wl = W.C2.scaled(n=32, steps=3)
    el, vx = wl.mesh()
    dom, w, S = _api(el, vx, wl, "fp32c")
    S.stepper(); S.compute_fluxes(); S.compute_new_val()
    w_in = w.cell.copy()
    S.stepper(); S.compute_fluxes(); S.compute_new_val()
    o = _oracle(el, vx, wl)
    o.w[:] = w_in
    o.stepper()
    o.compute_fluxes()
    assert rel_max(w.convective, o.rez) < 1e-13
    assert rel_max(w.dissipative, o.dissip) < 1e-13


def _sw_api(el, vx, wl, precision):
    dom = M.Domain(dim=2, mesh=(el, vx))
    vs = [M.Variable(domain=dom) for _ in range(5)]
    for var, a in zip(vs, wl.init_sw(dom.cells.center)):
        var.cell = a
    S = M.ShallowWaterSolver(vs[0], hvel=(vs[1], vs[2]), hc=vs[3], Z=vs[4],
                             conf=M.Struct(order=wl.order, cfl=wl.cfl, grav=wl.grav, precision=precision))
    return dom, vs, S


# shallow water (compensated state as above; the SRNH flux itself in FP32): hu, hv start
# at zero, so their errors are relative to the largest |hu|, |hv| reached.  Measured:
# h 3e-8, hu / hv up to 5.8e-6 (L2) and 4.3e-6 (Linf) here; 6.5e-6 after 503 steps at 8M cells
SW_L2_TOL = 1e-5
SW_LINF_TOL = 1e-5


@pytest.mark.parametrize("n,steps", [(40, 60), (100, 150)])
def test_fp32c_shallow_water_vs_fp64_oracle(n, steps, cuda):
    wl = W.C3.scaled(n=n, steps=steps, order=1)
    el, vx = wl.mesh()
    dom, vs, S = _sw_api(el, vx, wl, "fp32c")
    A = dom.host_arrays
    so = O.ShallowWaterOracle(A, order=1, cfl=wl.cfl, grav=wl.grav)
    for k, a in zip(("h", "hu", "hv", "hc", "Z"), wl.init_sw(A["cells_center"])):
        so.state()[k][:] = a
    m0 = S.mass()
    S.advance(steps)
    for _ in range(steps):
        so.step()
    for k, var in zip(("h", "hu", "hv"), vs[:3]):
        ref = so.state()[k]
        got = var.cell
        assert np.all(np.isfinite(got)), k
        l2, linf = rel_l2(got, ref), rel_max(got, ref)
        print("SW n=%d %s fp32c after %d steps: L2 %.2e Linf %.2e" % (n, k, steps, l2, linf))
        assert l2 <= SW_L2_TOL and linf <= SW_LINF_TOL, (k, l2, linf)
    # the FP64 mass of the FP32 state follows the FP64 oracle's (Neumann walls let mass through)
    m_ref = float(np.sum(so.h * A["cells_volume"]))
    print("SW n=%d mass: start %.15e fp32c %.15e oracle %.15e" % (n, m0, S.mass(), m_ref))
    assert abs(S.mass() - m_ref) / m_ref < 1e-8  # measured 4e-9
