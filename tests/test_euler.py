"""2D Euler (``manapy/solvers/euler/fvm_utils2d.py``): the oracle against golden
vectors of the reference kernels (CPU), and the CUDA kernels against the oracle (GPU)."""
import os

import numpy as np
import pytest

from manapy_b200 import geometry as G
from manapy_b200.workloads import pressure_pulse

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ("rho", "P", "rhou", "rhov", "rhoE")


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(HERE, "golden", "k_euler.npz"))


@pytest.fixture(scope="module")
def mesh(gold):
    import oracle as O
    return O.Mesh(G.build(gold["in_elements"], gold["in_vertex"], 2))


def _q0(gold):
    return [gold[k + "0"].copy() for k in NAMES]


def _close(a, b, rtol):
    scale = max(1.0, float(np.max(np.abs(b))))
    return float(np.max(np.abs(np.asarray(a) - b))) <= rtol * scale


def test_oracle_matches_reference_kernels(gold, mesh):
    import oracle as O
    q = _q0(gold)
    g, ug, vg = O.ghost_neumann_euler_2d(mesh, q)
    for k, a in zip(NAMES, g):
        assert np.array_equal(a, gold["g_" + k]), k
    assert _close(ug, gold["g_u"], 1e-15) and _close(vg, gold["g_v"], 1e-15)
    rez = O.euler_rusanov_2d(mesh, q, g, float(gold["gamma"]))
    for k, a in zip(("rho", "rhou", "rhov", "rhoE"), rez):
        assert np.array_equal(a, gold["rez_" + k]), k          # same operations, same order: bit for bit
    # manapy compiles time_step_euler_2d with fastmath: agreement to rounding
    dt_c = O.time_step_euler_2d(mesh, q, float(gold["cfl"]), float(gold["gamma"]))
    assert _close(dt_c, gold["dt_c"], 1e-14)
    O.update_euler_2d(mesh, q, [gold["rez_" + k] for k in ("rho", "rhou", "rhov", "rhoE")], float(gold["gamma"]),
                      float(gold["dts"][0]))
    for k, a in zip(NAMES, q):
        assert _close(a, gold["new_" + k], 1e-14), k


def test_oracle_run_matches_reference_run(gold, mesh):
    import oracle as O
    q = _q0(gold)
    dts = [O.euler_step_2d(mesh, q, float(gold["cfl"]), float(gold["gamma"])) for _ in range(len(gold["dts"]))]
    assert np.allclose(dts, gold["dts"], rtol=1e-13, atol=0)
    for k, a in zip(NAMES, q):
        assert _close(a, gold["final_" + k], 1e-12), k


# ---------------------------------------------------------------- GPU: the CUDA kernels
def _fn(name):
    def f():
        pass
    f.__name__ = name
    return f


def _solver(el, vx, q0, cfl=0.5, gamma=1.4):
    import manapy_b200 as M
    dom = M.Domain(dim=2, mesh=(el, vx))
    vs = [M.Variable(domain=dom) for _ in NAMES]
    for v, a in zip(vs, q0):
        v.cell = a
    return dom, vs, M.EulerSolver(*vs, conf=M.Struct(cfl=cfl, gamma=gamma))


@pytest.mark.gpu
def test_compiled_kernels_take_manapy_arguments(gold, mesh, cuda):
    """ghost_value_Neumann, explicitscheme_euler_2d_rusanov, time_step_euler_2d and
    update_euler_2d_fvc with manapy's argument lists, bit for bit against the oracle."""
    import manapy_b200 as M
    import oracle as O
    dom = M.Domain(dim=2, mesh=(gold["in_elements"], gold["in_vertex"]))
    be, c, f = dom.backend, dom.cells, dom.faces
    gamma, cfl = float(gold["gamma"]), float(gold["cfl"])
    q = _q0(gold)
    nf, nc = mesh.nf, mesh.nc
    g = [np.zeros(nf) for _ in NAMES]
    ug, vg = np.zeros(nf), np.zeros(nf)
    be.compile(_fn("ghost_value_Neumann"))(g[0], g[1], g[2], g[3], ug, vg, g[4], *q, f.cellid, f.name, f.normal,
                                           f.mesure, f.center, 0.0)
    og, oug, ovg = O.ghost_neumann_euler_2d(mesh, q)
    for k, a, b in zip(NAMES, g, og):
        assert np.array_equal(a, b) and np.array_equal(a, gold["g_" + k]), k
    assert np.array_equal(ug, oug) and np.array_equal(vg, ovg)
    rez = [np.zeros(nc) for _ in range(4)]
    z = np.zeros(1)
    be.compile(_fn("explicitscheme_euler_2d_rusanov"))(*rez, *q, *g, z, z, z, z, z, f.cellid, np.zeros(1, np.int32),
                                                       f.normal, f.mesure, f.name, gamma)
    for k, a in zip(("rho", "rhou", "rhov", "rhoE"), rez):
        assert np.array_equal(a, gold["rez_" + k]), k
    dt_c = np.zeros(nc)
    be.compile(_fn("time_step_euler_2d"))(q[0], q[1], q[2], q[3], cfl, f.normal, f.mesure, c.volume, c.faceid, gamma,
                                          dt_c)
    assert np.array_equal(dt_c, O.time_step_euler_2d(mesh, q, cfl, gamma))
    dt = float(gold["dts"][0])
    be.compile(_fn("update_euler_2d_fvc"))(*q, *rez, gamma, dt, c.volume)
    oq = _q0(gold)
    O.update_euler_2d(mesh, oq, rez, gamma, dt)
    for k, a, b in zip(NAMES, q, oq):
        assert np.array_equal(a, b), k


@pytest.mark.gpu
def test_fused_steps_match_reference_run(gold, mesh, cuda):
    """20 fused steps: the reference run's trajectory, and the oracle's bit for bit."""
    import oracle as O
    _, vs, S = _solver(gold["in_elements"], gold["in_vertex"], _q0(gold), float(gold["cfl"]), float(gold["gamma"]))
    oq = _q0(gold)
    dts = []
    for _ in range(len(gold["dts"])):
        dts.append(S.stepper())
        S.compute_new_val()
        assert dts[-1] == O.euler_step_2d(mesh, oq, float(gold["cfl"]), float(gold["gamma"]))
    assert np.allclose(dts, gold["dts"], rtol=1e-13, atol=0)
    for k, v, b in zip(NAMES, vs, oq):
        assert np.array_equal(v.cell, b), k
        assert _close(v.cell, gold["final_" + k], 1e-12), k
    assert abs(S.time - sum(dts)) <= 1e-15 * len(dts)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [60, 200])
def test_fused_step_bit_identical_to_kernel_sequence(n, cuda):
    """The fused launch against the oracle's ghost -> residual -> min dt -> update sequence,
    on a pressure pulse (n = 200: 80,000 triangles); graph and eager runs agree."""
    import manapy_b200 as M
    import oracle as O
    from manapy_b200 import meshgen
    el, vx = meshgen.square_triangles(n, seed=3)
    q0 = pressure_pulse(M.Domain(dim=2, mesh=(el, vx)).cells.center)
    dom, vs, S = _solver(el, vx, q0)
    m = O.Mesh(dom.host_arrays)
    oq = [a.copy() for a in q0]
    steps = 30
    for _ in range(steps):
        O.euler_step_2d(m, oq, S.cfl, S.gamma)
    S.advance(steps, graph=True)
    for k, v, b in zip(NAMES, vs, oq):
        assert np.array_equal(v.cell, b), k
    # residuals of the unfused kernels on the final state
    S.compute_fluxes()
    g, _, _ = O.ghost_neumann_euler_2d(m, oq)
    rez = O.euler_rusanov_2d(m, oq, g, S.gamma)
    for k, r in zip(("rho", "rhou", "rhov", "rhoE"), rez):
        assert np.array_equal(vs[NAMES.index(k)].convective, r), k
    # the same run eagerly, from the start
    _, vs2, S2 = _solver(el, vx, q0)
    S2.advance(steps)
    for v, w in zip(vs, vs2):
        assert np.array_equal(v.cell, w.cell)
    S.check()


@pytest.mark.gpu
def test_solver_rejects_non_neumann_boundaries(cuda):
    import manapy_b200 as M
    from manapy_b200 import meshgen
    el, vx = meshgen.square_triangles(4, seed=1)
    dom = M.Domain(dim=2, mesh=(el, vx))
    vs = [M.Variable(domain=dom) for _ in NAMES]
    vs[0] = M.Variable(domain=dom, BC={"in": "dirichlet", "out": "neumann", "upper": "neumann",
                                       "bottom": "neumann"}, values={"in": 1.0})
    S = M.EulerSolver(*vs)
    with pytest.raises(NotImplementedError):
        S._setup()
    with pytest.raises(ValueError):
        M.EulerSolver(vs[0], vs[1], vs[2], vs[3], None)
