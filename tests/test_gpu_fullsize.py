"""Full-size parity: the GPU path against the oracle over whole configured runs.

The fixtures ``tests/golden/full_<name>.npz`` hold the oracle's run of each large
configuration at its stated size and length (``tests/golden/make_fullsize.py``):
C2 (2,000,000 triangles, order 2 + diffusion, 1000 steps), C4 (1,572,864 tetrahedra,
300 steps) and C3 (8,000,000 triangles, shallow water, 500 steps, checkpoint at 100).
A full state is too large to commit, so the comparison uses size-independent
summaries of the final state: L2 / Linf norms, four fixed-weight projections (sums
over every cell), a seeded sample of cells, the FP64 mass and the dt sequence.

Tolerances, norm-relative (|a - b| / |b|, over cells: the Linf norm of the oracle's
field as the denominator):

* plain FP64: 1e-12 (sample, norms, projections relative to sum |weight x value|,
  mass); dt 1e-14;
* FP32-compensated (C2, C4; C3 h): L2 over the sample 1e-6, Linf over the sample
  1e-5; C3 momentum (FP32 SRNH flux arithmetic): L2 1e-4.
"""
import os

import numpy as np
import pytest

import manapy_b200 as M
from manapy_b200 import workloads as W

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-12


def _fixture(name):
    p = os.path.join(GOLDEN, "full_%s.npz" % name.lower())
    if not os.path.exists(p):
        pytest.skip("fixture %s not generated (tests/golden/make_fullsize.py %s)" % (os.path.basename(p), name))
    return np.load(p)


def _weights(n, k):
    h = ((np.arange(n, dtype=np.uint64) + np.uint64(0x9E3779B9 * (k + 1) & 0xFFFFFFFF))
         * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)
    return h.astype(np.float64) / 4294967296.0 - 0.5


def _compare_fp64(got, g, key):
    """got: full field (manapy numbering); key: fixture prefix such as 's1000_w'."""
    n = len(got)
    linf = float(g[key + "_linf"])
    idx = g["sample_idx"]
    err = {"sample": float(np.max(np.abs(got[idx] - g[key + "_sample"])) / linf),
           "l2": abs(float(np.sqrt(np.dot(got, got))) - float(g[key + "_l2"])) / float(g[key + "_l2"]),
           "linf": abs(float(np.max(np.abs(got))) - linf) / linf}
    for k in range(len(g[key + "_proj"])):
        p = float(np.dot(_weights(n, k), got))
        err["proj%d" % k] = abs(p - float(g[key + "_proj"][k])) / float(g[key + "_projabs"][k])
    return err


def _sample_errors(got, g, key):
    idx = g["sample_idx"]
    ref = g[key + "_sample"]
    d = got[idx] - ref
    return (float(np.linalg.norm(d) / np.linalg.norm(ref)), float(np.max(np.abs(d)) / float(g[key + "_linf"])))


def _advdiff_solver(dom, wl, precision):
    w = M.Variable(domain=dom, BC=wl.bc, values=wl.bc_values)
    vel = [M.Variable(domain=dom) for _ in range(3)]
    for var, a in zip(vel, wl.velocity(dom.faces.center)):
        var.face = a
        var.interpolate_facetocell()
    w.cell = wl.init(dom.cells.center)
    S = M.AdvectionDiffusionSolver(w, vel=tuple(vel), conf=M.Struct(
        Dxx=wl.diffusion[0], Dyy=wl.diffusion[1], Dzz=wl.diffusion[2], order=wl.order, cfl=wl.cfl,
        precision=precision))
    return w, S


@pytest.mark.parametrize("name", ["C2", "C4"])
def test_full_size_advection_diffusion_matches_the_oracle(name, cuda):
    g = _fixture(name)
    wl = W.ALL[name]
    el, vx = wl.mesh()
    dom = M.Domain(dim=wl.dim, mesh=(el, vx))
    assert int(dom.nbcells) == int(g["nbcells"]) == wl.cells
    vol = dom.cells.volume
    w, S = _advdiff_solver(dom, wl, "fp64")
    assert abs(float(np.dot(vol, w.cell)) - float(g["mass0"])) <= TOL * abs(float(g["mass0"]))
    dt = S.stepper()
    # steady velocity: the oracle's dt is the same number at every step
    assert np.all(np.abs(g["dts"] - dt) <= 1e-14 * dt)
    done = 0
    for s in g["checkpoints"]:
        S.advance(int(s) - done, graph=True)
        done = int(s)
        got = w.cell
        err = _compare_fp64(got, g, "s%d_w" % s)
        print(name, "step", s, {k: "%.2e" % v for k, v in err.items()})
        assert max(err.values()) <= TOL, err
        m = float(np.dot(vol, got))
        assert abs(m - float(g["mass"][s - 1])) <= TOL * abs(float(g["mass"][s - 1]))
    S.release_graphs()
    # FP32-compensated over the same run
    w32, S32 = _advdiff_solver(dom, wl, "fp32c")
    S32.advance(int(g["checkpoints"][-1]), graph=True)
    s = int(g["checkpoints"][-1])
    l2, linf = _sample_errors(w32.cell, g, "s%d_w" % s)
    print(name, "fp32c step", s, "L2 %.2e Linf %.2e (sample)" % (l2, linf))
    assert l2 <= 1e-6 and linf <= 1e-5
    S32.release_graphs()


def test_full_size_shallow_water_matches_the_oracle(cuda):
    g = _fixture("C3")
    wl = W.C3
    el, vx = wl.mesh()
    dom = M.Domain(dim=2, mesh=(el, vx))
    assert int(dom.nbcells) == int(g["nbcells"]) == wl.cells
    vol = dom.cells.volume

    def solver(precision):
        vs = [M.Variable(domain=dom) for _ in range(5)]
        for var, a in zip(vs, wl.init_sw(dom.cells.center)):
            var.cell = a
        return vs, M.ShallowWaterSolver(vs[0], hvel=(vs[1], vs[2]), hc=vs[3], Z=vs[4],
                                        conf=M.Struct(order=wl.order, cfl=wl.cfl, grav=wl.grav,
                                                      precision=precision))

    vs, S = solver("fp64")
    assert abs(S.mass() - float(g["mass0"])) <= TOL * float(g["mass0"])
    done = 0
    dts = []
    for s in g["checkpoints"]:
        for _ in range(int(s) - done):
            dts.append(S.stepper())
            S.compute_fluxes()
            S.compute_new_val()
        done = int(s)
        for f, var in zip(("h", "hu", "hv"), vs[:3]):
            err = _compare_fp64(var.cell, g, "s%d_%s" % (s, f))
            print("C3 step", s, f, {k: "%.2e" % v for k, v in err.items()})
            assert max(err.values()) <= TOL, (f, err)
        # FP64 mass to 1e-12 relative of the oracle's
        assert abs(S.mass() - float(g["mass"][s - 1])) <= TOL * float(g["mass"][s - 1])
    dts = np.array(dts)
    assert np.max(np.abs(dts - g["dts"][:len(dts)]) / g["dts"][:len(dts)]) <= 1e-12
    # FP32-compensated, same steps
    vs32, S32 = solver("fp32c")
    S32.advance(done)
    for f, var, tol in zip(("h", "hu", "hv"), vs32[:3], (1e-6, 1e-4, 1e-4)):
        l2, linf = _sample_errors(var.cell, g, "s%d_%s" % (done, f))
        print("C3 fp32c step", done, f, "L2 %.2e Linf %.2e (sample)" % (l2, linf))
        assert l2 <= tol
    assert abs(S32.mass() - float(g["mass"][done - 1])) <= 1e-7 * float(g["mass"][done - 1])
