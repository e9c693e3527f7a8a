"""Continuous-batching server: every request's result is the same alone and in the mix.

The batched kernels run the single-mesh FP32-compensated block bodies on each
item's own tables, so a request's result must be bit-for-bit identical whether
it runs alone, in a mix admitted at once, or in a mix admitted while others run;
and equal to the single-mesh FP32-compensated solver through the public API.
Against the FP64 oracle the stated FP32-compensated tolerances apply.
"""
import numpy as np
import pytest

from conftest import rel_max
import manapy_b200 as M
from manapy_b200 import boundary as B, geometry as G, meshgen
from manapy_b200.serving import BatchServer, Request, SIDES, initial_state
import oracle as O

pytestmark = pytest.mark.gpu


def _mix():
    rs = []
    k = 0
    for n, steps in ((12, 30), (25, 47), (8, 64), (31, 20), (17, 51)):
        rs.append(Request(rid=k, kind="advdiff", n=n, seed=100 + k, steps=steps, ux=0.9 - 0.3 * k,
                          uy=0.2 + 0.25 * k, D=10 ** (-4 + 0.5 * k)))
        k += 1
    for n, steps, ratio in ((14, 33, 1.5), (22, 58, 2.5), (9, 17, 2.0)):
        rs.append(Request(rid=k, kind="sw", n=n, seed=100 + k, steps=steps, ratio=ratio))
        k += 1
    return rs


def _by_rid(recs):
    return {r["rid"]: r for r in recs}


def test_alone_and_in_the_mix_are_identical(cuda):
    reqs = _mix()
    mixed = _by_rid(BatchServer(workers=0, chunk=8).serve(reqs, keep_results=True))
    assert sorted(mixed) == [r.rid for r in reqs]
    for r in reqs:
        alone = BatchServer(workers=0, chunk=8).serve([r], keep_results=True)[0]
        for a, b in zip(alone["result"], mixed[r.rid]["result"]):
            assert np.array_equal(a, b), r


def test_staggered_admission_and_worker_pool(cuda):
    """Requests arriving while others run (prepared by worker processes) give the same results."""
    reqs = _mix()
    for k, r in enumerate(reqs):
        r.arrival = 0.05 * k
    staggered = _by_rid(BatchServer(workers=2, chunk=4, max_active=3).serve(reqs, keep_results=True))
    blocking = _by_rid(BatchServer(workers=2, chunk=4, max_active=3, poll=False).serve(reqs, keep_results=True))
    for r in reqs:
        r.arrival = 0.0
    at_once = _by_rid(BatchServer(workers=0, chunk=16).serve(reqs, keep_results=True))
    for r in reqs:
        for a, b, c in zip(staggered[r.rid]["result"], at_once[r.rid]["result"], blocking[r.rid]["result"]):
            assert np.array_equal(a, b) and np.array_equal(c, b), r
        for rec in (staggered[r.rid], blocking[r.rid]):
            assert rec["done"] >= rec["admitted"] >= 0 and rec["latency"] > 0
            # handed over at arrival or later, prepared in a worker, received, then admitted
            assert rec["arrival"] <= rec["submitted"] <= rec["prep_start"] <= rec["prep_end"] <= rec["received"]
            assert rec["received"] <= rec["admitted"]


def test_batched_equals_the_single_mesh_solver_and_the_oracle(cuda):
    r = Request(rid=0, kind="advdiff", n=20, seed=7, steps=40, ux=0.7, uy=-0.4, D=3e-3)
    got = BatchServer(workers=0).serve([r], keep_results=True)[0]["result"][0]
    el, vx = meshgen.square_triangles(r.n, seed=r.seed)
    dom = M.Domain(dim=2, mesh=(el, vx))
    w = M.Variable(domain=dom, BC={s: "dirichlet" for s in SIDES}, values={s: 0.0 for s in SIDES})
    u, v = M.Variable(domain=dom), M.Variable(domain=dom)
    u.face = np.full(dom.nbfaces, r.ux)
    v.face = np.full(dom.nbfaces, r.uy)
    u.cell = np.full(dom.nbcells, r.ux)  # the server's constant cell velocity, exactly
    v.cell = np.full(dom.nbcells, r.uy)
    w.cell = initial_state(r, dom.cells.center)[0]
    S = M.AdvectionDiffusionSolver(w, vel=(u, v), conf=M.Struct(Dxx=r.D, Dyy=r.D, order=2, cfl=0.8,
                                                                 precision="fp32c"))
    S.advance(r.steps)
    assert np.array_equal(got, w.cell)
    A = G.build(el, vx, 2)
    o = O.AdvDiffOracle(A, B.resolve(A, {s: "dirichlet" for s in SIDES}, {s: 0.0 for s in SIDES}),
                        r.D, r.D, 0.0, order=2, cfl=0.8)
    o.set_velocity(np.full(A["nbfaces"], r.ux), np.full(A["nbfaces"], r.uy), np.zeros(A["nbfaces"]))
    o.w[:] = initial_state(r, A["cells_center"])[0]
    for _ in range(r.steps):
        o.step()
    assert rel_max(got, o.w) < 1e-5


def test_batched_shallow_water_matches_the_single_mesh_step(cuda):
    r = Request(rid=0, kind="sw", n=16, seed=3, steps=25, ratio=2.2)
    got = BatchServer(workers=0).serve([r], keep_results=True)[0]["result"]
    el, vx = meshgen.square_triangles(r.n, seed=r.seed)
    dom = M.Domain(dim=2, mesh=(el, vx))
    vs = [M.Variable(domain=dom) for _ in range(5)]
    for var, a in zip(vs, initial_state(r, dom.cells.center)):
        var.cell = a
    S = M.ShallowWaterSolver(vs[0], hvel=(vs[1], vs[2]), hc=vs[3], Z=vs[4],
                             conf=M.Struct(order=1, cfl=0.5, grav=9.81, precision="fp32c"))
    S.advance(r.steps)
    for a, var in zip(got, vs[:3]):
        assert np.array_equal(a, var.cell)


def _single_fp64(r):
    """The request solved alone through the public FP64 solvers (manapy's arithmetic)."""
    el, vx = meshgen.square_triangles(r.n, seed=r.seed)
    dom = M.Domain(dim=2, mesh=(el, vx))
    if r.kind == "advdiff":
        w = M.Variable(domain=dom, BC={s: "dirichlet" for s in SIDES}, values={s: 0.0 for s in SIDES})
        u, v = M.Variable(domain=dom), M.Variable(domain=dom)
        u.face = np.full(dom.nbfaces, r.ux)
        v.face = np.full(dom.nbfaces, r.uy)
        u.cell = np.full(dom.nbcells, r.ux)
        v.cell = np.full(dom.nbcells, r.uy)
        w.cell = initial_state(r, dom.cells.center)[0]
        S = M.AdvectionDiffusionSolver(w, vel=(u, v), conf=M.Struct(Dxx=r.D, Dyy=r.D, order=2, cfl=0.8))
        S.advance(r.steps)
        return [w.cell]
    vs = [M.Variable(domain=dom) for _ in range(5)]
    for var, a in zip(vs, initial_state(r, dom.cells.center)):
        var.cell = a
    S = M.ShallowWaterSolver(vs[0], hvel=(vs[1], vs[2]), hc=vs[3], Z=vs[4],
                             conf=M.Struct(order=1, cfl=0.5, grav=9.81))
    S.advance(r.steps)
    return [var.cell for var in vs[:3]]


def test_batched_fp64_matches_the_single_mesh_fp64_solver(cuda):
    """The FP64 batches run the single-mesh FP64 block bodies, so every request of a mix
    equals its own plain FP64 solve to rounding: the FP64 kernels let the compiler contract
    multiply-adds, and it may contract differently in the batched and single-mesh kernel
    instantiations (measured at the last bits; tolerance 1e-13, norm-relative).  Within
    the batched kernels a request's result is bit-identical alone and in any mix (below)."""
    reqs = _mix()
    mixed = _by_rid(BatchServer(workers=0, chunk=8, precision="fp64").serve(reqs, keep_results=True))
    for r in reqs:
        for a, b in zip(mixed[r.rid]["result"], _single_fp64(r)):
            assert rel_max(a, b) <= 1e-13, r


def test_batched_fp64_alone_and_in_the_mix_are_identical(cuda):
    reqs = _mix()
    mixed = _by_rid(BatchServer(workers=0, chunk=8, precision="fp64").serve(reqs, keep_results=True))
    for r in reqs[::3]:
        alone = BatchServer(workers=0, chunk=8, precision="fp64").serve([r], keep_results=True)[0]
        for a, b in zip(alone["result"], mixed[r.rid]["result"]):
            assert np.array_equal(a, b), r


def test_batched_fp64_staggered_admission(cuda):
    reqs = _mix()
    for k, r in enumerate(reqs):
        r.arrival = 0.03 * k
    staggered = _by_rid(BatchServer(workers=0, chunk=4, max_active=3, precision="fp64").serve(reqs,
                                                                                             keep_results=True))
    for r in reqs:
        r.arrival = 0.0
    at_once = _by_rid(BatchServer(workers=0, chunk=16, precision="fp64").serve(reqs, keep_results=True))
    for r in reqs:
        for a, b in zip(staggered[r.rid]["result"], at_once[r.rid]["result"]):
            assert np.array_equal(a, b), r


@pytest.mark.parametrize("skip", [True, False])
def test_small_requests_pass_one_that_does_not_fit(skip, cuda):
    """Under an HBM budget that the first request and a large second one exceed together,
    the later small ones are admitted before the large one (or, with max_skip_wait=0, after
    it, in arrival order); every result equals the request's result alone."""
    from manapy_b200 import serving as SV
    reqs = [Request(rid=0, kind="advdiff", n=20, seed=7, steps=40, ux=0.5, uy=0.3, D=1e-3),
            Request(rid=1, kind="advdiff", n=60, seed=8, steps=20, ux=0.4, uy=0.2, D=1e-3),
            Request(rid=2, kind="sw", n=12, seed=9, steps=25, ratio=2.0),
            Request(rid=3, kind="advdiff", n=14, seed=10, steps=30, ux=0.2, uy=0.6, D=1e-4)]

    def est(r):
        dm = SV.prepare(r)[1]
        return dm.nbytes() + 48.0 * dm.nbcells + 16.0 * dm.nbfaces
    e = [est(r) for r in reqs]
    budget = 1.2 * (e[0] + e[2] + e[3])
    assert e[0] + e[1] > budget
    srv = BatchServer(workers=0, chunk=4, hbm_budget=budget, max_skip_wait=1e9 if skip else 0.0)
    recs = _by_rid(srv.serve(reqs, keep_results=True))
    if skip:
        assert recs[2]["admitted"] < recs[1]["admitted"] and recs[3]["admitted"] < recs[1]["admitted"]
    else:
        assert recs[1]["admitted"] <= recs[2]["admitted"] <= recs[3]["admitted"]
    for r in reqs:
        alone = BatchServer(workers=0, chunk=4).serve([r], keep_results=True)[0]
        for a, b in zip(alone["result"], recs[r.rid]["result"]):
            assert np.array_equal(a, b), r
