"""Whole steps through the public API (fused CUDA path) against the reference and the oracle.

Tolerance: the plain FP64 path must stay within 1e-12 relative (max-norm over
cells) of the reference after the full run; per-kernel rounding differences
(fused multiply-adds) are ~1e-16 per step.
"""
import numpy as np
import pytest

from conftest import golden, rel_max
import manapy_b200 as M
from manapy_b200 import boundary as B, geometry as G, workloads as W
import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _advdiff_api(el, vx, wl):
    dom = M.Domain(dim=wl.dim, mesh=(el, vx))
    w = M.Variable(domain=dom, BC=wl.bc, values=wl.bc_values)
    u, v, wz = (M.Variable(domain=dom) for _ in range(3))
    uf, vf, wf = wl.velocity(dom.faces.center)
    u.face = uf
    v.face = vf
    wz.face = wf
    for x in (u, v, wz):
        x.interpolate_facetocell()
    w.cell = wl.init(dom.cells.center)
    S = M.AdvectionDiffusionSolver(w, vel=(u, v, wz), conf=M.Struct(Dxx=wl.diffusion[0], Dyy=wl.diffusion[1],
                                                                     Dzz=wl.diffusion[2], order=wl.order,
                                                                     cfl=wl.cfl))
    return dom, w, S


def _oracle(el, vx, wl):
    A = G.build(el, vx, wl.dim)
    o = O.AdvDiffOracle(A, B.resolve(A, wl.bc, wl.bc_values), *wl.diffusion, order=wl.order, cfl=wl.cfl)
    o.set_velocity(*wl.velocity(A["faces_center"]))
    o.w[:] = wl.init(A["cells_center"])
    return o


@pytest.mark.parametrize("name,wl", [("traj_c1", W.C1), ("traj_o2", W.C2.scaled(n=32, steps=100)),
                                     ("traj_3d", W.C4.scaled(n=6, steps=30))])
def test_manapy_loop_matches_reference(name, wl, cuda):
    g = golden(name)
    el, vx = g["in_elements"], g["in_vertex"]
    dom, w, S = _advdiff_api(el, vx, wl)
    dts = []
    for it in range(int(g["steps"])):
        dts.append(S.stepper())
        S.compute_fluxes()
        S.compute_new_val()
        key = "w_step%d" % (it + 1)
        if key in g.files:
            assert rel_max(w.cell, g[key]) < TOL, key
    assert rel_max(np.array(dts), g["dts"]) < 1e-15
    assert rel_max(w.cell, g["w_final"]) < TOL


@pytest.mark.parametrize("wl", [W.C1.scaled(n=60, steps=40), W.C2.scaled(n=150, steps=25),
                                W.C4.scaled(n=10, steps=15), W.C4.scaled(n=8, steps=10, order=1)])
def test_advance_matches_oracle(wl, cuda):
    el, vx = wl.mesh()
    dom, w, S = _advdiff_api(el, vx, wl)
    o = _oracle(el, vx, wl)
    S.advance(wl.steps, graph=True)
    for _ in range(wl.steps):
        o.step()
    assert rel_max(w.cell, o.w) < TOL


@pytest.mark.parametrize("wl", [W.C2.scaled(n=120, steps=30), W.C4.scaled(n=10, steps=15)])
def test_stencil_layouts_agree(wl, cuda):
    """The slot-shared least-squares stencil (the default) and manapy's order give the same
    states to rounding, and both the oracle's."""
    el, vx = wl.mesh()
    runs = []
    for stencil in ("shared", "manapy"):
        dom = M.Domain(dim=wl.dim, mesh=(el, vx), stencil=stencil)
        assert dom.device_mesh.stencil == stencil
        w = M.Variable(domain=dom, BC=wl.bc, values=wl.bc_values)
        vel = [M.Variable(domain=dom) for _ in range(3)]
        for var, a in zip(vel, wl.velocity(dom.faces.center)):
            var.face = a
            var.interpolate_facetocell()
        w.cell = wl.init(dom.cells.center)
        S = M.AdvectionDiffusionSolver(w, vel=tuple(vel), conf=M.Struct(
            Dxx=wl.diffusion[0], Dyy=wl.diffusion[1], Dzz=wl.diffusion[2], order=wl.order, cfl=wl.cfl))
        S.advance(wl.steps, graph=True)
        runs.append(w.cell)
    o = _oracle(el, vx, wl)
    for _ in range(wl.steps):
        o.step()
    assert rel_max(runs[0], runs[1]) < 1e-13
    assert rel_max(runs[0], o.w) < TOL and rel_max(runs[1], o.w) < TOL


def test_graph_and_eager_agree_bitwise(cuda):
    wl = W.C2.scaled(n=40, steps=9)
    el, vx = wl.mesh()
    _, w1, S1 = _advdiff_api(el, vx, wl)
    _, w2, S2 = _advdiff_api(el, vx, wl)
    S1.advance(wl.steps, graph=True)
    S2.advance(wl.steps, graph=False)
    assert np.array_equal(w1.cell, w2.cell)


@pytest.mark.parametrize("precision,depth", [("fp64", 2), ("fp32c", 2), ("fp64", 4), ("fp32c", 4)])
def test_graph_runs_resume_after_odd_step_counts(precision, depth, cuda):
    """advance() calls of odd lengths, a manapy-style step and a cell edit in between: the
    replayed graphs continue from the current state exactly as eager steps do."""
    wl = W.C2.scaled(n=30)
    el, vx = wl.mesh()
    runs = []
    for graph in (True, False):
        dom = M.Domain(dim=2, mesh=(el, vx))
        w = M.Variable(domain=dom, BC=wl.bc, values=wl.bc_values)
        u, v = M.Variable(domain=dom), M.Variable(domain=dom)
        uf, vf, _ = wl.velocity(dom.faces.center)
        u.face, v.face = uf, vf
        u.interpolate_facetocell(); v.interpolate_facetocell()
        w.cell = wl.init(dom.cells.center)
        S = M.AdvectionDiffusionSolver(w, vel=(u, v), conf=M.Struct(Dxx=5e-4, Dyy=5e-4, order=2, cfl=0.8,
                                                                     precision=precision, graph_depth=depth))
        S.advance(3, graph=graph)
        S.advance(4, graph=graph)
        S.stepper(); S.compute_fluxes(); S.compute_new_val()
        S.advance(5, graph=graph)
        w.cell = w.cell * 0.75
        S.advance(6, graph=graph)
        S.advance(11, graph=graph)
        runs.append(w.cell)
    assert np.array_equal(runs[0], runs[1])


def test_intermediate_arrays_match_reference_kernels(cuda):
    """After compute_fluxes, manapy's intermediate arrays are readable and exact."""
    g = golden("traj_o2")
    wl = W.C2.scaled(n=32, steps=3)
    el, vx = g["in_elements"], g["in_vertex"]
    dom, w, S = _advdiff_api(el, vx, wl)
    o = _oracle(el, vx, wl)
    for _ in range(2):
        S.stepper(); S.compute_fluxes(); S.compute_new_val()
        o.step()
    S.stepper()
    S.compute_fluxes()
    o.stepper()
    o.compute_fluxes()
    assert rel_max(w.convective, o.rez) < 1e-13
    assert rel_max(w.dissipative, o.dissip) < 1e-13
    assert rel_max(w.gradcellx, o.gx) < 1e-13 and rel_max(w.psi, o.psi) < 1e-13
    assert rel_max(w.gradfacex, o.gfx) < 1e-13
    # reading convective switched this step to the unfused update; still exact
    S.compute_new_val()
    o.compute_new_val()
    assert rel_max(w.cell, o.w) < TOL


def test_user_edit_of_residual_is_honoured(cuda):
    wl = W.C1.scaled(n=20, steps=1)
    el, vx = wl.mesh()
    dom, w, S = _advdiff_api(el, vx, wl)
    o = _oracle(el, vx, wl)
    S.stepper(); S.compute_fluxes()
    o.stepper(); o.compute_fluxes()
    rez = w.convective
    rez[:] = rez * 0.5
    w.convective = rez
    o.rez *= 0.5
    S.compute_new_val(); o.compute_new_val()
    assert rel_max(w.cell, o.w) < TOL


def test_full_size_c2_steps(cuda):
    """The 2,000,000-triangle mesh: three steps against the oracle, and conservation of
    the update (sum V dw = dt * sum of residuals) on the device."""
    wl = W.C2.scaled(steps=3)
    el, vx = wl.mesh()
    dom, w, S = _advdiff_api(el, vx, wl)
    o = _oracle(el, vx, wl)
    for _ in range(3):
        S.stepper(); S.compute_fluxes(); S.compute_new_val()
        o.step()
    assert rel_max(w.cell, o.w) < TOL


def _sw_api(el, vx, wl):
    dom = M.Domain(dim=2, mesh=(el, vx))
    h, hu, hv, hc, Z = (M.Variable(domain=dom) for _ in range(5))
    for var, a in zip((h, hu, hv, hc, Z), wl.init_sw(dom.cells.center)):
        var.cell = a
    S = M.ShallowWaterSolver(h, hvel=(hu, hv), hc=hc, Z=Z, conf=M.Struct(order=wl.order, cfl=wl.cfl, grav=wl.grav))
    return dom, (h, hu, hv, hc, Z), S


@pytest.mark.parametrize("order,n,steps", [(1, 40, 60), (2, 40, 60), (1, 120, 150)])
def test_shallow_water_matches_oracle(order, n, steps, cuda):
    wl = W.C3.scaled(n=n, steps=steps, order=order)
    el, vx = wl.mesh()
    dom, vs, S = _sw_api(el, vx, wl)
    A = dom.host_arrays
    so = O.ShallowWaterOracle(A, order=order, cfl=wl.cfl, grav=wl.grav)
    for k, a in zip(("h", "hu", "hv", "hc", "Z"), wl.init_sw(A["cells_center"])):
        so.state()[k][:] = a
    for _ in range(wl.steps):
        S.stepper(); S.compute_fluxes(); S.compute_new_val()
        so.step()
    for k, var in zip(("h", "hu", "hv", "hc", "Z"), vs):
        ref = so.state()[k]
        if np.any(ref):
            assert rel_max(var.cell, ref) < TOL, k
    # mass: FP64 sum of V h changes only through boundary fluxes (Neumann walls leak)
    assert abs(np.sum(vs[0].cell * A["cells_volume"]) - np.sum(so.h * A["cells_volume"])) < 1e-12


@pytest.mark.parametrize("name", ["traj_sw1", "traj_sw2"])
def test_shallow_water_matches_reference(name, cuda):
    import os
    from conftest import GOLDEN
    if not os.path.exists(os.path.join(GOLDEN, name + ".npz")):
        pytest.skip("fixture not generated")
    g = golden(name)
    wl = W.C3.scaled(n=30, order=int(g["order"]), steps=int(g["steps"]))
    dom, vs, S = _sw_api(g["in_elements"], g["in_vertex"], wl)
    for _ in range(wl.steps):
        S.stepper(); S.compute_fluxes(); S.compute_new_val()
    for k, var in zip(("h", "hu", "hv"), vs[:3]):
        assert rel_max(var.cell, g[k + "_final"]) < TOL, k


def test_autotuned_graph_depth_changes_no_result(cuda):
    """graph_depth='auto' times several depths on the solver's own state and restores it."""
    from manapy_b200 import autotune
    autotune.clear()
    wl = W.C1.scaled(n=30, steps=40)
    el, vx = wl.mesh()
    _, w1, S1 = _advdiff_api(el, vx, wl)
    _, w2, S2 = _advdiff_api(el, vx, wl)
    S1.advance(wl.steps, graph=True)
    assert S1.graph_depth in autotune.CANDIDATES
    S2.advance(wl.steps, graph=False)
    assert np.array_equal(w1.cell, w2.cell)


@pytest.mark.parametrize("name", ["traj_advec", "traj_diff"])
def test_advection_and_diffusion_solvers_match_reference(name, cuda):
    g = golden(name)
    wl = W.C2.scaled(n=24)
    dom = M.Domain(dim=2, mesh=(g["in_elements"], g["in_vertex"]))
    w = M.Variable(domain=dom, BC=wl.bc, values=wl.bc_values)
    u, v, wz = (M.Variable(domain=dom) for _ in range(3))
    uf, vf, wf = wl.velocity(dom.faces.center)
    u.face, v.face, wz.face = uf, vf, wf
    for x in (u, v, wz):
        x.interpolate_facetocell()
    w.cell = g["w0"]
    if name == "traj_advec":
        S = M.AdvectionSolver(w, vel=(u, v, wz), conf=M.Struct(order=2, cfl=wl.cfl))
    else:
        S = M.DiffusionSolver(w, vel=(u, v, wz), conf=M.Struct(Dxx=1e-3, Dyy=1e-3, cfl=wl.cfl))
    dts = []
    for it in range(int(g["steps"])):
        dts.append(S.stepper())
        S.compute_fluxes()
        S.compute_new_val()
        if it + 1 in (1, 10):
            assert rel_max(w.cell, g["w_step%d" % (it + 1)]) < TOL
    assert rel_max(np.array(dts), g["dts"]) < 1e-14
    assert rel_max(w.cell, g["w_final"]) < TOL


def test_state_checks_raise(cuda):
    wl = W.C3.scaled(n=10, steps=1, order=1)
    el, vx = wl.mesh()
    dom, vs, S = _sw_api(el, vx, wl)
    S.advance(2)
    S.check()                        # a sound state passes
    h = vs[0].cell
    h[3] = -0.5
    vs[0].cell = h
    with pytest.raises(ValueError, match="negative"):
        S.check()
    h[3] = np.nan
    vs[0].cell = h
    with pytest.raises(FloatingPointError):
        S.check()
    wl2 = W.C1.scaled(n=10, steps=1)
    el, vx = wl2.mesh()
    _, w, S2 = _advdiff_api(el, vx, wl2)
    S2.advance(2)
    S2.check()
    x = w.cell
    x[0] = np.inf
    w.cell = x
    with pytest.raises(FloatingPointError):
        S2.check()


@pytest.mark.parametrize("wl", [W.C2.scaled(n=50), W.C4.scaled(n=7)])
def test_row_carrying_step_matches_the_plain_step(wl, cuda):
    """mb_advdiff_step_rows (rows {centre, value} in, rows of the result out) gives the
    results of mb_advdiff_step, and its rows_out are the rows mb_pack_rows makes of w_out."""
    import gpuutil as U
    from manapy_b200 import _lib
    el, vx = wl.mesh()
    A = G.build(el, vx, wl.dim)
    dm = U.mesh(A, reorder=True)
    db = U.bc(A, B.resolve(A, wl.bc, wl.bc_values), dm)
    R = dm.R
    uf, vf, wf = wl.velocity(A["faces_center"])
    st = U.stream()
    nc, nn = A["nbcells"], A["nbnodes"]
    sign = U.Z(4 * nc)
    u_, v_, w_ = U.T(uf[R.fperm]), U.T(vf[R.fperm]), U.T(wf[R.fperm])
    U.call("mb_cell_face_sign", dm.struct, U.P(u_), U.P(v_), U.P(w_), U.P(sign), st)
    cells = [U.Z(nc) for _ in range(3)]
    for f, c in zip((u_, v_, w_), cells):
        U.call("mb_facetocell", dm.struct, U.P(f), U.P(c), st)
    dt = U.Z(1)
    U.call("mb_time_step", dm.struct, *[U.P(c) for c in cells], wl.cfl, *wl.diffusion, U.P(dt), st)
    prm = _lib.MbAdvDiffParams(wl.order, 1, *wl.diffusion)
    w0 = U.T(wl.init(A["cells_center"])[R.cperm])
    cs, ns = U.Z((4 if wl.dim == 2 else 8) * nc), U.Z(nn)
    ref = U.Z(nc)
    U.call("mb_advdiff_step", dm.struct, db.struct, prm, U.P(w0), U.P(ref), U.P(sign), None, U.P(dt), U.P(cs),
           U.P(ns), st)
    rin, rout, packed = U.Z(4 * nc), U.Z(4 * nc), U.Z(4 * nc)
    U.call("mb_pack_rows", dm.struct, U.P(w0), U.P(rin), st)
    got = U.Z(nc)
    U.call("mb_advdiff_step_rows", dm.struct, db.struct, prm, U.P(w0), U.P(got), U.P(rin), U.P(rout), U.P(sign),
           None, U.P(dt), U.P(cs), U.P(ns), st)
    U.call("mb_pack_rows", dm.struct, U.P(got), U.P(packed), st)
    assert rel_max(U.H(got), U.H(ref)) <= 1e-14
    assert np.array_equal(U.H(rout), U.H(packed))


@pytest.mark.parametrize("wl", [W.C2.scaled(n=60, steps=6), W.C4.scaled(n=8, steps=6)])
def test_every_launch_variant_gives_the_default_result(wl, cuda):
    """The pre-built launch shapes of the fused phases (mb_mesh.variant) compute the same
    operations: results agree with the default shapes to rounding (1e-13), and tuning
    leaves the state as it found it."""
    from manapy_b200 import autotune
    el, vx = wl.mesh()
    outs = {}
    for v in (0, 1, 2, 3, 4, 8, 12, 15):
        _, w, S = _advdiff_api(el, vx, wl)
        S.launch = v
        S._setup()
        S._dm.struct.variant = v
        S.advance(wl.steps, graph=True)
        outs[v] = w.cell
    for v, a in outs.items():
        assert rel_max(a, outs[0]) <= 1e-13, v
    autotune.clear()
    big = wl.scaled(n=200) if wl.dim == 2 else wl.scaled(n=24)     # above the tuner's lower size bound
    el, vx = big.mesh()
    _, w, S = _advdiff_api(el, vx, big)
    w0 = w.cell.copy()
    assert autotune.launch_variant(S, steps=4) in range(16)
    assert np.array_equal(w.cell, w0)


def test_precomputed_moment_matrix(cuda):
    """mb_lsq_matrix: every tetrahedron's moment matrix (cofactors, determinant) matches
    the sum over its stencil formed on the host, and the second-order step that reads it
    gives the step that forms the matrix itself, to rounding."""
    import gpuutil as U
    from manapy_b200 import _lib
    wl = W.C4.scaled(n=7)
    el, vx = wl.mesh()
    A = G.build(el, vx, 3)
    dm = U.mesh(A, reorder=True)
    db = U.bc(A, B.resolve(A, wl.bc, wl.bc_values), dm)
    R = dm.R
    nc, nn = A["nbcells"], A["nbnodes"]
    st = U.stream()
    lsq = U.Z(12 * nc)
    U.call("mb_lsq_matrix", dm.struct, U.P(lsq), st)
    got = U.H(lsq).reshape(nc, 12)[R.cinv]         # manapy numbering
    c = A["cells_center"][:, :3]
    ptr, idx = A["cellnid_ptr"], A["cellnid_idx"]
    gptr, gidx = A["ghostnid_ptr"], A["ghostnid_idx"]
    M_ = np.zeros((nc, 3, 3))
    D_ = np.zeros((nc, 3))
    for i in range(nc):
        pts = np.concatenate([c[idx[ptr[i]:ptr[i + 1]]], A["faces_ghostcenter"][gidx[gptr[i]:gptr[i + 1]], :3]])
        d = pts - c[i]
        M_[i] = d.T @ d
        D_[i] = (c[idx[ptr[i]:ptr[i + 1]]] - c[i]).sum(axis=0)
    det = np.linalg.det(M_)
    cof = np.stack([M_[:, 1, 1] * M_[:, 2, 2] - M_[:, 1, 2] ** 2, M_[:, 0, 2] * M_[:, 1, 2] - M_[:, 0, 1] * M_[:, 2, 2],
                    M_[:, 0, 1] * M_[:, 1, 2] - M_[:, 0, 2] * M_[:, 1, 1], M_[:, 0, 0] * M_[:, 2, 2] - M_[:, 0, 2] ** 2,
                    M_[:, 0, 1] * M_[:, 0, 2] - M_[:, 1, 2] * M_[:, 0, 0], M_[:, 0, 0] * M_[:, 1, 1] - M_[:, 0, 1] ** 2],
                   axis=1)
    assert rel_max(got[:, :6], cof) < 1e-12
    assert rel_max(got[:, 6], det) < 1e-12
    assert np.all(got[:, 7] == 0) and np.all(got[:, 11] == 0)
    assert np.abs(got[:, 8:11] - D_).max() < 1e-12 * np.abs(c).max()
    # the step with and without the table
    uf, vf, wf = wl.velocity(A["faces_center"])
    sign = U.Z(4 * nc)
    u_, v_, w_ = U.T(uf[R.fperm]), U.T(vf[R.fperm]), U.T(wf[R.fperm])
    U.call("mb_cell_face_sign", dm.struct, U.P(u_), U.P(v_), U.P(w_), U.P(sign), st)
    cells = [U.Z(nc) for _ in range(3)]
    for f, cc in zip((u_, v_, w_), cells):
        U.call("mb_facetocell", dm.struct, U.P(f), U.P(cc), st)
    dt = U.Z(1)
    U.call("mb_time_step", dm.struct, *[U.P(x) for x in cells], wl.cfl, *wl.diffusion, U.P(dt), st)
    prm = _lib.MbAdvDiffParams(2, 1, *wl.diffusion)
    w0 = U.T(wl.init(A["cells_center"])[R.cperm])
    cs, ns = U.Z(8 * nc), U.Z(nn)
    outs = []
    for table in (None, lsq):
        dm.struct.cell_lsq = U.P(table) if table is not None else None
        out = U.Z(nc)
        U.call("mb_advdiff_step", dm.struct, db.struct, prm, U.P(w0), U.P(out), U.P(sign), None, U.P(dt), U.P(cs),
               U.P(ns), st)
        outs.append(U.H(out))
    dm.struct.cell_lsq = None
    assert rel_max(outs[1], outs[0]) < 1e-14
    assert not np.array_equal(outs[0], U.H(w0))
    # a table not 32-byte aligned is refused
    dm.struct.cell_lsq = U.P(lsq) + 8
    out = U.Z(nc)
    assert _lib.lib().mb_advdiff_step(dm.struct, db.struct, prm, U.P(w0), U.P(out), U.P(sign), None, U.P(dt),
                                      U.P(cs), U.P(ns), st) == _lib.MB_EINVAL
    dm.struct.cell_lsq = None


@pytest.mark.parametrize("wl", [W.C2.scaled(n=40), W.C4.scaled(n=6)])
def test_split_step_equals_the_whole_step(wl, cuda):
    """mb_advdiff_step_split part 0 (first phase, second phase of cells [0, nfirst)) then
    part 1 (second phase of the rest) computes exactly mb_advdiff_step's result, with the
    first cells numbered first as a sharded run numbers the cells its peers read."""
    import gpuutil as U
    from manapy_b200 import _lib
    from manapy_b200.device import DeviceMesh
    el, vx = wl.mesh()
    A = G.build(el, vx, wl.dim)
    nc, nn = A["nbcells"], A["nbnodes"]
    first = np.random.default_rng(3).random(nc) < 0.2
    dm = DeviceMesh(A, "cuda", first_cells=first)
    assert dm.nfirst == int(first.sum())
    assert np.all(first[dm.R.cperm[:dm.nfirst]]) and not np.any(first[dm.R.cperm[dm.nfirst:]])
    db = U.bc(A, B.resolve(A, wl.bc, wl.bc_values), dm)
    R = dm.R
    st = U.stream()
    uf, vf, wf = wl.velocity(A["faces_center"])
    sign = U.Z(4 * nc)
    u_, v_, w_ = U.T(uf[R.fperm]), U.T(vf[R.fperm]), U.T(wf[R.fperm])
    U.call("mb_cell_face_sign", dm.struct, U.P(u_), U.P(v_), U.P(w_), U.P(sign), st)
    cells = [U.Z(nc) for _ in range(3)]
    for f, c in zip((u_, v_, w_), cells):
        U.call("mb_facetocell", dm.struct, U.P(f), U.P(c), st)
    dt = U.Z(1)
    U.call("mb_time_step", dm.struct, *[U.P(c) for c in cells], wl.cfl, *wl.diffusion, U.P(dt), st)
    w0 = U.T(wl.init(A["cells_center"])[R.cperm])
    for order in (1, 2):
        prm = _lib.MbAdvDiffParams(order, 1, *wl.diffusion)
        cs, ns = U.Z((4 if wl.dim == 2 else 8) * nc), U.Z(nn)
        ref, got = U.Z(nc), U.Z(nc)
        U.call("mb_advdiff_step", dm.struct, db.struct, prm, U.P(w0), U.P(ref), U.P(sign), None, U.P(dt), U.P(cs),
               U.P(ns), st)
        args = (dm.struct, db.struct, prm, U.P(w0), U.P(got), U.P(sign), None, U.P(dt), U.P(cs), U.P(ns))
        U.call("mb_advdiff_step_split", *args, 0, dm.nfirst, st)
        part0 = U.H(got)[:dm.nfirst].copy()
        U.call("mb_advdiff_step_split", *args, 1, dm.nfirst, st)
        assert np.array_equal(U.H(got), U.H(ref))
        assert np.array_equal(part0, U.H(ref)[:dm.nfirst])
    L = _lib.lib()
    assert L.mb_advdiff_step_split(*args, 2, dm.nfirst, st) == _lib.MB_EINVAL
    assert L.mb_advdiff_step_split(*args, 0, nc + 1, st) == _lib.MB_EINVAL


@pytest.mark.parametrize("walls", ["neumann", "reflective"])
def test_split_shallow_water_step_equals_the_whole_step(walls, cuda):
    """mb_sw_step_split part 0 (every face flux, cells [0, nfirst)) then part 1 (the other
    cells) computes exactly mb_sw_step_ex's new state and next dt."""
    import gpuutil as U
    import torch
    from manapy_b200 import _lib
    from manapy_b200.device import DeviceMesh
    wl = W.C3.scaled(n=30)
    el, vx = wl.mesh()
    A = G.build(el, vx, 2)
    nc, nf = A["nbcells"], A["nbfaces"]
    first = np.random.default_rng(7).random(nc) < 0.25
    dm = DeviceMesh(A, "cuda", first_cells=first)
    R = dm.R
    st = U.stream()
    q = [U.T(a[R.cperm]) for a in wl.init_sw(A["cells_center"])]      # h, hu, hv, hc, Z
    dt = U.Z(1)
    U.call("mb_sw_dt", dm.struct, U.P(q[0]), U.P(q[1]), U.P(q[2]), wl.cfl, wl.grav, U.P(dt), st)
    ff = torch.empty(4 * nf, dtype=torch.float64, device="cuda")
    outs = []
    for split in (False, True):
        qo = [U.Z(nc) for _ in range(4)] + [q[4]]
        dn = U.Z(1)
        args = (dm.struct, _lib.p5([U.P(t) for t in q]), _lib.p5([U.P(t) for t in qo]), wl.cfl, wl.grav, 1,
                _lib.WALLS[walls], None, U.P(ff), U.P(dt), U.P(dn))
        if split:
            U.call("mb_sw_step_split", *args, 0, dm.nfirst, st)
            U.call("mb_sw_step_split", *args, 1, dm.nfirst, st)
        else:
            U.call("mb_sw_step_ex", *args, st)
        outs.append([U.H(t) for t in qo[:4]] + [U.H(dn)])
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
    assert _lib.lib().mb_sw_step_split(*args, 2, dm.nfirst, st) == _lib.MB_EINVAL


@pytest.mark.parametrize("order", [2])
def test_edge_sums_step_equals_the_stencil_step(order, cuda):
    """Tetrahedra: the second-order step with the least-squares sums by inclusion-exclusion
    (vertex, edge and face-neighbour sums; the struct's edge tables) gives the step that
    gathers every stencil neighbour, to rounding, over several steps."""
    import gpuutil as U
    from manapy_b200 import _lib
    wl = W.C4.scaled(n=8)
    el, vx = wl.mesh()
    A = G.build(el, vx, 3)
    dm = U.mesh(A, reorder=True)
    db = U.bc(A, B.resolve(A, wl.bc, wl.bc_values), dm)
    R = dm.R
    nc, nn = A["nbcells"], A["nbnodes"]
    st = U.stream()
    dm.ensure_lsq_matrix(st)
    uf, vf, wf = wl.velocity(A["faces_center"])
    sign = U.Z(4 * nc)
    u_, v_, w_ = U.T(uf[R.fperm]), U.T(vf[R.fperm]), U.T(wf[R.fperm])
    U.call("mb_cell_face_sign", dm.struct, U.P(u_), U.P(v_), U.P(w_), U.P(sign), st)
    cells = [U.Z(nc) for _ in range(3)]
    for f, cc in zip((u_, v_, w_), cells):
        U.call("mb_facetocell", dm.struct, U.P(f), U.P(cc), st)
    dt = U.Z(1)
    U.call("mb_time_step", dm.struct, *[U.P(x) for x in cells], wl.cfl, *wl.diffusion, U.P(dt), st)
    prm = _lib.MbAdvDiffParams(order, 1, *wl.diffusion)
    w0 = U.T(wl.init(A["cells_center"])[R.cperm])
    runs = []
    for sums in (False, True):
        if sums:
            assert dm.use_edge_sums()
        cs, ns = U.Z(dm.cell_scratch_size()), U.Z(nn)
        a, b = w0.clone(), U.Z(nc)
        for _ in range(6):
            U.call("mb_advdiff_step", dm.struct, db.struct, prm, U.P(a), U.P(b), U.P(sign), None, U.P(dt),
                   U.P(cs), U.P(ns), st)
            a, b = b, a
        runs.append(U.H(a))
    assert dm.cell_scratch_size() == 8 * nc + 4 * (nn + dm.nbedges)
    assert rel_max(runs[1], runs[0]) < 1e-13
    assert not np.array_equal(runs[0], U.H(w0))


def test_pinned_uploads_between_steps_match_host_arrays(cuda):
    """manapy's driver loop with the face velocities uploaded from pinned host memory every
    step and the state fetched into pinned memory gives the bits of the same loop fed numpy
    arrays."""
    import torch
    wl = W.C2.scaled(n=40)
    el, vx = wl.mesh()
    runs = []
    for pinned in (False, True):
        dom = M.Domain(dim=2, mesh=(el, vx))
        w = M.Variable(domain=dom, BC=wl.bc, values=wl.bc_values)
        u, v = M.Variable(domain=dom), M.Variable(domain=dom)
        uf, vf, _ = wl.velocity(dom.faces.center)
        w.cell = wl.init(dom.cells.center)
        S = M.AdvectionDiffusionSolver(w, vel=(u, v), conf=M.Struct(Dxx=5e-4, Dyy=5e-4, order=2, cfl=0.8))
        out = torch.empty(int(dom.nbcells), dtype=torch.float64, pin_memory=True)
        states = []
        for k in range(6):
            a, b = (1.0 + 0.1 * k) * uf, (1.0 - 0.05 * k) * vf     # a new velocity every step
            if pinned:
                pa, pb = torch.from_numpy(a).pin_memory(), torch.from_numpy(b).pin_memory()
                u.face, v.face = pa, pb
            else:
                u.face, v.face = a, b
            u.interpolate_facetocell(); v.interpolate_facetocell()
            S.stepper(); S.compute_fluxes(); S.compute_new_val()
            w.fetch("cell", out=out)
            torch.cuda.synchronize()
            states.append(out.numpy().copy())
        runs.append(states)
    for a, b in zip(*runs):
        assert np.array_equal(a, b)
