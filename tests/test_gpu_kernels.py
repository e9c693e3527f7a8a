"""Each CUDA kernel, called through the C ABI, against the oracle and the reference's outputs.

Tolerance: results may differ from the oracle only by rounding (fused
multiply-adds, division/sqrt/acos/cos implementations), so every array is
compared as max|gpu - oracle| / max|oracle| <= 1e-13.
"""
import numpy as np
import pytest

from conftest import golden, rel_max
from manapy_b200 import boundary as B, geometry as G, meshgen
import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _case(name, dim):
    g = golden(name)
    A = G.build(g["in_elements"], g["in_vertex"], dim)
    bcs = {"in": "dirichlet", "out": "dirichlet", "upper": "neumann", "bottom": "neumann"}
    if dim == 3:
        bcs.update({"front": "nonslip", "back": "neumann"})
    return g, A, B.resolve(A, bcs, {"in": 0.25, "out": -0.5})


def _random_case(dim, n, seed):
    el, vx = (meshgen.square_triangles(n, seed=seed) if dim == 2 else meshgen.cube_tetrahedra(n, seed=seed))
    A = G.build(el, vx, dim)
    # dirichlet sides first: manapy's value array is the cell array after a neumann side
    sides = ("in", "upper", "back", "out", "bottom", "front") if dim == 3 else ("in", "upper", "out", "bottom")
    kinds = ("dirichlet", "dirichlet", "dirichlet", "neumann", "nonslip", "neumann") if dim == 3 else \
        ("dirichlet", "dirichlet", "neumann", "nonslip")
    bcs = dict(zip(sides, kinds))
    vals = {s: (lambda x, y, z: 0.3 + x - 2 * y) for s, k in bcs.items() if k == "dirichlet"}
    return A, B.resolve(A, bcs, vals)


def _check_all(A, resolved, w, uf, vf, wf, D, cuda, reorder=False):
    import gpuutil as U
    m = O.Mesh(A)
    dm = U.mesh(A, reorder=reorder)
    db = U.bc(A, resolved, dm if reorder else None)
    R = dm.R
    st = U.stream()
    M = dm.struct
    # device arrays live in the mesh's numbering: permute in, permute back out
    Tc = lambda a: U.T(np.asarray(a)[R.cperm])  # noqa: E731
    Tf = lambda a: U.T(np.asarray(a)[R.fperm])  # noqa: E731
    Tn = lambda a: U.T(np.asarray(a)[R.nperm])  # noqa: E731
    Hc = lambda t: U.H(t)[R.cinv]  # noqa: E731
    Hf = lambda t: U.H(t)[R.finv]  # noqa: E731
    Hn = lambda t: U.H(t)[R.ninv]  # noqa: E731
    # ghost
    ghost_o = np.zeros(m.nf)
    O.ghost_update(m, resolved, w, ghost_o)
    wd, gd = Tc(w), U.Z(m.nf)
    U.call("mb_ghost_value", M, db.struct, U.P(wd), U.P(gd), st)
    got = Hf(gd)
    bf = A["boundaryfaces"]
    assert rel_max(got[bf], ghost_o[bf]) == 0
    gd = Tf(ghost_o)
    # facetocell
    uc_o = O.facetocell(m, uf)
    ucd = U.Z(m.nc)
    U.call("mb_facetocell", M, U.P(Tf(uf)), U.P(ucd), st)
    assert rel_max(Hc(ucd), uc_o) <= 1e-15
    # gradient + limiter
    gx, gy, gz, psi = (np.zeros(m.nc) for _ in range(4))
    O.cell_gradient(m, w, ghost_o, gx, gy, gz)
    O.barthlimiter(m, w, ghost_o, gx, gy, gz, psi)
    gxd, gyd, gzd, psid = (U.Z(m.nc) for _ in range(4))
    U.call("mb_cell_gradient", M, U.P(wd), U.P(gd), U.P(gxd), U.P(gyd), U.P(gzd), st)
    U.call("mb_barthlimiter", M, U.P(wd), U.P(gd), U.P(gxd), U.P(gyd), U.P(gzd), U.P(psid), st)
    assert rel_max(Hc(gxd), gx) < TOL and rel_max(Hc(gyd), gy) < TOL
    if m.dim == 3:
        assert rel_max(Hc(gzd), gz) < TOL
    # the limiter on the oracle's gradients, to isolate it
    psid2 = U.Z(m.nc)
    gxt, gyt, gzt = Tc(gx), Tc(gy), Tc(gz)
    U.call("mb_barthlimiter", M, U.P(wd), U.P(gd), U.P(gxt), U.P(gyt), U.P(gzt), U.P(psid2), st)
    assert rel_max(Hc(psid2), psi) < TOL
    # centre -> vertex
    node = np.zeros(m.nn)
    O.centertovertex(m, w, ghost_o, node)
    nd = U.Z(m.nn)
    U.call("mb_centertovertex", M, U.P(wd), U.P(gd), U.P(nd), st)
    assert rel_max(Hn(nd), node) < TOL
    # face gradient
    fx, fy, fz = (np.zeros(m.nf) for _ in range(3))
    O.face_gradient(m, w, ghost_o, node, fx, fy, fz, resolved.dirichletfaces, resolved.neumannfaces)
    fxd, fyd, fzd = (U.Z(m.nf) for _ in range(3))
    nodet = Tn(node)
    U.call("mb_face_gradient", M, db.struct, U.P(wd), U.P(gd), U.P(nodet), U.P(fxd), U.P(fyd), U.P(fzd), st)
    assert rel_max(Hf(fxd), fx) < TOL and rel_max(Hf(fyd), fy) < TOL
    if m.dim == 3:
        assert rel_max(Hf(fzd), fz) < TOL
    # convective, orders 1 and 2, on the oracle's gradients
    uft, vft, wft = Tf(uf), Tf(vf), Tf(wf)
    gxt, gyt, gzt, psit = Tc(gx), Tc(gy), Tc(gz), Tc(psi)
    for order in (1, 2):
        rez = np.zeros(m.nc)
        O.convective(m, rez, w, ghost_o, uf, vf, wf, gx, gy, gz, psi, order)
        rd = U.Z(m.nc)
        U.call("mb_explicitscheme_convective", M, U.P(rd), U.P(wd), U.P(gd), U.P(uft), U.P(vft), U.P(wft),
               U.P(gxt), U.P(gyt), U.P(gzt), U.P(psit), order, st)
        assert rel_max(Hc(rd), rez) < TOL, order
        gxt, gyt, gzt, psit = Tc(gx), Tc(gy), Tc(gz), Tc(psi)
        uft, vft, wft = Tf(uf), Tf(vf), Tf(wf)
    # dissipative
    dis = np.zeros(m.nc)
    O.dissipative(m, fx, fy, fz, dis, *D)
    dd = U.Z(m.nc)
    fxt, fyt, fzt = Tf(fx), Tf(fy), Tf(fz)
    U.call("mb_explicitscheme_dissipative", M, U.P(fxt), U.P(fyt), U.P(fzt), U.P(dd), *D, st)
    assert rel_max(Hc(dd), dis) < TOL
    # time step
    vc = O.facetocell(m, vf)
    wc = O.facetocell(m, wf)
    dt_o = O.time_step(m, uc_o, vc, wc, 0.8, *D)
    dtd = U.Z(1)
    a, b, c = Tc(uc_o), Tc(vc), Tc(wc)
    U.call("mb_time_step", M, U.P(a), U.P(b), U.P(c), 0.8, *D, U.P(dtd), st)
    assert rel_max(U.H(dtd)[0], dt_o) < 1e-15
    # update
    src = np.linspace(-1, 1, m.nc) * 1e-3
    w2 = w.copy()
    O.update_new_value(m, w2, rez, dis, src, dt_o)
    w2d = Tc(w)
    r_t, d_t, s_t, dt_t = Tc(rez), Tc(dis), Tc(src), U.T([dt_o])
    U.call("mb_update_new_value", M, U.P(w2d), U.P(r_t), U.P(d_t), U.P(s_t), U.P(dt_t), st)
    assert rel_max(Hc(w2d), w2) < 1e-14
    return ghost_o, gx, gy, gz, psi, node, fx, fy, fz


@pytest.mark.parametrize("name,dim", [("k2d", 2), ("k3d", 3)])
def test_kernels_on_golden_inputs(name, dim, cuda):
    g, A, resolved = _case(name, dim)
    D = (1e-3, 2e-3, 3e-3 if dim == 3 else 0.0)
    ghost, gx, gy, gz, psi, node, fx, fy, fz = _check_all(A, resolved, g["w_cell"], g["u_face"], g["v_face"],
                                                          g["wz_face"], D, cuda)
    # and the reference's own outputs
    assert rel_max(gx, g["gradx"]) < 1e-14 and rel_max(node, g["w_node"]) < 1e-13


@pytest.mark.parametrize("reorder", [False, True])
@pytest.mark.parametrize("dim,n", [(2, 40), (3, 6)])
def test_kernels_on_random_fields(dim, n, reorder, cuda):
    A, resolved = _random_case(dim, n, seed=7 + dim)
    rng = np.random.default_rng(5)
    w = rng.standard_normal(A["nbcells"])
    uf, vf, wf = (rng.uniform(-1, 1, A["nbfaces"]) for _ in range(3))
    if dim == 2:
        wf = np.zeros(A["nbfaces"])
    _check_all(A, resolved, w, uf, vf, wf, (2e-3, 1e-3, 5e-4 if dim == 3 else 0.0), cuda, reorder=reorder)


def test_srnh_flux_batch(cuda):
    import gpuutil as U
    g = golden("k2d")
    st = g["srnh_states"]
    nrm = np.column_stack([st[:, 10], st[:, 11], np.zeros(len(st))])
    mes = np.hypot(st[:, 10], st[:, 11])
    out = U.Z(5 * len(st))
    U.call("mb_srnh_flux", len(st), U.P(U.T(st[:, :10])), U.P(U.T(nrm)), U.P(U.T(mes)), 9.81, U.P(out), U.stream())
    got = U.H(out).reshape(-1, 5)
    for k in range(len(st)):
        ref = O.srnh_scheme(*st[k, :10], nrm[k], mes[k], 9.81)
        assert rel_max(got[k], ref) < 1e-12
        assert rel_max(got[k], g["srnh_flux"][k]) < 1e-12


def test_sw_kernels(cuda):
    import gpuutil as U
    g = golden("k2d")
    A = G.build(g["in_elements"], g["in_vertex"], 2)
    m = O.Mesh(A)
    dm = U.mesh(A)
    M, s = dm.struct, U.stream()
    from manapy_b200 import _lib
    for order in (1, 2):
        so = O.ShallowWaterOracle(A, order=order, cfl=0.5)
        for k, key in zip(("h", "hu", "hv", "hc", "Z"), ("sw_h", "sw_hu", "sw_hv", "sw_hc", "sw_Z")):
            so.state()[k][:] = g[key]
        dt = so.stepper()
        dtd = U.Z(1)
        U.call("mb_time_step_sw", M, U.P(U.T(so.h)), U.P(U.T(so.hu)), U.P(U.T(so.hv)), 0.5, 9.81, 0., 0.,
               U.P(dtd), s)
        assert rel_max(U.H(dtd)[0], dt) < 1e-15
        so.compute_fluxes()
        names = ("h", "hu", "hv", "hc", "Z")
        q = [U.T(so.state()[k]) for k in names]
        gh = [U.T(so.g[k]) for k in names]
        rz = [U.Z(m.nc) for _ in names]
        grads = [U.T(a) for a in (so.hgx, so.hgy, so.cgx, so.cgy)]
        ff = U.Z(5 * m.nf)
        U.call("mb_explicitscheme_convective_sw", M, _lib.p5([U.P(t) for t in rz]), _lib.p5([U.P(t) for t in q]),
               _lib.p5([U.P(t) for t in gh]), _lib.p4([U.P(t) for t in grads]), U.P(U.T(so.cpsi)), 9.81, order,
               U.P(ff), s)
        for k, t in zip(names, rz):
            ref = so.rez[k]
            got = U.H(t)
            if np.any(ref):
                assert rel_max(got, ref) < 1e-12, (k, order)
            else:
                assert np.all(got == 0)
        shu, shv = U.Z(m.nc), U.Z(m.nc)
        U.call("mb_term_source_srnh_sw", M, U.P(q[0]), U.P(q[4]), U.P(gh[0]), U.P(gh[4]), 9.81, U.P(shu), U.P(shv), s)
        assert rel_max(U.H(shu), so.src["hu"]) < 1e-12 and rel_max(U.H(shv), so.src["hv"]) < 1e-12
    # update
    so.compute_new_val()
    q0 = [U.T(g[k]) for k in ("sw_h", "sw_hu", "sw_hv", "sw_hc", "sw_Z")]
    U.call("mb_update_sw", M, _lib.p5([U.P(t) for t in q0]), _lib.p5([U.P(U.T(so.rez[k])) for k in names]),
           U.P(U.T(so.src["hu"])), U.P(U.T(so.src["hv"])), U.P(U.T([so.dt])), s)
    for k, t in zip(names, q0):
        assert rel_max(U.H(t), so.state()[k]) < 1e-14


def test_invalid_arguments_are_rejected(cuda):
    import ctypes
    from manapy_b200 import _lib
    L = _lib.lib()
    assert L.mb_facetocell(None, None, None, None) == _lib.MB_EINVAL
    assert L.mb_srnh_flux(-1, None, None, None, 9.81, None, None) == _lib.MB_EINVAL
    assert L.mb_srnh_flux(0, None, None, None, 9.81, None, None) == _lib.MB_OK
    bad = _lib.MbMesh()
    bad.dim = 4
    assert L.mb_time_step(ctypes.byref(bad), None, None, None, 0.5, 0., 0., 0., None, None) == _lib.MB_EINVAL
