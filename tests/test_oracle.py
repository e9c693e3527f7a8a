"""The oracle (C restatement of the reference kernels) against the reference's own outputs."""
import numpy as np
import pytest

from conftest import golden, rel_max
from manapy_b200 import boundary as B, geometry as G, workloads as W
import oracle as O

TOL = 1e-14  # the oracle rounds differently from Numba's fastmath build only in the last bits


def _setup(name, dim):
    g = golden(name)
    A = G.build(g["in_elements"], g["in_vertex"], dim)
    bcs = {"in": "dirichlet", "out": "dirichlet", "upper": "neumann", "bottom": "neumann"}
    if dim == 3:
        bcs.update({"front": "nonslip", "back": "neumann"})
    bc = B.resolve(A, bcs, {"in": 0.25, "out": -0.5})
    return g, A, O.Mesh(A), bc


@pytest.mark.parametrize("name,dim", [("k2d", 2), ("k3d", 3)])
def test_kernels_match_reference(name, dim):
    g, A, m, bc = _setup(name, dim)
    assert np.array_equal(bc.dirichletfaces, g["dirichletfaces"])
    assert np.array_equal(bc.neumannfaces, g["neumannfaces"])
    w = g["w_cell"].copy()
    assert rel_max(O.facetocell(m, g["u_face"]), g["u_cell"]) == 0
    ghost = np.zeros(m.nf)
    O.ghost_update(m, bc, w, ghost)
    assert rel_max(ghost, g["w_ghost"]) == 0
    gx, gy, gz, psi = (np.zeros(m.nc) for _ in range(4))
    O.cell_gradient(m, w, ghost, gx, gy, gz)
    assert rel_max(gx, g["gradx"]) < TOL and rel_max(gy, g["grady"]) < TOL
    if dim == 3:
        assert rel_max(gz, g["gradz"]) < TOL
    O.barthlimiter(m, w, ghost, g["gradx"].copy(), g["grady"].copy(), g["gradz"].copy(), psi)
    assert rel_max(psi, g["psi"]) < TOL
    node = np.zeros(m.nn)
    O.centertovertex(m, w, ghost, node)
    assert rel_max(node, g["w_node"]) < 1e-13
    gfx, gfy, gfz = (np.zeros(m.nf) for _ in range(3))
    O.face_gradient(m, w, ghost, g["w_node"].copy(), gfx, gfy, gfz, bc.dirichletfaces, bc.neumannfaces)
    assert rel_max(gfx, g["gfx"]) < TOL and rel_max(gfy, g["gfy"]) < TOL
    D = (1e-3, 2e-3, 3e-3 if dim == 3 else 0.0)
    vc = O.facetocell(m, g["v_face"])
    wc = O.facetocell(m, g["wz_face"])
    assert O.time_step(m, O.facetocell(m, g["u_face"]), vc, wc, 0.8, *D) == float(g["dt"])
    for order in (1, 2):
        rez = np.zeros(m.nc)
        O.convective(m, rez, w, ghost, g["u_face"], g["v_face"], g["wz_face"], g["gradx"].copy(),
                     g["grady"].copy(), g["gradz"].copy(), g["psi"].copy(), order)
        assert rel_max(rez, g["rez_o%d" % order]) < TOL
    dis = np.zeros(m.nc)
    O.dissipative(m, g["gfx"].copy(), g["gfy"].copy(), g["gfz"].copy(), dis, *D)
    assert rel_max(dis, g["dissip"]) < TOL
    w2 = w.copy()
    O.update_new_value(m, w2, g["rez_o1"].copy(), g["dissip"].copy(), g["source"].copy(), float(g["dt"]))
    assert rel_max(w2, g["w_updated"]) < TOL


def test_sw_kernels_match_reference():
    g, A, m, _ = _setup("k2d", 2)
    for k in range(16):
        s = g["srnh_states"][k]
        f = O.srnh_scheme(*s[:10], np.array([s[10], s[11], 0.0]), float(np.hypot(s[10], s[11])), 9.81)
        assert rel_max(f, g["srnh_flux"][k]) < 1e-14
    so = O.ShallowWaterOracle(A, order=1, cfl=0.5)
    for order in (1, 2):
        so.order = order
        for k, key in zip(("h", "hu", "hv", "hc", "Z"), ("sw_h", "sw_hu", "sw_hv", "sw_hc", "sw_Z")):
            so.state()[k][:] = g[key]
        assert rel_max(so.stepper(), g["sw_dt"]) < 1e-15
        so.compute_fluxes()
        for v in ("h", "hu", "hv", "hc"):
            assert rel_max(so.rez[v], g["sw_rez_%s_o%d" % (v, order)]) < 1e-14, (v, order)
        assert np.all(so.rez["Z"] == 0) and np.all(g["sw_rez_Z_o%d" % order] == 0)
        # the source term subtracts nearly equal face terms: 1e-14 of its max
        assert rel_max(so.src["hu"], g["sw_src_hu_o%d" % order]) < 1e-13
        assert rel_max(so.src["hv"], g["sw_src_hv_o%d" % order]) < 1e-13
    so.compute_new_val()
    for v in ("h", "hu", "hv", "hc", "Z"):
        assert rel_max(so.state()[v], g["sw_new_" + v]) < 1e-14


@pytest.mark.parametrize("name,wl", [("traj_c1", W.C1), ("traj_o2", W.C2.scaled(n=32, steps=100)),
                                     ("traj_3d", W.C4.scaled(n=6, steps=30))])
def test_trajectories_match_reference(name, wl):
    g = golden(name)
    A = G.build(g["in_elements"], g["in_vertex"], wl.dim)
    bc = B.resolve(A, wl.bc, wl.bc_values)
    o = O.AdvDiffOracle(A, bc, *wl.diffusion, order=wl.order, cfl=wl.cfl)
    o.set_velocity(*wl.velocity(A["faces_center"]))
    o.w[:] = wl.init(A["cells_center"])
    assert rel_max(o.w, g["w0"]) == 0
    dts = [o.step() for _ in range(int(g["steps"]))]
    assert rel_max(np.array(dts), g["dts"]) < 1e-15
    assert rel_max(o.w, g["w_final"]) < 1e-14


@pytest.mark.parametrize("name", ["traj_sw1", "traj_sw2"])
def test_sw_trajectories_match_reference(name):
    import os
    from conftest import GOLDEN
    if not os.path.exists(os.path.join(GOLDEN, name + ".npz")):
        pytest.skip("fixture not generated")
    g = golden(name)
    wl = W.C3.scaled(n=30, order=int(g["order"]), steps=int(g["steps"]))
    A = G.build(g["in_elements"], g["in_vertex"], 2)
    so = O.ShallowWaterOracle(A, order=wl.order, cfl=wl.cfl, grav=wl.grav)
    for k, a in zip(("h", "hu", "hv", "hc", "Z"), wl.init_sw(A["cells_center"])):
        so.state()[k][:] = a
    dts = []
    mass = []
    for _ in range(wl.steps):
        dts.append(so.step())
        mass.append(np.sum(so.h * so.m.volume))
    assert rel_max(np.array(dts), g["dts"]) < 1e-13
    assert rel_max(np.array(mass), g["mass"]) < 1e-14
    for k in ("h", "hu", "hv"):
        assert rel_max(so.state()[k], g[k + "_final"]) < 1e-12, k


@pytest.mark.parametrize("name", ["traj_advec", "traj_diff"])
def test_oracle_matches_reference_advection_and_diffusion_solvers(name):
    """manapy's advection-only and diffusion-only solvers are the advection-diffusion step
    with no diffusion / with zero velocity (their own time steps differ only where those
    terms vanish)."""
    from manapy_b200 import workloads as W
    g = golden(name)
    wl = W.C2.scaled(n=24)
    A = G.build(g["in_elements"], g["in_vertex"], 2)
    if name == "traj_advec":
        D, order, vel = (0., 0., 0.), 2, wl.velocity(A["faces_center"])
    else:
        D, order = (1e-3, 1e-3, 0.), 1
        vel = tuple(np.zeros(A["nbfaces"]) for _ in range(3))
    o = O.AdvDiffOracle(A, B.resolve(A, wl.bc, wl.bc_values), *D, order=order, cfl=wl.cfl)
    o.set_velocity(*vel)
    o.w[:] = g["w0"]
    dts = [o.step() for _ in range(int(g["steps"]))]
    assert rel_max(np.array(dts), g["dts"]) < 1e-15
    assert rel_max(o.w, g["w_final"]) < 1e-14
