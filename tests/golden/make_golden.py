"""Generate the golden vectors in this directory by running the reference manapy.

Usage (needs the reference source tree, named by ``MANAPY_REFERENCE``; not run by
the test suite)::

    MANAPY_REFERENCE=<reference tree> python tests/golden/make_golden.py    # all parts
    MANAPY_REFERENCE=<reference tree> python tests/golden/make_golden.py --part dom2d

Each part runs in its own process because the reference compiles its
``Variable`` kernels once per process for the first dimension it sees
(``manapy/ast/core.py:85-102``).

Outputs (``*.npz``, committed):

* ``dom2d.npz`` / ``dom3d.npz``: every ``Domain`` array the explicit step
  reads, for a small seeded mesh.
* ``k2d.npz`` / ``k3d.npz``: inputs and outputs of one call of each hot-path
  kernel on seeded random fields.
* ``traj_c1.npz``: the 20,000-triangle first-order advection-diffusion run
  (200 steps), final field and dt sequence.
* ``traj_o2.npz``, ``traj_3d.npz``, ``traj_sw1.npz``, ``traj_sw2.npz``:
  short second-order 2D, 3D and shallow-water runs.
* ``traj_advec.npz``, ``traj_diff.npz``: the advection-only and diffusion-only solvers
  (``manapy/solvers/advec``, ``manapy/solvers/diffusion``), short 2D runs.
* ``k_euler.npz``: the 2D Euler kernels of ``manapy/solvers/euler/fvm_utils2d.py``
  (Neumann ghosts, Rusanov residuals, per-cell dt, update) on seeded random
  states, plus a 20-step first-order run driven by those kernels.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

import refharness  # noqa: E402,F401  (first: keeps caches out of the reference tree)
from manapy_b200 import meshgen  # noqa: E402
from manapy_b200 import workloads  # noqa: E402

PARTS = ["dom2d", "dom3d", "k2d", "k3d", "traj_c1", "traj_o2", "traj_3d", "traj_sw1", "traj_sw2", "traj_advec",
         "traj_diff", "k_euler"]


def _domain_arrays(d, dim):
    out = {
        "cells_center": d.cells.center, "cells_volume": d.cells.volume,
        "cells_faceid": d.cells.faceid, "cells_cellnid": d.cells.cellnid,
        "cells_ghostnid": d.cells.ghostnid, "cells_cellfid": d.cells.cellfid,
        "cells_nodeid": d.cells.nodeid,
        "faces_nodeid": d.faces.nodeid, "faces_cellid": d.faces.cellid,
        "faces_name": d.faces.name, "faces_normal": d.faces.normal,
        "faces_mesure": d.faces.mesure, "faces_center": d.faces.center,
        "faces_ghostcenter": d.faces.ghostcenter, "faces_airDiamond": d.faces.airDiamond,
        "faces_f_1": d.faces.f_1, "faces_f_2": d.faces.f_2,
        "faces_param1": d.faces.param1, "faces_param2": d.faces.param2,
        "faces_param3": d.faces.param3,
        "nodes_cellid": d.nodes.cellid, "nodes_ghostid": d.nodes.ghostid,
        "nodes_R_x": d.nodes.R_x, "nodes_R_y": d.nodes.R_y, "nodes_R_z": d.nodes.R_z,
        "nodes_lambda_x": d.nodes.lambda_x, "nodes_lambda_y": d.nodes.lambda_y,
        "nodes_lambda_z": d.nodes.lambda_z, "nodes_number": d.nodes.number,
        "nodes_name": d.nodes.name, "nodes_vertex": d.nodes.vertex,
        "innerfaces": d.innerfaces, "boundaryfaces": d.boundaryfaces,
        "infaces": d.infaces, "outfaces": d.outfaces, "upperfaces": d.upperfaces,
        "bottomfaces": d.bottomfaces,
    }
    if dim == 2:
        out.update({"cells_nf": d.cells.nf, "faces_f_3": d.faces.f_3, "faces_f_4": d.faces.f_4,
                    "faces_param4": d.faces.param4, "faces_dist_ortho": d.faces.dist_ortho})
    else:
        out.update({"frontfaces": d._frontfaces, "backfaces": d._backfaces})
    return {k: np.asarray(v) for k, v in out.items()}


def _ref():
    from refharness import import_reference
    import_reference()


def _run(mesh, dim):
    from refharness import ReferenceRun
    el, vx = mesh
    return ReferenceRun(el, vx, dim)


def part_dom(dim):
    if dim == 2:
        el, vx = meshgen.square_triangles(6, seed=11)
    else:
        el, vx = meshgen.cube_tetrahedra(2, seed=12)
    r = _run((el, vx), dim)
    arrs = _domain_arrays(r.domain, dim)
    arrs["in_elements"] = el
    arrs["in_vertex"] = vx
    return arrs


def _rand_fields(rng, n, nf):
    return rng.standard_normal(n), rng.standard_normal(nf)


def part_kernels(dim):
    """One call of each kernel on seeded random fields."""
    _ref()
    from manapy.ast import Variable
    from manapy.solvers.advecdiff import AdvectionDiffusionSolver
    from manapy.base.base import Struct
    if dim == 2:
        el, vx = meshgen.square_triangles(12, seed=21)
    else:
        el, vx = meshgen.cube_tetrahedra(3, seed=22)
    r = _run((el, vx), dim)
    d = r.domain
    rng = np.random.default_rng(1234 + dim)
    out = {"in_elements": el, "in_vertex": vx}
    bcs = {"in": "dirichlet", "out": "dirichlet", "upper": "neumann", "bottom": "neumann"}
    vals = {"in": 0.25, "out": -0.5}
    if dim == 3:
        bcs.update({"front": "nonslip", "back": "neumann"})
    w = Variable(domain=d, BC=bcs, values=vals)
    u = Variable(domain=d)
    v = Variable(domain=d)
    wz = Variable(domain=d)
    w.cell[:] = rng.standard_normal(d.nbcells)
    u.face[:] = rng.uniform(-1, 1, d.nbfaces)
    v.face[:] = rng.uniform(-1, 1, d.nbfaces)
    wz.face[:] = rng.uniform(-1, 1, d.nbfaces) if dim == 3 else 0.0
    out.update(w_cell=w.cell.copy(), u_face=u.face.copy(), v_face=v.face.copy(), wz_face=wz.face.copy())

    u.interpolate_facetocell()
    v.interpolate_facetocell()
    wz.interpolate_facetocell()
    out.update(u_cell=u.cell.copy(), v_cell=v.cell.copy(), wz_cell=wz.cell.copy())

    w.update_ghost_value()
    out["w_ghost"] = w.ghost.copy()
    out["dirichletfaces"] = np.asarray(w.dirichletfaces)
    out["neumannfaces"] = np.asarray(w.neumannfaces)

    w.compute_cell_gradient()
    out.update(gradx=w.gradcellx.copy(), grady=w.gradcelly.copy(), gradz=w.gradcellz.copy(),
               psi=w.psi.copy())
    w.interpolate_celltonode()
    out["w_node"] = w.node.copy()
    w.compute_face_gradient()
    out.update(gfx=w.gradfacex.copy(), gfy=w.gradfacey.copy(), gfz=w.gradfacez.copy())

    D = (1e-3, 2e-3, 3e-3 if dim == 3 else 0.0)
    for order in (1, 2):
        S = AdvectionDiffusionSolver(w, vel=(u, v, wz), conf=Struct(Dxx=D[0], Dyy=D[1], Dzz=D[2],
                                                                     order=order, cfl=0.8))
        dt = S.stepper()
        out["dt"] = np.float64(dt)
        S.explicit_convective()
        out[f"rez_o{order}"] = w.convective.copy()
        if order == 1:
            S.explicit_dissipative()
            out["dissip"] = w.dissipative.copy()
            w.source[:] = rng.standard_normal(d.nbcells) * 0.1
            out["source"] = w.source.copy()
            cell0 = w.cell.copy()
            S.compute_new_val()
            out["w_updated"] = w.cell.copy()
            w.cell[:] = cell0
            # the solver's compute_fluxes recomputes gradients for order 2;
            # restore the order-1 inputs for the next iteration of the loop.
    if dim == 2:
        out.update(_sw_kernels(d, rng))
    return out


def _sw_kernels(d, rng):
    _ref()
    from manapy.ast import Variable
    from manapy.solvers.shallowater import ShallowWaterSolver
    from manapy.solvers.shallowater import fvm_utils as swf
    from manapy.base.base import Struct
    h = Variable(domain=d)
    hu = Variable(domain=d)
    hv = Variable(domain=d)
    hc = Variable(domain=d)
    Z = Variable(domain=d)
    n = d.nbcells
    h.cell[:] = rng.uniform(0.8, 2.0, n)
    hu.cell[:] = rng.uniform(-0.3, 0.3, n)
    hv.cell[:] = rng.uniform(-0.3, 0.3, n)
    hc.cell[:] = rng.uniform(0.0, 0.5, n)
    Z.cell[:] = rng.uniform(0.0, 0.2, n)
    out = {"sw_h": h.cell.copy(), "sw_hu": hu.cell.copy(), "sw_hv": hv.cell.copy(),
           "sw_hc": hc.cell.copy(), "sw_Z": Z.cell.copy()}
    for order in (1, 2):
        S = ShallowWaterSolver(h, hvel=(hu, hv), hc=hc, Z=Z, conf=Struct(order=order, cfl=0.5))
        S.stepper()
        out["sw_dt"] = np.float64(S.dt)
        S.update_ghost_values()
        S.explicit_convective()
        for nm, var in (("h", h), ("hu", hu), ("hv", hv), ("hc", hc), ("Z", Z)):
            out[f"sw_rez_{nm}_o{order}"] = var.convective.copy()
        if order == 2:
            out.update(sw_hgx=h.gradcellx.copy(), sw_hgy=h.gradcelly.copy(),
                       sw_hcpsi=hc.psi.copy(), sw_hcgx=hc.gradcellx.copy(),
                       sw_hcgy=hc.gradcelly.copy())
        S.update_term_source()
        out[f"sw_src_hu_o{order}"] = hu.source.copy()
        out[f"sw_src_hv_o{order}"] = hv.source.copy()
    cells0 = [x.cell.copy() for x in (h, hu, hv, hc, Z)]
    S.compute_new_val()
    for nm, var in (("h", h), ("hu", hu), ("hv", hv), ("hc", hc), ("Z", Z)):
        out[f"sw_new_{nm}"] = var.cell.copy()
    for x, c in zip((h, hu, hv, hc, Z), cells0):
        x.cell[:] = c
    # one srnh flux evaluation on a handful of random states (A12)
    rs = np.random.default_rng(99)
    states = np.column_stack([rs.uniform(-0.5, 0.5, 16), rs.uniform(-0.5, 0.5, 16),
                              rs.uniform(-0.5, 0.5, 16), rs.uniform(-0.5, 0.5, 16),
                              rs.uniform(0.5, 2.0, 16), rs.uniform(0.5, 2.0, 16),
                              rs.uniform(0, 1, 16), rs.uniform(0, 1, 16),
                              rs.uniform(0, 0.2, 16), rs.uniform(0, 0.2, 16),
                              rs.uniform(-1, 1, 16), rs.uniform(-1, 1, 16)])
    fl = np.zeros((16, 5))
    for k in range(16):
        nrm = np.array([states[k, 10], states[k, 11], 0.0])
        mes = float(np.hypot(nrm[0], nrm[1]))
        f = np.zeros(5)
        swf.srnh_scheme(*states[k, :10], nrm, mes, 9.81, f)
        fl[k] = f
    out["srnh_states"] = states
    out["srnh_flux"] = fl
    return out


def _adv_run(dim, mesh, init, vel, D, order, cfl, steps, bcs, vals, snap=(), solver="advecdiff"):
    _ref()
    from manapy.ast import Variable
    from manapy.base.base import Struct
    if solver == "advec":
        from manapy.solvers.advec import AdvectionSolver as AdvectionDiffusionSolver
    elif solver == "diffusion":
        from manapy.solvers.diffusion import DiffusionSolver as AdvectionDiffusionSolver
    else:
        from manapy.solvers.advecdiff import AdvectionDiffusionSolver
    r = _run(mesh, dim)
    d = r.domain
    w = Variable(domain=d, BC=bcs, values=vals)
    u = Variable(domain=d)
    v = Variable(domain=d)
    wv = Variable(domain=d)
    fc = d.faces.center
    cc = d.cells.center
    uf, vf, wf = vel(fc)
    u.face[:] = uf
    v.face[:] = vf
    wv.face[:] = wf
    u.interpolate_facetocell()
    v.interpolate_facetocell()
    wv.interpolate_facetocell()
    w.cell[:] = init(cc)
    w0 = w.cell.copy()
    S = AdvectionDiffusionSolver(w, vel=(u, v, wv), conf=Struct(Dxx=D[0], Dyy=D[1], Dzz=D[2],
                                                                 order=order, cfl=cfl))
    dts = []
    snaps = {}
    t0 = time.perf_counter()
    for it in range(steps):
        dts.append(S.stepper())
        S.compute_fluxes()
        S.compute_new_val()
        if it + 1 in snap:
            snaps[f"w_step{it + 1}"] = w.cell.copy()
    el = time.perf_counter() - t0
    out = {"w0": w0, "w_final": w.cell.copy(), "dts": np.array(dts), "steps": steps,
           "seconds": el, "cells": d.nbcells}
    out.update(snaps)
    return out


def part_traj(name):
    if name == "traj_c1":
        wl = workloads.C1
        el, vx = meshgen.square_triangles(wl.n, seed=wl.seed)
        out = _adv_run(2, (el, vx), wl.init, wl.velocity, wl.diffusion, wl.order, wl.cfl,
                       wl.steps, wl.bc, wl.bc_values, snap=(1, 10, 100))
    elif name == "traj_o2":
        wl = workloads.C2.scaled(n=32, steps=100)
        el, vx = meshgen.square_triangles(wl.n, seed=wl.seed)
        out = _adv_run(2, (el, vx), wl.init, wl.velocity, wl.diffusion, wl.order, wl.cfl,
                       wl.steps, wl.bc, wl.bc_values, snap=(1, 10))
    elif name == "traj_3d":
        wl = workloads.C4.scaled(n=6, steps=30)
        el, vx = meshgen.cube_tetrahedra(wl.n, seed=wl.seed)
        out = _adv_run(3, (el, vx), wl.init, wl.velocity, wl.diffusion, wl.order, wl.cfl,
                       wl.steps, wl.bc, wl.bc_values, snap=(1, 10))
    elif name in ("traj_advec", "traj_diff"):
        wl = workloads.C2.scaled(n=24, steps=60)
        el, vx = meshgen.square_triangles(wl.n, seed=wl.seed)
        if name == "traj_advec":
            out = _adv_run(2, (el, vx), wl.init, wl.velocity, (0.0, 0.0, 0.0), 2, wl.cfl, wl.steps, wl.bc,
                           wl.bc_values, snap=(1, 10), solver="advec")
        else:
            out = _adv_run(2, (el, vx), wl.init, wl.velocity, (1e-3, 1e-3, 0.0), 1, wl.cfl, wl.steps, wl.bc,
                           wl.bc_values, snap=(1, 10), solver="diffusion")
    else:
        order = 1 if name == "traj_sw1" else 2
        wl = workloads.C3.scaled(n=30, steps=100 if order == 1 else 60, order=order)
        el, vx = meshgen.square_triangles(wl.n, seed=wl.seed)
        out = _sw_run((el, vx), wl)
    out["in_elements"] = el
    out["in_vertex"] = vx
    return out


def _sw_run(mesh, wl):
    _ref()
    from manapy.ast import Variable
    from manapy.solvers.shallowater import ShallowWaterSolver
    from manapy.base.base import Struct
    r = _run(mesh, 2)
    d = r.domain
    h, hu, hv, hc, Z = (Variable(domain=d) for _ in range(5))
    h0, hu0, hv0, hc0, Z0 = wl.init_sw(d.cells.center)
    h.cell[:] = h0
    hu.cell[:] = hu0
    hv.cell[:] = hv0
    hc.cell[:] = hc0
    Z.cell[:] = Z0
    S = ShallowWaterSolver(h, hvel=(hu, hv), hc=hc, Z=Z,
                           conf=Struct(order=wl.order, cfl=wl.cfl, grav=wl.grav))
    dts = []
    mass = []
    t0 = time.perf_counter()
    for it in range(wl.steps):
        S.stepper()
        S.compute_fluxes()
        dts.append(S.dt)
        S.compute_new_val()
        mass.append(float(np.sum(h.cell * d.cells.volume)))
    el = time.perf_counter() - t0
    return {"h0": h0, "hu0": hu0, "hv0": hv0, "hc0": hc0, "Z0": Z0,
            "h_final": h.cell.copy(), "hu_final": hu.cell.copy(), "hv_final": hv.cell.copy(),
            "hc_final": hc.cell.copy(), "Z_final": Z.cell.copy(), "dts": np.array(dts),
            "mass": np.array(mass), "steps": wl.steps, "order": wl.order, "seconds": el,
            "cells": d.nbcells}


def part_euler():
    """The Euler kernels of ``manapy/solvers/euler/fvm_utils2d.py`` composed into a step:
    Neumann ghosts (names 1-4), Rusanov residuals, per-cell dt and its min, update."""
    _ref()
    from manapy.solvers.euler import fvm_utils2d as E
    el, vx = meshgen.square_triangles(7, seed=21)
    d = _run((el, vx), 2).domain
    nc, nf = d.nbcells, d.nbfaces
    gamma, cfl = 1.4, 0.5
    rng = np.random.default_rng(2024)
    rho = rng.uniform(0.5, 2.0, nc)
    P = rng.uniform(0.5, 2.0, nc)
    rhou = rng.uniform(-0.5, 0.5, nc)
    rhov = rng.uniform(-0.5, 0.5, nc)
    rhoE = P / (gamma - 1) + 0.5 * (rhou * rhou + rhov * rhov) / rho
    out = {"in_elements": el, "in_vertex": vx, "gamma": gamma, "cfl": cfl,
           "rho0": rho.copy(), "P0": P.copy(), "rhou0": rhou.copy(), "rhov0": rhov.copy(), "rhoE0": rhoE.copy()}
    cellid = np.ascontiguousarray(d.faces.cellid, dtype=np.int32)
    name = np.ascontiguousarray(d.faces.name, dtype=np.uint32)
    normal = np.ascontiguousarray(d.faces.normal, dtype=np.float64)
    mesure = np.ascontiguousarray(d.faces.mesure, dtype=np.float64)
    centerf = np.ascontiguousarray(d.faces.center, dtype=np.float64)
    faceid = np.ascontiguousarray(d.cells.faceid, dtype=np.int32)
    vol = np.ascontiguousarray(d.cells.volume, dtype=np.float64)
    halofid = np.zeros(1, dtype=np.int32)
    hal = [np.zeros(1) for _ in range(5)]

    def one_step(rho, P, rhou, rhov, rhoE):
        g = [np.zeros(nf) for _ in range(5)]
        ug, vg = np.zeros(nf), np.zeros(nf)
        E.ghost_value_Neumann(g[0], g[1], g[2], g[3], ug, vg, g[4], rho, P, rhou, rhov, rhoE, cellid, name, normal,
                              mesure, centerf, 0.0)
        rez = [np.zeros(nc) for _ in range(4)]
        E.explicitscheme_euler_2d_rusanov(*rez, rho, P, rhou, rhov, rhoE, *g, *hal, cellid, halofid, normal, mesure,
                                          name, gamma)
        dt_c = np.zeros(nc)
        E.time_step_euler_2d(rho, P, rhou, rhov, cfl, normal, mesure, vol, faceid, gamma, dt_c)
        return g, ug, vg, rez, dt_c

    g, ug, vg, rez, dt_c = one_step(rho, P, rhou, rhov, rhoE)
    for k, a in zip(("rho", "P", "rhou", "rhov", "rhoE"), g):
        out["g_" + k] = a.copy()
    out["g_u"], out["g_v"] = ug, vg
    for k, a in zip(("rho", "rhou", "rhov", "rhoE"), rez):
        out["rez_" + k] = a.copy()
    out["dt_c"] = dt_c.copy()
    dt = float(np.min(dt_c))
    E.update_euler_2d_fvc(rho, P, rhou, rhov, rhoE, *rez, gamma, dt, vol)
    for k, a in zip(("rho", "P", "rhou", "rhov", "rhoE"), (rho, P, rhou, rhov, rhoE)):
        out["new_" + k] = a.copy()
    dts = [dt]
    for _ in range(19):
        g, ug, vg, rez, dt_c = one_step(rho, P, rhou, rhov, rhoE)
        dt = float(np.min(dt_c))
        E.update_euler_2d_fvc(rho, P, rhou, rhov, rhoE, *rez, gamma, dt, vol)
        dts.append(dt)
    for k, a in zip(("rho", "P", "rhou", "rhov", "rhoE"), (rho, P, rhou, rhov, rhoE)):
        out["final_" + k] = a.copy()
    out["dts"] = np.array(dts)
    return out


def run_part(part):
    t0 = time.perf_counter()
    if part == "dom2d":
        out = part_dom(2)
    elif part == "dom3d":
        out = part_dom(3)
    elif part == "k2d":
        out = part_kernels(2)
    elif part == "k3d":
        out = part_kernels(3)
    elif part == "k_euler":
        out = part_euler()
    else:
        out = part_traj(part)
    np.savez_compressed(os.path.join(HERE, part + ".npz"), **out)
    print(f"{part}: {time.perf_counter() - t0:.1f}s", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--part", choices=PARTS)
    args = ap.parse_args()
    if args.part:
        run_part(args.part)
        return
    for p in PARTS:
        subprocess.run([sys.executable, __file__, "--part", p], check=True)


if __name__ == "__main__":
    main()
