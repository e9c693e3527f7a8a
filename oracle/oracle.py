"""ORACLE -- test infrastructure only.

Python front of ``fv_oracle.c``, the plain-C restatement of manapy's explicit
finite-volume kernels.  Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use it, and only as the checker or the timed
CPU baseline; the product path never imports it.

``AdvDiffOracle`` and ``ShallowWaterOracle`` run whole steps in the order of
the reference solvers (``manapy/solvers/advecdiff/system.py:149-172`` and
``manapy/solvers/shallowater/system.py:186-281``) on the mesh arrays of
``manapy_b200.geometry.build``, which the tests pin array-for-array against the
reference ``Domain``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfvoracle.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_lib = None


def build():
    """Compile ``libfvoracle.so`` next to this file."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.or_time_step.restype = ctypes.c_double
        L.or_time_step_sw.restype = ctypes.c_double
        _lib = L
    return _lib


def D(a):
    """double* of a C-contiguous float64 array (kept alive by the caller)."""
    assert a.dtype == np.float64 and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(_dp)


def I(a):  # noqa: E743
    assert a.dtype == np.int32 and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(_ip)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Mesh:
    """Reference-layout tables of one mesh, as the C kernels take them."""

    def __init__(self, A):
        from manapy_b200.geometry import padded_from_csr
        self.A = A
        self.dim = A["dim"]
        self.nc = int(A["nbcells"])
        self.nf = int(A["nbfaces"])
        self.nn = int(A["nbnodes"])
        self.center = f64(A["cells_center"])
        self.volume = f64(A["cells_volume"])
        self.faceid = i32(A["cells_faceid"])
        self.cellfid = i32(A["cells_cellfid"])
        self.nodeid = i32(A["cells_nodeid"])
        self.cellidf = i32(A["faces_cellid"])
        self.nodeidf = i32(A["faces_nodeid"])
        self.namef = i32(A["faces_name"])
        self.normal = f64(A["faces_normal"])
        self.mesure = f64(A["faces_mesure"])
        self.centerf = f64(A["faces_center"])
        self.ghostc = f64(A["faces_ghostcenter"])
        self.air = f64(A["faces_airDiamond"])
        self.f = [f64(A["faces_f_%d" % k]) for k in (1, 2, 3, 4)]
        self.vertex = f64(A["nodes_vertex"])
        self.ncellid = padded_from_csr(A["n2c_ptr"], A["n2c_idx"])
        self.nghostid = padded_from_csr(A["n2g_ptr"], A["n2g_idx"])
        self.cellnid = (padded_from_csr(A["cellnid_ptr"], A["cellnid_idx"])
                        if "cellnid_ptr" in A else None)
        self.ghostnid = padded_from_csr(A["ghostnid_ptr"], A["ghostnid_idx"])
        self.Rx, self.Ry, self.Rz = (f64(A["nodes_R_" + c]) for c in "xyz")
        self.lx, self.ly, self.lz = (f64(A["nodes_lambda_" + c]) for c in "xyz")
        self.number = i32(A["nodes_number"])
        self.inner = i32(A["innerfaces"])
        self.bnd = i32(A["boundaryfaces"])
        self.dist = f64(A["faces_dist_ortho"])
        self.nf_cell = f64(A["cells_nf"]) if "cells_nf" in A else None


# ---------------------------------------------------------------- kernels
def facetocell(m, u_face):
    out = np.zeros(m.nc)
    lib().or_facetocell(D(f64(u_face)), D(out), I(m.faceid), m.faceid.shape[1], m.nc)
    return out


def ghost_update(m, bc, w_c, w_ghost):
    """Ghost values of every boundary side (``manapy/ast/core.py:492-497``)."""
    from manapy_b200 import boundary as B
    L = lib()
    for side, (bct, faces) in bc.sides.items():
        faces = i32(faces)
        k = bc.kind[faces[0]] if len(faces) else B.G_NEUMANN
        if k == B.G_DIRICHLET:
            L.or_ghost_value(0, D(bc.value), D(w_c), D(w_ghost), I(m.cellidf), I(faces), len(faces),
                             D(bc.value), D(m.dist))
        elif k == B.G_CELL_AT_FACE:
            L.or_ghost_value(0, D(w_c), D(w_c), D(w_ghost), I(m.cellidf), I(faces), len(faces),
                             D(bc.value), D(m.dist))
        elif k == B.G_NEUMANN:
            L.or_ghost_value(1, D(w_c), D(w_c), D(w_ghost), I(m.cellidf), I(faces), len(faces),
                             D(bc.value), D(m.dist))
        elif k == B.G_NONSLIP:
            L.or_ghost_value(2, D(w_c), D(w_c), D(w_ghost), I(m.cellidf), I(faces), len(faces),
                             D(bc.value), D(m.dist))
        elif k == B.G_NEUMANN_NH:
            L.or_ghost_value(3, D(w_c), D(w_c), D(w_ghost), I(m.cellidf), I(faces), len(faces),
                             D(bc.value), D(m.dist))


def cell_gradient(m, w_c, w_ghost, gx, gy, gz):
    fn = lib().or_cell_gradient_2d if m.dim == 2 else lib().or_cell_gradient_3d
    fn(D(w_c), D(w_ghost), D(m.center), I(m.cellnid), m.cellnid.shape[1], I(m.ghostnid),
       m.ghostnid.shape[1], D(m.ghostc), m.nc, D(gx), D(gy), D(gz))


def barthlimiter(m, w_c, w_ghost, gx, gy, gz, psi):
    lib().or_barthlimiter(m.dim, D(w_c), D(w_ghost), D(gx), D(gy), D(gz), D(psi), I(m.cellidf),
                          I(m.faceid), m.faceid.shape[1], I(m.namef), D(m.center), D(m.centerf),
                          m.nc)


def centertovertex(m, w_c, w_ghost, w_n):
    lib().or_centertovertex(m.dim, D(w_c), D(w_ghost), D(m.center), I(m.ncellid),
                            m.ncellid.shape[1], I(m.nghostid), m.nghostid.shape[1], D(m.vertex),
                            D(m.ghostc), m.ghostc.shape[1], D(m.Rx), D(m.Ry), D(m.Rz), D(m.lx),
                            D(m.ly), D(m.lz), I(m.number), m.nn, D(w_n))


def face_gradient(m, w_c, w_ghost, w_node, gfx, gfy, gfz, dirichletfaces, neumannfaces):
    d = i32(dirichletfaces)
    n = i32(neumannfaces)
    if m.dim == 2:
        lib().or_face_gradient_2d(D(w_c), D(w_ghost), D(w_node), I(m.cellidf), I(m.nodeidf),
                                  m.nodeidf.shape[1], D(m.air), D(m.f[0]), D(m.f[1]), D(m.f[2]),
                                  D(m.f[3]), D(gfx), D(gfy), I(m.inner), len(m.inner), I(d), len(d),
                                  I(n), len(n))
    else:
        lib().or_face_gradient_3d(D(w_c), D(w_ghost), D(w_node), I(m.cellidf), I(m.nodeidf),
                                  m.nodeidf.shape[1], D(m.air), D(m.normal), D(m.f[0]), D(m.f[1]),
                                  D(gfx), D(gfy), D(gfz), I(m.inner), len(m.inner), I(d), len(d),
                                  I(n), len(n))


def convective(m, rez, w_c, w_ghost, uf, vf, wf, gx, gy, gz, psi, order):
    lib().or_explicitscheme_convective(m.dim, D(rez), D(w_c), D(w_ghost), D(uf), D(vf), D(wf),
                                       D(gx), D(gy), D(gz), D(psi), D(m.center), D(m.centerf),
                                       I(m.cellidf), D(m.normal), I(m.inner), len(m.inner),
                                       I(m.bnd), len(m.bnd), m.nc, int(order))


def dissipative(m, gfx, gfy, gfz, dissip, Dxx, Dyy, Dzz):
    lib().or_explicitscheme_dissipative(D(gfx), D(gfy), D(gfz), I(m.cellidf), D(m.normal),
                                        I(m.namef), m.nf, D(dissip), m.nc, ctypes.c_double(Dxx),
                                        ctypes.c_double(Dyy), ctypes.c_double(Dzz))


def time_step(m, u, v, w, cfl, Dxx, Dyy, Dzz):
    return lib().or_time_step(D(u), D(v), D(w), ctypes.c_double(cfl), D(m.normal), D(m.volume),
                              I(m.faceid), m.faceid.shape[1], m.nc, ctypes.c_double(Dxx),
                              ctypes.c_double(Dyy), ctypes.c_double(Dzz))


def update_new_value(m, w_c, rez, dissip, src, dt):
    lib().or_update_new_value(D(w_c), D(rez), D(dissip), D(src), ctypes.c_double(dt), D(m.volume),
                              m.nc)


def srnh_scheme(hu_l, hu_r, hv_l, hv_r, h_l, h_r, hc_l, hc_r, Z_l, Z_r, normal, mesure, grav):
    flux = np.zeros(5)
    nrm = f64(normal)
    c = ctypes.c_double
    lib().or_srnh_scheme(c(hu_l), c(hu_r), c(hv_l), c(hv_r), c(h_l), c(h_r), c(hc_l), c(hc_r),
                         c(Z_l), c(Z_r), D(nrm), c(mesure), c(grav), D(flux))
    return flux


def time_step_sw(m, h, hu, hv, cfl, grav, Dxx=0.0, Dyy=0.0):
    c = ctypes.c_double
    return lib().or_time_step_sw(D(h), D(hu), D(hv), c(cfl), D(m.normal), D(m.mesure),
                                 D(m.volume), I(m.faceid), m.faceid.shape[1], m.nc, c(grav), c(Dxx),
                                 c(Dyy))


# ---------------------------------------------------------------- steppers
class AdvDiffOracle:
    """The reference advection-diffusion step, kernel by kernel."""

    def __init__(self, A, bc, Dxx=0.0, Dyy=0.0, Dzz=0.0, order=1, cfl=0.4, mesh=None):
        self.m = mesh or Mesh(A)
        m = self.m
        self.bc = bc
        self.D = (float(Dxx), float(Dyy), float(Dzz))
        self.order = int(order)
        self.cfl = float(cfl)
        self.diffusion = not (Dxx == Dyy == Dzz == 0)
        z = lambda n: np.zeros(n)  # noqa: E731
        self.w = z(m.nc)
        self.ghost = z(m.nf)
        self.node = z(m.nn)
        self.gx, self.gy, self.gz = z(m.nc), z(m.nc), z(m.nc)
        self.psi = z(m.nc)
        self.gfx, self.gfy, self.gfz = z(m.nf), z(m.nf), z(m.nf)
        self.rez = z(m.nc)
        self.dissip = z(m.nc)
        self.src = z(m.nc)
        self.uf, self.vf, self.wf = z(m.nf), z(m.nf), z(m.nf)
        self.uc, self.vc, self.wc = z(m.nc), z(m.nc), z(m.nc)
        self.dt = 0.0

    def set_velocity(self, uf, vf, wf):
        self.uf, self.vf, self.wf = f64(uf).copy(), f64(vf).copy(), f64(wf).copy()
        self.uc = facetocell(self.m, self.uf)
        self.vc = facetocell(self.m, self.vf)
        self.wc = facetocell(self.m, self.wf)

    def stepper(self):
        self.dt = time_step(self.m, self.uc, self.vc, self.wc, self.cfl, *self.D)
        return self.dt

    def compute_fluxes(self):
        m = self.m
        ghost_update(m, self.bc, self.w, self.ghost)
        if self.order == 2:
            cell_gradient(m, self.w, self.ghost, self.gx, self.gy, self.gz)
            barthlimiter(m, self.w, self.ghost, self.gx, self.gy, self.gz, self.psi)
        convective(m, self.rez, self.w, self.ghost, self.uf, self.vf, self.wf, self.gx, self.gy,
                   self.gz, self.psi, self.order)
        if self.diffusion:
            centertovertex(m, self.w, self.ghost, self.node)
            face_gradient(m, self.w, self.ghost, self.node, self.gfx, self.gfy, self.gfz,
                          self.bc.dirichletfaces, self.bc.neumannfaces)
            dissipative(m, self.gfx, self.gfy, self.gfz, self.dissip, *self.D)

    def compute_new_val(self):
        update_new_value(self.m, self.w, self.rez, self.dissip, self.src, self.dt)

    def step(self):
        self.stepper()
        self.compute_fluxes()
        self.compute_new_val()
        return self.dt


class ShallowWaterOracle:
    """The reference shallow-water step (SRNH flux, bathymetry source), Neumann ghosts."""

    def __init__(self, A, order=1, cfl=0.8, grav=9.81, mesh=None):
        from manapy_b200 import boundary as B
        self.m = mesh or Mesh(A)
        m = self.m
        if m.dim != 2:
            raise ValueError("shallow water is 2D")
        self.order = int(order)
        self.cfl = float(cfl)
        self.grav = float(grav)
        self.bc = B.resolve(A, None)
        z = lambda n: np.zeros(n)  # noqa: E731
        self.h, self.hu, self.hv, self.hc, self.Z = (z(m.nc) for _ in range(5))
        self.g = {k: z(m.nf) for k in ("h", "hu", "hv", "hc", "Z")}
        self.rez = {k: z(m.nc) for k in ("h", "hu", "hv", "hc", "Z")}
        self.src = {k: z(m.nc) for k in ("h", "hu", "hv", "hc", "Z")}
        self.hgx, self.hgy, self.hgz, self.hpsi = z(m.nc), z(m.nc), z(m.nc), z(m.nc)
        self.cgx, self.cgy, self.cgz, self.cpsi = z(m.nc), z(m.nc), z(m.nc), z(m.nc)
        self.zero_c = z(m.nc)
        self.dt = 0.0

    def state(self):
        return {"h": self.h, "hu": self.hu, "hv": self.hv, "hc": self.hc, "Z": self.Z}

    def stepper(self):
        self.dt = time_step_sw(self.m, self.h, self.hu, self.hv, self.cfl, self.grav)
        return self.dt

    def compute_fluxes(self):
        m = self.m
        L = lib()
        st = self.state()
        for k in st:
            ghost_update(m, self.bc, st[k], self.g[k])
        if self.order == 2:
            cell_gradient(m, self.h, self.g["h"], self.hgx, self.hgy, self.hgz)
            barthlimiter(m, self.h, self.g["h"], self.hgx, self.hgy, self.hgz, self.hpsi)
            cell_gradient(m, self.hc, self.g["hc"], self.cgx, self.cgy, self.cgz)
            barthlimiter(m, self.hc, self.g["hc"], self.cgx, self.cgy, self.cgz, self.cpsi)
        r = self.rez
        g = self.g
        L.or_explicitscheme_convective_sw(
            D(r["h"]), D(r["hu"]), D(r["hv"]), D(r["hc"]), D(r["Z"]), D(self.h), D(self.hu),
            D(self.hv), D(self.hc), D(self.Z), D(g["h"]), D(g["hu"]), D(g["hv"]), D(g["hc"]),
            D(g["Z"]), D(self.hgx), D(self.hgy), D(self.cgx), D(self.cgy), D(self.cpsi),
            D(m.center), D(m.centerf), I(m.cellidf), D(m.mesure), D(m.normal), I(m.inner),
            len(m.inner), I(m.bnd), len(m.bnd), m.nc, ctypes.c_double(self.grav), self.order)
        s = self.src
        L.or_term_source_srnh_sw(D(s["h"]), D(s["hu"]), D(s["hv"]), D(s["hc"]), D(s["Z"]), D(self.h),
                                 D(self.Z), D(g["h"]), D(g["Z"]), I(m.nodeid), m.nodeid.shape[1],
                                 I(m.faceid), m.faceid.shape[1], I(m.cellfid), m.cellfid.shape[1],
                                 D(m.center), D(m.nf_cell), I(m.namef), D(m.vertex), m.nc,
                                 ctypes.c_double(self.grav))

    def compute_new_val(self):
        r, s = self.rez, self.src
        z = self.zero_c
        lib().or_update_sw(D(self.h), D(self.hu), D(self.hv), D(self.hc), D(self.Z), D(r["h"]),
                           D(r["hu"]), D(r["hv"]), D(r["hc"]), D(r["Z"]), D(s["h"]), D(s["hu"]),
                           D(s["hv"]), D(s["hc"]), D(s["Z"]), D(z), D(z), D(z), ctypes.c_double(0.),
                           ctypes.c_double(0.), ctypes.c_double(self.dt), D(self.m.volume), self.m.nc)

    def step(self):
        self.stepper()
        self.compute_fluxes()
        self.compute_new_val()
        return self.dt


# ---------------------------------------------------------------- Euler, 2D (manapy/solvers/euler/fvm_utils2d.py)

def _arr_ptrs(arrs):
    return (_dp * len(arrs))(*[a.ctypes.data_as(_dp) for a in arrs])


def ghost_neumann_euler_2d(m, q):
    """fvm_utils2d.py:592-646 ghost_value_Neumann: faces named 1-4 copy their cell's state.
    Returns (g[rho, P, rhou, rhov, rhoE], ug, vg) face arrays (zero elsewhere)."""
    g = [np.zeros(m.nf) for _ in range(5)]
    ug, vg = np.zeros(m.nf), np.zeros(m.nf)
    sel = np.isin(m.namef, (1, 2, 3, 4))
    c = m.cellidf[sel, 0]
    for k in range(5):
        g[k][sel] = np.asarray(q[k])[c]
    ug[sel] = g[2][sel] / g[0][sel]
    vg[sel] = g[3][sel] / g[0][sel]
    return g, ug, vg


def euler_rusanov_2d(m, q, g, gamma):
    """fvm_utils2d.py:1490-1611: residuals (rho, rhou, rhov, rhoE) of cell state q and face ghosts g."""
    q = [f64(a) for a in q]
    g = [f64(a) for a in g]
    rez = [np.zeros(m.nc) for _ in range(4)]
    lib().or_euler_rusanov_2d(_arr_ptrs(rez), _arr_ptrs(q), _arr_ptrs(g), I(m.cellidf), D(m.normal), D(m.mesure),
                              I(m.namef), m.nf, m.nc, ctypes.c_double(gamma))
    return rez


def time_step_euler_2d(m, q, cfl, gamma):
    """fvm_utils2d.py:1083-1102: per-cell dt of q = (rho, P, rhou, rhov, ...)."""
    q = [f64(a) for a in q]
    dt = np.zeros(m.nc)
    lib().or_time_step_euler_2d(D(q[0]), D(q[1]), D(q[2]), D(q[3]), ctypes.c_double(cfl), D(m.normal),
                                D(m.mesure), D(m.volume), I(m.faceid), m.faceid.shape[1], m.nc,
                                ctypes.c_double(gamma), D(dt))
    return dt


def update_euler_2d(m, q, rez, gamma, dt):
    """fvm_utils2d.py:1687-1696, in place on the float64 arrays q = (rho, P, rhou, rhov, rhoE)."""
    rez = [f64(a) for a in rez]
    lib().or_update_euler_2d(_arr_ptrs(q), _arr_ptrs(rez), ctypes.c_double(gamma), ctypes.c_double(dt),
                             D(m.volume), m.nc)


def euler_step_2d(m, q, cfl, gamma):
    """One first-order Euler step composed of the kernels above: Neumann ghosts, Rusanov
    residuals, dt = min of the per-cell dt, update (q in place).  Returns dt."""
    g, _, _ = ghost_neumann_euler_2d(m, q)
    rez = euler_rusanov_2d(m, q, g, gamma)
    dt = float(np.min(time_step_euler_2d(m, q, cfl, gamma)))
    update_euler_2d(m, q, rez, gamma, dt)
    return dt
