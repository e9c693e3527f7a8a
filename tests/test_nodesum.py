"""The node-sum form of the least-squares cell gradient (2D), on the CPU.

The fused 2D step forms each cell's least-squares sum from three node sums and its
face neighbours (``k_f2n_nodes`` / ``k_f2n_cells``) instead of reading its ~12 vertex
neighbours.  Here the same algebra runs in numpy on the device tables and is compared
with the oracle's direct sum (manapy's ``cell_gradient_2d``, ``manapy/ast/functions2d.py:5-104``)
on a seeded jittered mesh with ghosts on every boundary side.
"""
import numpy as np

from conftest import rel_max
from manapy_b200 import boundary as B, geometry as G, workloads as W
from manapy_b200.device import DeviceMesh
import oracle as O


def test_node_sum_gradient_equals_the_direct_least_squares_gradient():
    wl = W.C2.scaled(n=40)
    el, vx = wl.mesh()
    A = G.build(el, vx, 2)
    dm = DeviceMesh(A, device=None)
    T = {k: np.asarray(v) for k, v in dm.t.items()}
    R = dm.R
    rng = np.random.default_rng(9)
    w = wl.init(A["cells_center"]) + 0.1 * rng.standard_normal(A["nbcells"])
    m = O.Mesh(A)
    bc = B.resolve(A, wl.bc, {"in": 0.3, "out": -0.2, "upper": 0.1, "bottom": 0.0})
    ghost = np.zeros(m.nf)
    O.ghost_update(m, bc, w, ghost)
    gx, gy, gz = (np.zeros(m.nc) for _ in range(3))
    O.cell_gradient(m, w, ghost, gx, gy, gz)
    # the same quantities in the device numbering
    wd, gd = w[R.cperm], ghost[R.fperm]
    X = T["cell_xy"].reshape(-1, 2)
    V = T["node_coord"].reshape(-1, 2)
    nptr, nidx = T["n2c_ptr"], T["n2c_idx"]
    nn = len(nptr) - 1
    nrow = np.repeat(np.arange(nn), np.diff(nptr))
    Av = np.zeros((nn, 2))
    np.add.at(Av, nrow, (X[nidx] - V[nrow]) * wd[nidx][:, None])
    Bv = np.zeros(nn)
    np.add.at(Bv, nrow, wd[nidx])
    vt = T["cell_vtx"].reshape(-1, 4)[:, :3]
    nb = T["cell_nbr"].reshape(-1, 4)[:, :3]
    s = np.zeros((len(X), 2))
    for j in range(3):
        s += Av[vt[:, j]] + (V[vt[:, j]] - X) * Bv[vt[:, j]][:, None]
        o = nb[:, j]
        inner = o >= 0
        s[inner] -= (X[o[inner]] - X[inner]) * wd[o[inner]][:, None]
    J = s - wd[:, None] * T["cell_lsqs"].reshape(-1, 2)
    gp, gi = T["ghostnid_ptr"], T["ghostnid_idx"]
    grow = np.repeat(np.arange(len(X)), np.diff(gp))
    gc = T["face_ghostcenter"].reshape(-1, 3)[gi, :2] - X[grow]
    np.add.at(J, grow, gc * (gd[gi] - wd[grow])[:, None])
    L = T["cell_lsq"].reshape(-1, 4)
    gxd = L[:, 0] * J[:, 0] + L[:, 1] * J[:, 1]
    gyd = L[:, 1] * J[:, 0] + L[:, 2] * J[:, 1]
    assert rel_max(gxd[R.cinv], gx) < 1e-13
    assert rel_max(gyd[R.cinv], gy) < 1e-13
