"""The allocation-free step entry point against the regular one.

mb_advdiff_step_noalloc exists for callers that may not allocate device memory
(a plugin inside an application that owns all device allocations, a service
with a fixed memory budget, a loop that must not risk cudaMalloc's implicit
synchronisation).  It must give the same result as mb_advdiff_step, whose
scratch the caller allocates, call after call; this file is collected last so
that a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_max
from manapy_b200 import _lib, boundary as B, geometry as G, workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-12  # the tolerance of the whole-step parity tests


def _setup(wl):
    import gpuutil as U
    el, vx = wl.mesh()
    A = G.build(el, vx, wl.dim)
    dm = U.mesh(A, reorder=True)
    db = U.bc(A, B.resolve(A, wl.bc, wl.bc_values), dm)
    R = dm.R
    uf, vf, wf = wl.velocity(A["faces_center"])
    st = U.stream()
    sign = U.Z(4 * A["nbcells"])
    u_, v_, w_ = U.T(uf[R.fperm]), U.T(vf[R.fperm]), U.T(wf[R.fperm])
    U.call("mb_cell_face_sign", dm.struct, U.P(u_), U.P(v_), U.P(w_), U.P(sign), st)
    uc, vc, wc = U.Z(A["nbcells"]), U.Z(A["nbcells"]), U.Z(A["nbcells"])
    for src, dst in ((u_, uc), (v_, vc), (w_, wc)):
        U.call("mb_facetocell", dm.struct, U.P(src), U.P(dst), st)
    dt = U.Z(1)
    U.call("mb_time_step", dm.struct, U.P(uc), U.P(vc), U.P(wc), wl.cfl, *wl.diffusion, U.P(dt), st)
    prm = _lib.MbAdvDiffParams(wl.order, 1, *wl.diffusion)
    w0 = U.T(wl.init(A["cells_center"])[R.cperm])
    return U, A, dm, db, prm, sign, dt, w0, st


def _regular(U, A, dm, db, prm, sign, dt, w_in, st):
    nc, nn = A["nbcells"], A["nbnodes"]
    out = U.Z(nc)
    cell_scratch = U.Z((4 if A["dim"] == 2 else 8) * nc)
    node_scratch = U.Z(nn)
    U.call("mb_advdiff_step", dm.struct, db.struct, prm, U.P(w_in), U.P(out), U.P(sign), None, U.P(dt),
           U.P(cell_scratch), U.P(node_scratch), st)
    return out


@pytest.mark.parametrize("wl", [W.C2.scaled(n=120), W.C4.scaled(n=8)])
def test_noalloc_step_matches_regular_step_twice(wl, cuda):
    U, A, dm, db, prm, sign, dt, w0, st = _setup(wl)
    lib = _lib.lib()
    w1 = U.Z(A["nbcells"])
    w2 = U.Z(A["nbcells"])
    # two calls in a row; the second starts from the first one's output
    assert lib.mb_advdiff_step_noalloc(dm.struct, db.struct, prm, U.P(w0), U.P(w1), U.P(sign), None,
                                       U.P(dt), st) == _lib.MB_OK
    assert lib.mb_advdiff_step_noalloc(dm.struct, db.struct, prm, U.P(w1), U.P(w2), U.P(sign), None,
                                       U.P(dt), st) == _lib.MB_OK
    r1 = _regular(U, A, dm, db, prm, sign, dt, w0, st)
    r2 = _regular(U, A, dm, db, prm, sign, dt, r1, st)
    assert rel_max(U.H(w1), U.H(r1)) <= TOL
    assert rel_max(U.H(w2), U.H(r2)) <= TOL
    assert not np.array_equal(U.H(w1), U.H(w2))  # the two calls really advanced the state


@pytest.mark.parametrize("wl", [W.C2.scaled(n=20), W.C4.scaled(n=4)])
def test_noalloc_size_gate_at_its_limit(wl, cuda):
    """A mesh one double beyond the scratch array is refused with MB_ETOOBIG (2D needs
    4*cells + nodes doubles, 3D 8*cells + nodes); a mesh exactly at the limit passes the
    size gate and is then refused for w_in == w_out (MB_EINVAL), before any launch."""
    U, A, dm, db, prm, sign, dt, w0, st = _setup(wl)
    # doubles needed: a cells + b nodes, (a, b) = (4, 1) for triangles, (8, 1) for tetrahedra
    a, b = (4, 1) if wl.dim == 2 else (8, 1)
    limit = _lib.NOALLOC_SCRATCH_DOUBLES
    lib = _lib.lib()
    at = _lib.MbMesh.from_buffer_copy(dm.struct)
    at.nbnodes = 8000                                     # a multiple of a: a exact cell count below
    at.nbcells = (limit - b * at.nbnodes) // a
    assert a * at.nbcells + b * at.nbnodes == limit       # need == limit exactly
    rc = lib.mb_advdiff_step_noalloc(ctypes.byref(at), db.struct, prm, U.P(w0), U.P(w0), U.P(sign), None,
                                     U.P(dt), st)
    assert rc == _lib.MB_EINVAL
    over = _lib.MbMesh.from_buffer_copy(at)
    over.nbnodes = at.nbnodes + 1                          # need == limit + 1
    rc = lib.mb_advdiff_step_noalloc(ctypes.byref(over), db.struct, prm, U.P(w0), U.P(w0), U.P(sign), None,
                                     U.P(dt), st)
    assert rc == _lib.MB_ETOOBIG
