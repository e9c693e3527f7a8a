"""Persistent mesh cache: a cached mesh reloads array for array as built, the key follows
the mesh, and a solver on a cached mesh steps exactly as on a freshly built one."""
import os

import numpy as np
import pytest

from manapy_b200 import geometry as G, meshcache, meshgen
from manapy_b200.device import DeviceMesh


def _same(a, b):
    assert set(a) == set(b)
    for k in a:
        x, y = np.asarray(a[k]), np.asarray(b[k])
        assert x.dtype == y.dtype and x.shape == y.shape and np.array_equal(x, y, equal_nan=True), k


@pytest.mark.parametrize("dim", [2, 3])
def test_cached_mesh_reloads_as_built(tmp_path, dim):
    el, vx = meshgen.square_triangles(12, seed=4) if dim == 2 else meshgen.cube_tetrahedra(3, seed=4)
    A1, dm1, hit1 = meshcache.load_or_build(el, vx, dim, str(tmp_path))
    A2, dm2, hit2 = meshcache.load_or_build(el, vx, dim, str(tmp_path))
    assert not hit1 and hit2
    assert len(os.listdir(tmp_path)) == 1
    ref_A = G.build(el, vx, dim)
    ref = DeviceMesh(ref_A, device=None)
    for A, dm in ((A1, dm1), (A2, dm2)):
        _same(A, ref_A)
        _same(dm.t, ref.t)
        for k in ("cperm", "cinv", "fperm", "finv", "nperm", "ninv"):
            assert np.array_equal(getattr(dm.R, k), getattr(ref.R, k)), k
        assert (dm.dim, dm.nbcells, dm.nbfaces, dm.nbnodes, dm.nlf) == (ref.dim, ref.nbcells, ref.nbfaces,
                                                                        ref.nbnodes, ref.nlf)


def test_key_follows_the_mesh():
    el, vx = meshgen.square_triangles(6, seed=1)
    k = meshcache.mesh_key(el, vx, 2)
    vx2 = vx.copy()
    vx2[7, 0] += 1e-12
    assert meshcache.mesh_key(el, vx2, 2) != k
    assert meshcache.mesh_key(el, vx, 2, reorder=False) != k
    assert meshcache.mesh_key(el[::-1].copy(), vx, 2) != k
    assert meshcache.mesh_key(el.copy(), vx.copy(), 2) == k


@pytest.mark.gpu
def test_solver_on_cached_mesh_steps_identically(tmp_path, cuda):
    import manapy_b200 as M
    from manapy_b200 import workloads as W
    wl = W.C2.scaled(n=30)
    el, vx = wl.mesh()
    out = []
    for cache in (None, str(tmp_path), str(tmp_path)):
        dom = M.Domain(dim=2, mesh=(el, vx), mesh_cache=cache)
        w = M.Variable(domain=dom, BC=wl.bc, values=wl.bc_values)
        vel = [M.Variable(domain=dom) for _ in range(3)]
        for var, a in zip(vel, wl.velocity(dom.faces.center)):
            var.face = a
            var.interpolate_facetocell()
        w.cell = wl.init(dom.cells.center)
        S = M.AdvectionDiffusionSolver(w, vel=tuple(vel), conf=M.Struct(
            Dxx=wl.diffusion[0], Dyy=wl.diffusion[1], order=2, cfl=wl.cfl))
        S.advance(20)
        out.append((w.cell.copy(), dom.mesh_cache_hit))
    assert [h for _, h in out] == [False, False, True]
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][0], out[2][0])
