"""The maintainer path: ``CUDABackend.for_manapy_domain`` on a Domain that manapy built.

A maintainer who keeps manapy's own ``Domain`` and swaps only the kernel backend
(``manapy/backends/cpu/backend.py:69-93``) hands that Domain to
``CUDABackend.for_manapy_domain``, which rebuilds the device tables from the
Domain's element and vertex arrays.  Kernel calls then take their mesh arguments
from manapy's Domain, so the rebuilt tables must number cells, faces and nodes
exactly as manapy does.  ``tests/golden/dom2d.npz`` / ``dom3d.npz`` hold every
Domain array of a reference-built Domain (``tests/golden/make_golden.py``); with
``MANAPY_REFERENCE`` set, the same check also runs against a live reference Domain.
"""
import os
import types

import numpy as np
import pytest

from conftest import golden
from manapy_b200.backend import CUDABackend

INT_TABLES = ("cells_nodeid", "cells_faceid", "faces_cellid", "faces_nodeid", "faces_name", "innerfaces",
              "boundaryfaces")
REAL_TABLES = ("cells_center", "cells_volume", "faces_normal", "faces_mesure", "faces_center",
               "faces_ghostcenter", "faces_airDiamond", "nodes_vertex")


def _fake_manapy_domain(dim, nodeid, vertex):
    return types.SimpleNamespace(dim=dim, cells=types.SimpleNamespace(nodeid=nodeid),
                                 nodes=types.SimpleNamespace(vertex=vertex))


def _compare(A, ref):
    for k in INT_TABLES:
        a, r = np.asarray(A[k]), np.asarray(ref[k])
        if k in ("cells_nodeid", "cells_faceid", "faces_nodeid") and a.shape[1] != r.shape[1]:
            w = min(a.shape[1], r.shape[1])
            a, r = a[:, :w - 1], r[:, :w - 1]  # manapy keeps the row count in its last column
        assert np.array_equal(a.astype(np.int64), r.astype(np.int64)), k
    for k in REAL_TABLES:
        a, r = np.asarray(A[k], np.float64), np.asarray(ref[k], np.float64)
        if a.ndim == 2 and a.shape[1] != r.shape[1]:
            w = min(a.shape[1], r.shape[1])
            a, r = a[:, :w], r[:, :w]
        scale = max(float(np.max(np.abs(r))), 1e-300)
        assert float(np.max(np.abs(a - r))) <= 4e-16 * scale, k


@pytest.mark.parametrize("name,dim", [("dom2d", 2), ("dom3d", 3)])
def test_for_manapy_domain_numbers_the_mesh_as_manapy(name, dim):
    g = golden(name)
    be = CUDABackend.for_manapy_domain(_fake_manapy_domain(dim, g["cells_nodeid"], g["nodes_vertex"]),
                                       device="cpu")
    _compare(be.domain.host_arrays, g)
    assert be.compile(types.SimpleNamespace(__name__="facetocell")) is not None


def test_for_manapy_domain_on_a_live_reference_domain():
    if not os.environ.get("MANAPY_REFERENCE"):
        pytest.skip("MANAPY_REFERENCE (the reference source tree) is not set")
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from refharness import ReferenceRun
    from manapy_b200 import meshgen
    el, vx = meshgen.square_triangles(7, seed=11)
    run = ReferenceRun(el, vx, 2)
    try:
        d = run.domain
        ref = {"cells_nodeid": d.cells.nodeid, "cells_faceid": d.cells.faceid, "faces_cellid": d.faces.cellid,
               "faces_nodeid": d.faces.nodeid, "faces_name": d.faces.name, "innerfaces": d.innerfaces,
               "boundaryfaces": d.boundaryfaces, "cells_center": d.cells.center, "cells_volume": d.cells.volume,
               "faces_normal": d.faces.normal, "faces_mesure": d.faces.mesure, "faces_center": d.faces.center,
               "faces_ghostcenter": d.faces.ghostcenter, "faces_airDiamond": d.faces.airDiamond,
               "nodes_vertex": d.nodes.vertex}
        be = CUDABackend.for_manapy_domain(d, device="cpu")
        _compare(be.domain.host_arrays, ref)
    finally:
        run.close()
