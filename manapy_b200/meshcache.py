"""Persistent mesh cache (no counterpart in manapy, which rebuilds its ``Domain`` arrays
from the partition files on every run).

``load_or_build(elements, vertex, dim, cache_dir)`` returns the host geometry ``A`` of a
mesh (``geometry.build``: manapy's ``Domain`` arrays) and its device tables built on the
host (``DeviceMesh(A, device=None)``), reading both from ``cache_dir`` when an entry for the
same mesh and the same builder exists, and writing one otherwise.  Uploading the cached
tables gives the same device mesh as building it, array for array.

The key hashes the element and vertex arrays, the dimension, the renumbering switch and
the source files of the builder (``geometry.py``, ``reorder.py``, ``device.py`` and this
file), so an entry written by another version of the builder is never read.  An entry is
one uncompressed ``.npz`` file (about 1.4 kB per triangle), written under a temporary name
and renamed, so a reader never sees a partial file and concurrent writers of one entry
leave a complete one.
"""
from __future__ import annotations

import hashlib
import os
import tempfile
from types import SimpleNamespace

import numpy as np

__all__ = ["mesh_key", "load_or_build", "entry_path"]

FORMAT = 1
_SOURCES = ("geometry.py", "reorder.py", "device.py", "meshcache.py", "host/common.hpp", "host/mesh2d.cpp",
            "host/geom3d.cpp")
_digest = None


def _sources_digest():
    global _digest
    if _digest is None:
        h = hashlib.sha256()
        here = os.path.dirname(os.path.abspath(__file__))
        for name in _SOURCES:
            with open(os.path.join(here, name), "rb") as f:
                h.update(f.read())
        _digest = h.hexdigest()
    return _digest


def mesh_key(elements, vertex, dim, reorder=True, stencil="shared"):
    """Hex key of (mesh, dimension, renumbering, stencil layout, builder sources)."""
    h = hashlib.sha256()
    h.update(b"manapy_b200 mesh cache %d %d %d %s " % (FORMAT, int(dim), int(bool(reorder)), stencil.encode()))
    h.update(_sources_digest().encode())
    for a in (np.ascontiguousarray(elements, dtype=np.int32), np.ascontiguousarray(vertex, dtype=np.float64)):
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()[:40]


def entry_path(cache_dir, key):
    return os.path.join(cache_dir, "mesh-%s.npz" % key)


def _save(path, A, dm):
    arrays = {}
    for k, v in A.items():
        arrays["A/" + k] = np.asarray(v)
    for k, v in dm.t.items():
        arrays["T/" + k] = np.asarray(v)
    for k in ("cperm", "cinv", "fperm", "finv", "nperm", "ninv"):
        arrays["R/" + k] = np.asarray(getattr(dm.R, k))
    arrays["R/enabled"] = np.asarray(bool(dm.R.enabled))
    arrays["T/stencil"] = np.asarray(dm.stencil)
    d = os.path.dirname(path)
    fd, tmp = tempfile.mkstemp(prefix=".mesh-", suffix=".npz.tmp", dir=d)
    try:
        with os.fdopen(fd, "wb") as f:
            np.savez(f, **arrays)
        os.replace(tmp, path)
    except BaseException:
        if os.path.exists(tmp):
            os.unlink(tmp)
        raise


def _load(path):
    from .device import DeviceMesh
    A, T, R = {}, {}, {}
    with np.load(path, allow_pickle=False) as z:
        for name in z.files:
            part, k = name.split("/", 1)
            v = z[name]
            if part == "A":
                A[k] = int(v) if k in ("dim", "nbcells", "nbfaces", "nbnodes") else v
            elif part == "T":
                T[k] = v
            else:
                R[k] = v
    dm = DeviceMesh.from_host_tables(A, T, SimpleNamespace(
        cperm=R["cperm"], cinv=R["cinv"], fperm=R["fperm"], finv=R["finv"], nperm=R["nperm"], ninv=R["ninv"],
        enabled=bool(R["enabled"])))
    return A, dm


def load_or_build(elements, vertex, dim, cache_dir, reorder=True, stencil="shared"):
    """(A, host-built DeviceMesh, hit) for the mesh, through the cache in ``cache_dir``."""
    from . import geometry
    from .device import DeviceMesh
    os.makedirs(cache_dir, exist_ok=True)
    path = entry_path(cache_dir, mesh_key(elements, vertex, dim, reorder, stencil))
    if os.path.exists(path):
        A, dm = _load(path)
        return A, dm, True
    dm = None
    if reorder:
        from .domain import build_host_mesh
        A, dm = build_host_mesh(elements, vertex, int(dim), stencil)
    else:
        A = geometry.build(elements, vertex, int(dim))
    if len(A["unmatched_boundary_faces"]):
        return A, None, False          # the caller raises manapy's error; nothing is cached
    if dm is None:
        dm = DeviceMesh(A, device=None, reorder=reorder, stencil=stencil)
    _save(path, A, dm)
    return A, dm, False
