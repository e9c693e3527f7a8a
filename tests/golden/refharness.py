"""Run the reference manapy in-process, unmodified, to produce golden vectors.

Only ``make_golden.py`` uses this module, and only where the reference source
tree is present (it is not present where the GPU tests run; those read the
committed ``*.npz`` files instead).

The reference needs three things that are absent here, all replaced without
touching its source:

* ``mpi4py``: a one-rank stub (``COMM_WORLD`` of size 1; ``allreduce`` is the
  identity; the neighbour all-to-alls are no-ops because a one-rank domain has
  no halo cells, ``manapy/comms/communication.py:83-145``).
* ``meshio``: imported at ``manapy/ddm/domain.py:11`` but unused by the step.
* ``h5py``: ``read_mesh_file`` (``manapy/ddm/pure_ddm.py:13-33``) is replaced by
  a function returning the same tuple for an in-memory mesh.

``Domain()`` wipes ``./results`` (``manapy/ddm/domain.py:162-184``), so the
harness runs it inside a temporary working directory.
"""
from __future__ import annotations

import os
import sys
import tempfile
import types

import numpy as np

# The reference source tree: the directory holding the ``manapy`` package, given by the
# environment (``MANAPY_REFERENCE=<path> python tests/golden/make_golden.py``).
REFERENCE_ROOT = os.environ.get("MANAPY_REFERENCE")

# The reference tree is read-only input: keep Python's bytecode and numba's on-disk
# kernel cache (``@njit(cache=True)`` writes next to the source) out of it.
sys.dont_write_bytecode = True
os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "manapy_reference_numba_cache"))


def _install_stubs():
    if "mpi4py" in sys.modules and getattr(sys.modules["mpi4py"], "_is_stub", False):
        return

    class _Req:
        def Wait(self, *a, **k):
            return None

    class _Datatype:
        def Create_contiguous(self, n):
            return self

        def Commit(self):
            return self

        def Free(self):
            return None

    class _Comm:
        def Get_size(self):
            return 1

        def Get_rank(self):
            return 0

        def Barrier(self):
            return None

        def barrier(self):
            return None

        def allreduce(self, x, op=None):
            return x

        def reduce(self, x, op=None, root=0):
            return x

        def Reduce(self, sendbuf, recvbuf, op=None, root=0):
            try:
                recvbuf[...] = sendbuf
            except Exception:
                pass

        def bcast(self, x, root=0):
            return x

        def Create_dist_graph_adjacent(self, *a, **k):
            return self

        def Neighbor_alltoallv(self, s, r):
            return None

        def Ineighbor_alltoallv(self, s, r):
            return _Req()

    class _Request:
        @staticmethod
        def Waitall(reqs):
            return None

    mpi = types.ModuleType("mpi4py.MPI")
    mpi.COMM_WORLD = _Comm()
    mpi.MIN = "min"
    mpi.MAX = "max"
    mpi.SUM = "sum"
    mpi.DOUBLE_PRECISION = _Datatype()
    mpi.DOUBLE = mpi.DOUBLE_PRECISION
    mpi.FLOAT = _Datatype()
    mpi.INT = _Datatype()
    mpi.Wtime = lambda: __import__("time").perf_counter()
    mpi.Request = _Request
    mpi.Prequest = _Request
    pkg = types.ModuleType("mpi4py")
    pkg.MPI = mpi
    pkg._is_stub = True
    sys.modules["mpi4py"] = pkg
    sys.modules["mpi4py.MPI"] = mpi

    meshio = types.ModuleType("meshio")
    meshio.__version__ = "5.0.0"
    sys.modules["meshio"] = meshio


def import_reference():
    """Import the reference package with the stubs installed."""
    if not REFERENCE_ROOT or not os.path.isdir(os.path.join(REFERENCE_ROOT, "manapy")):
        raise RuntimeError("set MANAPY_REFERENCE to the reference source tree (the directory holding manapy/)")
    _install_stubs()
    if REFERENCE_ROOT not in sys.path:
        sys.path.insert(0, REFERENCE_ROOT)
    import manapy  # noqa: F401
    import manapy.ddm.domain as ddm_domain
    return ddm_domain


class ReferenceRun:
    """Builds the reference ``Domain`` for an in-memory mesh and keeps a temp cwd."""

    def __init__(self, elements, vertex, dim, conf=None):
        ddm_domain = import_reference()
        from manapy.base.base import Struct

        elements = np.ascontiguousarray(elements, dtype=np.int32)
        vertex = np.ascontiguousarray(vertex, dtype=np.float64)

        def read_mesh_file(size, rank, mesh_dir, precision):
            n = len(elements)
            tc = np.arange(n, dtype=np.int32)
            return (tc, elements.copy(), vertex.copy(), np.zeros((2, 2), np.int32),
                    np.zeros((2, 2), np.int32), np.zeros((2, 2), precision),
                    np.arange(n, dtype=np.int32), np.arange(n, dtype=np.int32),
                    np.arange(len(vertex), dtype=np.int32), [], [])

        ddm_domain.read_mesh_file = read_mesh_file
        self._old_cwd = os.getcwd()
        self._tmp = tempfile.TemporaryDirectory()
        os.chdir(self._tmp.name)
        try:
            if conf is None:
                conf = Struct(backend="numba", signature=True, cache=False)
            self.domain = ddm_domain.Domain(dim=dim, conf=conf)
        finally:
            os.chdir(self._old_cwd)

    def close(self):
        self._tmp.cleanup()
