"""``Variable``: a field on a ``Domain``, stored on the GPU.

Mirrors ``manapy.ast.Variable`` (``manapy/ast/core.py:24-575``): the same
arrays (``cell``, ``node``, ``face``, ``ghost``, ``gradcellx/y/z``, ``psi``,
``gradfacex/y/z`` and any solver terms such as ``convective``), the same
boundary-condition set-up and the same methods, each running the CUDA kernel
of the manapy function it names.

Storage: every array lives in a device tensor.  Reading an attribute
(``var.cell``) returns a host numpy array synchronised from the device; the
host array is then treated as possibly modified and is uploaded again before
the next kernel reads it, so ``var.cell[:] = ...`` works as in manapy.  Keep
no reference to a returned array across kernel calls: read the attribute
again to see new values.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from . import boundary as B

__all__ = ["Variable"]

_CELL = ("cell", "gradcellx", "gradcelly", "gradcellz", "psi")
_FACE = ("face", "ghost", "gradfacex", "gradfacey", "gradfacez")
_NODE = ("node",)


class _Store:
    """Device tensors (in the device mesh numbering) with lazily synchronised host
    mirrors (in manapy's numbering)."""

    def __init__(self, device, mesh_fn):
        self.dev = {}
        self.host = {}
        self.kind = {}   # "cell" / "face" / "node" / None: which permutation applies
        self.state = {}  # "dev": device authoritative; "host": host authoritative
        self.lazy = {}   # name -> callable materialising the device tensor on demand
        self.version = {}  # bumped whenever the device contents may change
        self.device = device
        self.mesh_fn = mesh_fn

    def add(self, name, n, kind=None):
        self.dev[name] = torch.zeros(int(n), dtype=torch.float64, device=self.device)
        self.state[name] = "dev"
        self.version[name] = 0
        self.kind[name] = kind if n else None

    def _upload(self, name, arr):
        if isinstance(arr, torch.Tensor):  # e.g. pinned host memory: asynchronous copy
            src = arr.to(device=self.device, dtype=torch.float64, non_blocking=True)
        else:
            src = torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float64)).to(self.device)
        if self.kind[name] is None:
            self.dev[name].copy_(src)
        else:
            self.mesh_fn().to_device_order(self.kind[name], src, self.dev[name])

    def d(self, name):
        """Device tensor, uploading host edits first."""
        if name in self.lazy:
            self.lazy.pop(name)()
        if self.state[name] == "host":
            self._upload(name, self.host[name])
            self.state[name] = "dev"
            self.version[name] += 1
        return self.dev[name]

    def w(self, name):
        """Device tensor about to be overwritten entirely by a kernel."""
        self.lazy.pop(name, None)
        self.state[name] = "dev"
        self.version[name] += 1
        return self.dev[name]

    def h(self, name):
        t = self.d(name)
        if name not in self.host:
            self.host[name] = np.empty(t.numel(), dtype=np.float64)
        if self.kind[name] is not None:
            t = self.mesh_fn().to_host_order(self.kind[name], t)
        self.host[name][...] = t.cpu().numpy()
        self.state[name] = "host"
        return self.host[name]

    def set(self, name, value):
        t = self.w(name)
        if isinstance(value, torch.Tensor):
            if value.numel() != t.numel():
                raise ValueError("%s expects %d values, got %d" % (name, t.numel(), value.numel()))
            self._upload(name, value.reshape(-1))
            return
        v = np.asarray(value, dtype=np.float64)
        if v.ndim == 0:
            t.fill_(float(v))
        else:
            if v.shape != (t.numel(),):
                raise ValueError("%s expects shape (%d,), got %s" % (name, t.numel(), v.shape))
            self._upload(name, v)


def _ptr(t):
    return t.data_ptr()


class Variable:
    def __init__(self, domain=None, terms=None, comm=None, name=None, BC=None, values=None, *args, **kwargs):
        if domain is None:
            raise ValueError("domain must be given")
        object.__setattr__(self, "_s", _Store(domain.device, lambda: domain.device_mesh))
        self._domain = domain
        self._BC = BC
        self._values = values
        self._name = name
        self._dim = domain.dim
        self.backend = domain.backend
        self.float_precision = domain.float_precision
        self.int_precision = domain.int_precision
        nc, nf, nn = int(domain.nbcells), int(domain.nbfaces), int(domain.nbnodes)
        for n in _CELL:
            self._s.add(n, nc, "cell")
        for n in _FACE:
            self._s.add(n, nf, "face")
        for n in _NODE:
            self._s.add(n, nn, "node")
        for n in ("halo", "gradhalocellx", "gradhalocelly", "gradhalocellz", "psihalo", "haloghost"):
            self._s.add(n, 0)
        if terms is not None:
            for t in terms:
                self._s.add(t, nc, "cell")
        self._bc = B.resolve(domain.host_arrays, BC, values)
        self.dirichletfaces = self._bc.dirichletfaces
        self.neumannfaces = self._bc.neumannfaces
        self.neumannNHfaces = np.sort(np.concatenate(
            [f for (t, f) in self._bc.sides.values() if t == "neumannNH"] or [np.zeros(0, np.int32)])
        ).astype(np.int32)
        if self._bc.cell_writes is not None:
            f, v = self._bc.cell_writes
            c = self._s.h("cell")
            c[f] = v
        self._dbc = None

    # ------------------------------------------------------------ storage plumbing
    def add_term(self, name):
        """A cell-sized array (manapy's solvers attach ``convective`` etc. this way)."""
        if name not in self._s.dev:
            self._s.add(name, int(self._domain.nbcells), "cell")

    def __getattr__(self, name):
        s = self.__dict__.get("_s")
        if s is not None and name in s.dev:
            return s.h(name)
        raise AttributeError(name)

    def __setattr__(self, name, value):
        s = self.__dict__.get("_s")
        if s is not None and name in s.dev:
            s.set(name, value)
        else:
            object.__setattr__(self, name, value)

    def dev(self, name):
        """Device tensor of an array (after host edits are uploaded)."""
        return self._s.d(name)

    def dev_out(self, name):
        return self._s.w(name)

    def fetch(self, name="cell", out=None):
        """Copy array ``name`` (manapy's numbering) into the host tensor ``out`` without a
        host synchronisation and without handing authority to the host: the copy is queued
        on the current stream (asynchronous when ``out`` is pinned memory), the device
        array stays the one kernels use.  Returns ``out`` (allocated pinned if None); its
        contents are valid once the stream has reached the copy (``torch.cuda.synchronize``
        or an event).  No counterpart in manapy, whose arrays are host arrays."""
        s = self._s
        t = s.d(name)
        if out is None:
            out = torch.empty(t.numel(), dtype=torch.float64, pin_memory=True)
        if out.numel() != t.numel() or out.dtype != torch.float64:
            raise ValueError("%s needs a float64 tensor of %d values" % (name, t.numel()))
        if s.kind[name] is not None:
            t = s.mesh_fn().to_host_order(s.kind[name], t)
        out.copy_(t, non_blocking=True)
        return out

    def set_lazy(self, name, fn):
        self._s.lazy[name] = fn

    def version(self, name):
        """Counter that changes whenever the array's contents may have changed."""
        s = self._s
        return s.version[name] + (1 << 40 if s.state[name] == "host" else 0)

    def swap_cell(self, t):
        """Install tensor ``t`` (same shape) as the cell array; returns the previous one."""
        s = self._s
        old = s.d("cell")
        s.dev["cell"] = t
        s.state["cell"] = "dev"
        s.version["cell"] += 1
        return old

    @property
    def device_bc(self):
        if self._dbc is None:
            from .device import DeviceBC
            self._dbc = DeviceBC(self._domain.host_arrays, self._bc, self._domain.device,
                                 mesh=self._domain.device_mesh)
        return self._dbc

    @property
    def resolved_bc(self):
        return self._bc

    # ------------------------------------------------------------ manapy methods
    def _m(self):
        return self._domain.device_mesh.struct

    def _stream(self):
        return torch.cuda.current_stream(self._s.device).cuda_stream

    def update_halo_value(self):
        """Single-rank domains have no halo cells (manapy/ast/core.py:415-419)."""
        return None

    def update_ghost_value(self):
        """manapy/ast/core.py:492-497 -> mb_ghost_value."""
        _lib.call("mb_ghost_value", self._m(), self.device_bc.struct, _ptr(self.dev("cell")),
                  _ptr(self._s.d("ghost")), self._stream())
        self._s.state["ghost"] = "dev"

    def interpolate_facetocell(self):
        """manapy/ast/core.py:422-423 -> mb_facetocell."""
        _lib.call("mb_facetocell", self._m(), _ptr(self.dev("face")), _ptr(self.dev_out("cell")),
                  self._stream())

    def interpolate_celltoface(self):
        """manapy/ast/core.py:425-427 (manapy/ast/ast_utils.py:20-36): face = mean of the two
        cells (inner) or of the cell and its ghost (boundary)."""
        A = self._domain.host_arrays
        dm = self._domain.device_mesh
        cid = dm.t["face_cellid"].long().view(-1, 2)
        c = self.dev("cell")
        g = self.dev("ghost")
        out = self.dev("face")
        inner = torch.as_tensor(dm.R.finv[A["innerfaces"]], device=c.device).long()
        bnd = torch.as_tensor(dm.R.finv[A["boundaryfaces"]], device=c.device).long()
        out[inner] = .5 * (c[cid[inner, 0]] + c[cid[inner, 1]])
        out[bnd] = .5 * (c[cid[bnd, 0]] + g[bnd])

    def interpolate_celltonode(self):
        """manapy/ast/core.py:429-439 -> mb_centertovertex (uses the stored ghost values)."""
        _lib.call("mb_centertovertex", self._m(), _ptr(self.dev("cell")), _ptr(self.dev("ghost")),
                  _ptr(self.dev_out("node")), self._stream())

    def compute_cell_gradient(self):
        """manapy/ast/core.py:442-478 -> mb_cell_gradient + mb_barthlimiter."""
        m, st = self._m(), self._stream()
        c, g = _ptr(self.dev("cell")), _ptr(self.dev("ghost"))
        gx, gy, gz = (_ptr(self.dev_out(n)) for n in ("gradcellx", "gradcelly", "gradcellz"))
        _lib.call("mb_cell_gradient", m, c, g, gx, gy, gz, st)
        _lib.call("mb_barthlimiter", m, c, g, gx, gy, gz, _ptr(self.dev_out("psi")), st)

    def compute_face_gradient(self):
        """manapy/ast/core.py:480-490 -> mb_face_gradient."""
        _lib.call("mb_face_gradient", self._m(), self.device_bc.struct, _ptr(self.dev("cell")),
                  _ptr(self.dev("ghost")), _ptr(self.dev("node")), _ptr(self.dev("gradfacex")),
                  _ptr(self.dev("gradfacey")), _ptr(self.dev("gradfacez")), self._stream())

    def norml2(self, exact, order=None):
        """manapy/ast/core.py:500-515."""
        if order is None:
            order = 1
        cell = self.cell
        assert len(cell) == len(exact), "exact solution must have length of cells"
        vol = self._domain.cells.volume
        err = np.fabs(cell - exact) * vol
        ex = np.fabs(np.asarray(exact)) * vol
        return np.linalg.norm(err, ord=order) / np.linalg.norm(ex, ord=order)

    # ------------------------------------------------------------ accessors
    domain = property(lambda self: self._domain)
    dim = property(lambda self: self._dim)
    comm = property(lambda self: self._domain.comm)
    nbfaces = property(lambda self: self._domain.nbfaces)
    nbcells = property(lambda self: self._domain.nbcells)
    nbnodes = property(lambda self: self._domain.nbnodes)
    nbhalos = property(lambda self: 0)
    name = property(lambda self: self._name)

    def __str__(self):
        return ("\n> dim   :: %d\n> total cells  :: %d\n> total nodes  :: %d\n> total faces  :: %d\n"
                % (self.dim, self.nbcells, self.nbnodes, self.nbfaces))
