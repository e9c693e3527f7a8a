"""``Domain``: manapy's mesh object, built on the host and mirrored on the GPU.

Mirrors ``manapy.ddm.Domain`` (``manapy/ddm/domain.py:36-961``) for a
single-rank mesh: the same constructor options, the same ``cells`` /
``faces`` / ``nodes`` / ``halos`` accessors holding manapy-layout numpy
arrays, and the same face lists.  manapy reads its mesh from per-rank HDF5
files written by ``MeshPartition``; here the mesh is passed in memory
(``mesh=(elements, vertex)`` in manapy's reader layout, see ``meshgen``) or
read from a gmsh file with ``Domain.from_msh``.  The device tables the CUDA
kernels read are built on first use (``domain.device_mesh``).
"""
from __future__ import annotations

import os

import numpy as np

from . import geometry
from .base import Struct, make_get_conf, process_conf

__all__ = ["Domain"]


class _NS:
    """Read-only attribute namespace over a dict of arrays."""

    def __init__(self, **items):
        self.__dict__.update(items)

    def __repr__(self):
        return "<%s>" % ", ".join(sorted(self.__dict__))


class _OneRankComm:
    """Communicator stand-in of a one-rank domain (no halo cells)."""

    def Get_size(self):
        return 1

    def Get_rank(self):
        return 0

    def Barrier(self):
        return None

    def allreduce(self, x, op=None):
        return x


def build_host_mesh(elements, vertex, dim, stencil="shared"):
    """(A, host-built DeviceMesh or None) through the native host builder, bit-identical to
    the Python builder: for triangles every ``geometry.build`` array and device table in one
    C++ pass; for tetrahedra the ``geometry.build`` arrays (the device tables then come from
    ``DeviceMesh``).  A mesh the native builder rejects goes through ``geometry.build``, which
    reports it."""
    from . import native
    try:
        if native.available():
            if dim == 2:
                from .device import DeviceMesh
                dm = DeviceMesh.from_native(elements, vertex, device=None, full=True, stencil=stencil)
                return dm.A, dm
            if dim == 3:
                return native.geometry3d(elements, vertex), None
    except ValueError:
        pass
    return geometry.build(elements, vertex, dim), None


class Domain:
    _parameters = [
        ("backend", "str", "cuda", False, "kernel backend: cuda (sm_100a)"),
        ("multithreading", "str", "single", None, "accepted for compatibility; unused"),
        ("signature", "bool", True, False, "accepted for compatibility; unused"),
        ("cache", "bool", False, False, "accepted for compatibility; unused"),
        ("float_precision", "str", "double", None, "precision of the float arrays"),
        ("int_precision", "str", "signed", None, "precision of the integer arrays"),
        ("device", "str", "cuda", None, "torch device holding the mesh tables"),
        ("mesh_cache", "str", None, None, "directory of the persistent mesh cache (geometry and device tables "
                                           "stored once per mesh; also MANAPY_B200_MESH_CACHE); no counterpart "
                                           "in manapy"),
        ("check_tables", "bool", False, False, "check every index table of the mesh on the device once, when "
                                                "it is first used (mb_check_tables); no counterpart in manapy"),
        ("stencil", "str", "shared", None, "layout of the least-squares stencil: 'shared' (neighbours shared by "
                                           "the cells of one warp read in one slot; fastest) or 'manapy' (each "
                                           "cell's neighbours in manapy's order, so results do not depend on the "
                                           "numbering of other cells, e.g. when the mesh is sharded); no "
                                           "counterpart in manapy"),
    ]

    @classmethod
    def process_conf(cls, conf, kwargs):
        return process_conf(cls._parameters, conf, kwargs)

    def __init__(self, dim=None, comm=None, conf=None, mesh=None, **kwargs):
        if conf is None:
            conf = Struct()
        self.conf = self.process_conf(conf, kwargs)
        get = make_get_conf(self.conf, kwargs)
        if dim is None:
            raise ValueError("dim must be given")
        if int(dim) not in (2, 3):
            raise ValueError("dim must be 2 or 3")
        if get("float_precision") == "single":
            raise ValueError("float_precision='single' is not supported by the FP64 CUDA path; "
                             "use the FP32-compensated solvers instead")
        self.float_precision = "f8"
        self.int_precision = "i4" if get("int_precision") == "signed" else "u4"
        self.signature = get("signature")
        self.device = get("device")
        self.stencil = get("stencil")
        self.check_tables = bool(get("check_tables"))
        from .device import STENCILS
        if self.stencil not in STENCILS:
            raise ValueError("stencil must be one of %s" % (STENCILS,))
        if mesh is None:
            mesh = getattr(conf, "mesh", None)
        if mesh is None:
            raise ValueError("no mesh given: pass mesh=(elements, vertex) or use Domain.from_msh(path)")
        elements, vertex = mesh
        self._comm = comm if comm is not None else _OneRankComm()
        self._dim = np.int32(dim)
        cache_dir = get("mesh_cache") or os.environ.get("MANAPY_B200_MESH_CACHE")
        self._host_dm = None
        self.mesh_cache_hit = False
        if cache_dir:
            from . import meshcache
            self._A, self._host_dm, self.mesh_cache_hit = meshcache.load_or_build(elements, vertex, int(dim),
                                                                                  cache_dir, stencil=self.stencil)
        else:
            self._A, self._host_dm = build_host_mesh(elements, vertex, int(dim), self.stencil)
        if len(self._A["unmatched_boundary_faces"]):
            raise ValueError("%d boundary faces match no boundary side (their vertices carry "
                             "incompatible tags)" % len(self._A["unmatched_boundary_faces"]))
        self._build_views()
        from .backend import CUDABackend
        self.backend = CUDABackend(self)
        self._dmesh = None

    @classmethod
    def from_msh(cls, path, dim, conf=None, **kwargs):
        """Build from a gmsh 4.1 ASCII file (boundary vertex tags from its physical groups)."""
        from .gmsh import read_msh
        return cls(dim=dim, conf=conf, mesh=read_msh(path, dim), **kwargs)

    @classmethod
    def from_hdf5(cls, mesh_dir, dim, conf=None, **kwargs):
        """Build from a manapy mesh directory ``meshes<P>PROC`` (``mesh<r>.hdf5``, written by
        manapy's partitioner, ``manapy/partitions/meshpartitioning.py:238-275``; read as
        ``manapy/ddm/pure_ddm.py:13-102`` does, without h5py): one rank's file, or the
        rank files reassembled into the whole mesh."""
        from .hdf5 import read_mesh_dir
        return cls(dim=dim, conf=conf, mesh=read_mesh_dir(mesh_dir), **kwargs)

    # ------------------------------------------------------------------ views
    def _build_views(self):
        A = self._A
        P = geometry.padded_from_csr
        nc, nf, nn = A["nbcells"], A["nbfaces"], A["nbnodes"]
        self._cells = _NS(
            nodeid=A["cells_nodeid"], faceid=A["cells_faceid"], cellfid=A["cells_cellfid"],
            center=A["cells_center"], volume=A["cells_volume"],
            cellnid=P(A["cellnid_ptr"], A["cellnid_idx"]),
            ghostnid=P(A["ghostnid_ptr"], A["ghostnid_idx"]),
            nf=A.get("cells_nf", np.zeros((nc, 4, 3))),
            halonid=np.zeros((nc, 2), np.int32), haloghostnid=np.zeros((nc, 2), np.int32),
            haloghostcenter=np.zeros((0, 3)), periodicnid=np.zeros((nc, 2), np.int32),
            periodicfid=np.zeros(nc, np.int32), shift=np.zeros((nc, 3)),
            loctoglob=np.arange(nc, dtype=np.int32), globtoloc=np.arange(nc, dtype=np.int32),
            tc=np.arange(nc, dtype=np.int32), nbcells=nc)
        faces = dict(nodeid=A["faces_nodeid"], cellid=A["faces_cellid"], name=A["faces_name"],
                     oldname=A["faces_name"], normal=A["faces_normal"], mesure=A["faces_mesure"],
                     center=A["faces_center"], ghostcenter=A["faces_ghostcenter"],
                     airDiamond=A["faces_airDiamond"], f_1=A["faces_f_1"], f_2=A["faces_f_2"],
                     f_3=A["faces_f_3"], f_4=A["faces_f_4"], param1=A["faces_param1"],
                     param2=A["faces_param2"], param3=A["faces_param3"],
                     param4=A.get("faces_param4", np.zeros(nf)), dist_ortho=A["faces_dist_ortho"],
                     halofid=np.zeros(nf, np.int32), nbfaces=nf)
        self._faces = _NS(**faces)
        self._nodes = _NS(
            vertex=A["nodes_vertex"], name=A["nodes_name"], oldname=A["nodes_name"].copy(),
            cellid=P(A["n2c_ptr"], A["n2c_idx"]), ghostid=P(A["n2g_ptr"], A["n2g_idx"]),
            R_x=A["nodes_R_x"], R_y=A["nodes_R_y"], R_z=A["nodes_R_z"],
            lambda_x=A["nodes_lambda_x"], lambda_y=A["nodes_lambda_y"], lambda_z=A["nodes_lambda_z"],
            number=A["nodes_number"], halonid=np.zeros((nn, 2), np.int32),
            periodicid=np.zeros((nn, 2), np.int32), haloghostid=np.zeros((nn, 2), np.int32),
            loctoglob=np.arange(nn, dtype=np.int32), nbnodes=nn)
        self._halos = _NS(centvol=np.zeros((2, 2)), halosint=np.zeros((2, 2), np.int32),
                          halosext=np.zeros((2, 2), np.int32), sizehaloghost=0,
                          indsend=np.zeros(1, np.int32), scount=np.zeros(1, np.uint32),
                          rcount=np.zeros(1, np.uint32), comm_ptr=self._comm)
        self._BCs = {"in": ["neumann", 1], "out": ["neumann", 2], "upper": ["neumann", 3],
                     "bottom": ["neumann", 4]}
        if self._dim == 3:
            self._BCs.update({"front": ["neumann", 5], "back": ["neumann", 6]})

    # ------------------------------------------------------------------ device
    @property
    def device_mesh(self):
        """The device tables (``mb_mesh``), built on first use."""
        if self._dmesh is None:
            if self._host_dm is not None:          # tables from the mesh cache
                self._dmesh, self._host_dm = self._host_dm.upload(self.device), None
            else:
                from .device import DeviceMesh
                self._dmesh = DeviceMesh(self._A, self.device, stencil=self.stencil)
            if self.check_tables:
                self._dmesh.check_tables()
        return self._dmesh

    @property
    def host_arrays(self):
        return self._A

    # ------------------------------------------------------------------ accessors
    cells = property(lambda self: self._cells)
    faces = property(lambda self: self._faces)
    nodes = property(lambda self: self._nodes)
    halos = property(lambda self: self._halos)
    dim = property(lambda self: self._dim)
    comm = property(lambda self: self._comm)
    nbcells = property(lambda self: np.int32(self._A["nbcells"]))
    nbfaces = property(lambda self: np.int32(self._A["nbfaces"]))
    nbnodes = property(lambda self: np.int32(self._A["nbnodes"]))
    nbhalos = property(lambda self: 0)
    innerfaces = property(lambda self: self._A["innerfaces"])
    infaces = property(lambda self: self._A["infaces"])
    outfaces = property(lambda self: self._A["outfaces"])
    upperfaces = property(lambda self: self._A["upperfaces"])
    bottomfaces = property(lambda self: self._A["bottomfaces"])
    frontfaces = property(lambda self: self._A.get("frontfaces", np.zeros(0, np.int32)))
    backfaces = property(lambda self: self._A.get("backfaces", np.zeros(0, np.int32)))
    halofaces = property(lambda self: np.zeros(0, np.int32))
    boundaryfaces = property(lambda self: self._A["boundaryfaces"])
    periodicboundaryfaces = property(lambda self: np.zeros(0, np.int32))
    halonodes = property(lambda self: np.zeros(0, np.int32))

    @property
    def bounds(self):
        v = self._A["nodes_vertex"]
        return np.array([[v[:, k].min(), v[:, k].max()] for k in range(int(self._dim))])

    # ------------------------------------------------------------------ output
    def _device_to_pinned(self, on, values):
        """Start the copies of device-resident values (``Variable`` objects or CUDA tensors
        in manapy's numbering) into pinned host buffers; returns (host arrays or pinned
        tensors, event after which they are valid, or None).  Each Variable's array is
        gathered into manapy's numbering on the current stream (ordered before any later
        step that overwrites it); the device-to-host copies run on a side stream."""
        import torch
        from .variable import Variable
        if not any(isinstance(v, Variable) or (isinstance(v, torch.Tensor) and v.is_cuda) for v in values):
            return [v.detach().cpu().numpy() if hasattr(v, "detach") else np.asarray(v) for v in values], None
        if getattr(self, "_io_stream", None) is None:
            self._io_stream = torch.cuda.Stream(device=torch.device(self.device))
        cur = torch.cuda.current_stream(torch.device(self.device))
        staged = []
        for v in values:
            if isinstance(v, Variable):
                t = v.dev(on)
                kind = v._s.kind[on]
                t = self.device_mesh.to_host_order(kind, t) if kind is not None else t
                staged.append(t.clone() if t is v.dev(on) else t)
            elif isinstance(v, torch.Tensor) and v.is_cuda:
                staged.append(v.detach().to(torch.float64).clone())
            else:
                staged.append(np.asarray(v))
        io = self._io_stream
        io.wait_stream(cur)
        out = []
        with torch.cuda.stream(io):
            for t in staged:
                if isinstance(t, np.ndarray):
                    out.append(t)
                    continue
                h = torch.empty(t.numel(), dtype=torch.float64, pin_memory=True)
                h.copy_(t, non_blocking=True)
                t.record_stream(io)         # the caching allocator keeps it until the copy ran
                out.append(h)
            ev = torch.cuda.Event()
            ev.record(io)
        return out, ev

    def _save(self, on, dt, time, niter, miter, variables, values, file_format, path, asynchronous=False):
        from . import vtu
        if values is None:
            raise ValueError("value must be given")
        if file_format != "vtu":
            raise ValueError("only the vtu format is written")
        n = int(self.nbcells if on == "cell" else self.nbnodes)
        vals, ev = self._device_to_pinned(on, values)
        k = 3 if self._dim == 2 else 4
        cells = self._A["cells_nodeid"][:, :k]
        points = self._A["nodes_vertex"][:, :3]
        rank = self._comm.Get_rank()

        def write():
            if ev is not None:
                ev.synchronize()
            arrs = [np.asarray(v.numpy() if hasattr(v, "numpy") else v, dtype=np.float64) for v in vals]
            assert len(arrs[0]) == n, "value size != number of %ss" % on
            data = {variables[j]: arrs[j] for j in range(len(arrs))}
            print(" **************************** Computing ****************************")
            print("$$$$$$$$$$$$$$$$$$$$$$$$$$$$ Saving Results $$$$$$$$$$$$$$$$$$$$$$$$$$$$$$$$$")
            print("Iteration = ", niter, "time = ", time, "time step = ", dt)
            print("max" + variables[0] + " =", float(np.max(arrs[0])))
            piece = "visu%d-%d.vtu" % (rank, miter)
            vtu.write_vtu(os.path.join(path, piece), points, cells,
                          cell_data=data if on == "cell" else None, point_data=data if on == "node" else None)
            vtu.write_pvtu(os.path.join(path, "visu%d.pvtu" % miter), [piece], list(variables), on=on)

        if not asynchronous:
            write()
            return None
        if getattr(self, "_writer", None) is None:
            import concurrent.futures as cf
            self._writer = cf.ThreadPoolExecutor(max_workers=1)
            self._pending = []
        fut = self._writer.submit(write)
        self._pending.append(fut)
        return fut

    def wait_saves(self):
        """Block until every asynchronous save has been written (re-raises a writer error)."""
        for f in getattr(self, "_pending", []):
            f.result()
        self._pending = []

    def save_on_cell_multi(self, dt=0, time=0, niter=0, miter=0, variables=None, values=None, file_format="vtu",
                           path="results", asynchronous=False):
        """Cell fields to ``results/visu<rank>-<miter>.vtu`` + ``visu<miter>.pvtu``
        (``manapy/ddm/domain.py:784-849``).  ``values``: host arrays as in manapy, or
        device-resident ``Variable`` objects / CUDA tensors (manapy numbering), which are
        copied to pinned host memory off the compute stream.  ``asynchronous=True`` (no
        counterpart in manapy) returns at once with a future; the file is written by a
        background thread once the copies have run, while later steps proceed
        (``wait_saves()`` joins)."""
        return self._save("cell", dt, time, niter, miter, variables, values, file_format, path, asynchronous)

    def save_on_node_multi(self, dt=0, time=0, niter=0, miter=0, variables=None, values=None, file_format="vtu",
                           path="results", asynchronous=False):
        """Node fields, as ``save_on_cell_multi`` (``manapy/ddm/domain.py:735-782``)."""
        return self._save("node", dt, time, niter, miter, variables, values, file_format, path, asynchronous)

    def __str__(self):
        return ("\n> dim   :: %d\n> total cells  :: %d\n> total nodes  :: %d\n> total faces  :: %d\n"
                % (self.dim, self.nbcells, self.nbnodes, self.nbfaces))
