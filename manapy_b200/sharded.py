"""One advection-diffusion mesh sharded over ranks (one process per GPU).

Each rank builds its shard (``partition.build_shards``: owned cells plus a two-layer
halo), runs the fused CUDA step on it, and refreshes its halo from the owners after
every step (``partition.HaloExchange``: NCCL point-to-point on device buffers, or gloo
through host memory).  dt is the min over ranks of each rank's CFL dt
(``manapy/solvers/advecdiff/system.py:152``: manapy's ``allreduce(MIN)``).  The owned
cells' results are bit-identical to the single-GPU run of the whole mesh.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib, boundary as B, geometry as G, partition as P
from .device import DeviceBC, DeviceMesh

__all__ = ["ShardedAdvectionDiffusion"]


def _p(t):
    return t.data_ptr() if t is not None else None


class ShardedAdvectionDiffusion:
    """``elements``/``vertex``: the whole mesh (every rank reads it, as every manapy rank
    reads the partition it owns); ``velocity``: f(face_centres) -> (u, v, w) face arrays;
    options as ``AdvectionDiffusionSolver`` (Dxx, Dyy, Dzz, order, cfl)."""

    def __init__(self, elements, vertex, dim, BC, values, velocity, Dxx=0., Dyy=0., Dzz=0., order=1, cfl=0.4,
                 group=None, device=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.dim = dim
        self.shard = P.build_shards(elements, vertex, dim, self.world)[self.rank]
        A = G.build(self.shard.elements, self.shard.vertex, dim, halo_rim=True)
        self.A = A
        self.dm = DeviceMesh(A, self.dev)
        self.bc = DeviceBC(A, B.resolve(A, BC, values), self.dev, mesh=self.dm)
        self.params = _lib.MbAdvDiffParams(int(order), int(not (Dxx == Dyy == Dzz == 0)), float(Dxx), float(Dyy),
                                           float(Dzz))
        self.order = int(order)
        nc, nn = self.dm.nbcells, self.dm.nbnodes
        f64 = torch.float64
        self.w = [torch.zeros(nc, dtype=f64, device=self.dev) for _ in range(2)]
        self.cur = 0
        self.cs = torch.empty((4 if dim == 2 else 8) * nc, dtype=f64, device=self.dev)
        self.ns = torch.empty(nn, dtype=f64, device=self.dev)
        self.sign = torch.empty(4 * nc, dtype=f64, device=self.dev)
        self.dt = torch.zeros(1, dtype=f64, device=self.dev)
        # halo indices in the device numbering of the shard
        inv = self.dm.inv["cell"].cpu().numpy()
        self.exchanger = P.HaloExchange(self._to_device_numbering(inv), group, device=self.dev)
        self._set_velocity(velocity, Dxx, Dyy, Dzz, cfl)

    def _staged(self):
        return self.dist.get_backend(self.group) == "gloo"

    def _to_device_numbering(self, inv):
        sh = self.shard
        return P.Shard(rank=sh.rank, cells=sh.cells, owned=sh.owned, nodes=sh.nodes, elements=sh.elements,
                       vertex=sh.vertex, send={q: inv[i] for q, i in sh.send.items()},
                       recv={q: inv[i] for q, i in sh.recv.items()})

    def _stream(self):
        return torch.cuda.current_stream(self.dev).cuda_stream

    def _dev_faces(self, a):
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(self.dev)
        out = torch.empty_like(t)
        self.dm.to_device_order("face", t, out)
        return out

    def _set_velocity(self, velocity, Dxx, Dyy, Dzz, cfl):
        uf, vf, wf = (self._dev_faces(a) for a in velocity(self.A["faces_center"]))
        st = self._stream()
        _lib.call("mb_cell_face_sign", self.dm.struct, _p(uf), _p(vf), _p(wf), _p(self.sign), st)
        cells = [torch.empty(self.dm.nbcells, dtype=torch.float64, device=self.dev) for _ in range(3)]
        for f, c in zip((uf, vf, wf), cells):
            _lib.call("mb_facetocell", self.dm.struct, _p(f), _p(c), st)
        _lib.call("mb_time_step", self.dm.struct, *[_p(c) for c in cells], float(cfl), float(Dxx), float(Dyy),
                  float(Dzz), _p(self.dt), st)
        # global dt: the min over ranks
        d = self.dt.cpu() if self._staged() else self.dt
        self.dist.all_reduce(d, op=self.dist.ReduceOp.MIN, group=self.group)
        if self._staged():
            self.dt.copy_(d)

    def set_cells(self, w_global):
        """The state from a whole-mesh cell array (manapy numbering)."""
        loc = torch.from_numpy(np.ascontiguousarray(np.asarray(w_global)[self.shard.cells], dtype=np.float64))
        self.dm.to_device_order("cell", loc.to(self.dev), self.w[self.cur])

    def step(self):
        x, y = self.w[self.cur], self.w[1 - self.cur]
        _lib.call("mb_advdiff_step", self.dm.struct, self.bc.struct, self.params, _p(x), _p(y), _p(self.sign), None,
                  _p(self.dt), _p(self.cs), _p(self.ns), self._stream())
        self.cur = 1 - self.cur
        self.exchanger.exchange(self.w[self.cur])

    def advance(self, n):
        for _ in range(int(n)):
            self.step()

    def owned_values(self):
        """(global cell ids, values) of the cells this rank owns."""
        host = self.dm.to_host_order("cell", self.w[self.cur]).cpu().numpy()
        return self.shard.cells[self.shard.owned], host[self.shard.owned]

    def gather(self):
        """The whole-mesh cell array on every rank (manapy numbering)."""
        ids, vals = self.owned_values()
        parts = [None] * self.world
        self.dist.all_gather_object(parts, (ids, vals), group=self.group)
        n = sum(len(p[0]) for p in parts)
        out = np.empty(n)
        for ids_, vals_ in parts:
            out[ids_] = vals_
        return out
