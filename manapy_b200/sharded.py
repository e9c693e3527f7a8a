"""One mesh sharded over ranks (one process per GPU): advection-diffusion and shallow water.

Each rank builds its shard (``partition.build_shards``: owned cells plus a two-layer
halo), runs the fused CUDA step on it, and refreshes its halo from the owners after
every step (``partition.HaloExchange``: all fields of all peers packed by one launch,
NCCL point-to-point on device buffers, or gloo through host memory).  dt is the min over
ranks of each rank's CFL dt (``manapy/solvers/advecdiff/system.py:152`` and
``manapy/solvers/shallowater/system.py:188``: manapy's ``allreduce(MIN)``).  The owned
cells' results are bit-identical to the single-GPU run of the whole mesh.

Both solvers overlap the exchange with the step: each shard numbers the cells its peers
read first, computes them (``mb_advdiff_step_split`` / ``mb_sw_step_split`` part 0), posts
the exchange, and computes the other cells (part 1) while the messages travel; the halo is
written after both.

Before each step every rank checks the run's failure record (``partition.FailureMonitor``):
a rank that failed between steps has posted it, and the others raise ``RankFailure``
instead of entering an exchange that would wait for it.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib, boundary as B, geometry as G, partition as P
from .device import DeviceBC, DeviceMesh

__all__ = ["ShardedAdvectionDiffusion", "ShardedShallowWater"]


def _p(t):
    return t.data_ptr() if t is not None else None


class _Sharded:
    """Shard, device mesh, halo exchange and failure monitor of one rank."""

    def __init__(self, elements, vertex, dim, group, device, store, extra_cells=None, sync_every=0, check_every=1,
                 A=None, send_first=False):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.dim = dim
        self.shard = P.build_shards(elements, vertex, dim, self.world, A=A, extra_cells=extra_cells)[self.rank]
        A = G.build(self.shard.elements, self.shard.vertex, dim, halo_rim=True)
        self.A = A
        # manapy's stencil order: every cell's sums formed as in the single-domain run;
        # with send_first the cells peers read are numbered first
        first = None
        if send_first:
            first = np.zeros(len(self.shard.cells), dtype=bool)
            for idx in self.shard.send.values():
                first[np.asarray(idx, dtype=np.int64)] = True
        self.dm = DeviceMesh(A, self.dev, stencil="manapy", first_cells=first)
        inv = self.dm.inv["cell"].cpu().numpy()
        self.exchanger = P.HaloExchange(self._to_device_numbering(inv), group, device=self.dev)
        self.monitor = P.FailureMonitor(self.rank, store, world=self.world)
        # heartbeat every sync_every steps; otherwise a failure-record lookup every check_every
        # steps (0: none; the process group's timeout still ends a run whose peer died)
        self.sync_every = int(sync_every)
        self.check_every = int(check_every)
        self.steps_done = 0

    def _before_step(self):
        k = self.steps_done
        if self.sync_every and k % self.sync_every == 0:
            self.monitor.sync(k)
        elif self.check_every and k % self.check_every == 0:
            self.monitor.check()
        self.steps_done += 1

    def _staged(self):
        return self.dist.get_backend(self.group) == "gloo"

    def _to_device_numbering(self, inv):
        sh = self.shard
        return P.Shard(rank=sh.rank, cells=sh.cells, owned=sh.owned, nodes=sh.nodes, elements=sh.elements,
                       vertex=sh.vertex, send={q: inv[i] for q, i in sh.send.items()},
                       recv={q: inv[i] for q, i in sh.recv.items()})

    def _stream(self):
        return torch.cuda.current_stream(self.dev).cuda_stream

    def _all_min(self, t):
        d = t.cpu() if self._staged() else t
        self.dist.all_reduce(d, op=self.dist.ReduceOp.MIN, group=self.group)
        if self._staged():
            t.copy_(d)

    def _local(self, a_global):
        loc = torch.from_numpy(np.ascontiguousarray(np.asarray(a_global)[self.shard.cells], dtype=np.float64))
        out = torch.empty(len(loc), dtype=torch.float64, device=self.dev)
        self.dm.to_device_order("cell", loc.to(self.dev), out)
        return out

    def _owned(self, t):
        host = self.dm.to_host_order("cell", t).cpu().numpy()
        return self.shard.cells[self.shard.owned], host[self.shard.owned]

    def _gather(self, t):
        ids, vals = self._owned(t)
        parts = [None] * self.world
        self.dist.all_gather_object(parts, (ids, vals), group=self.group)
        n = sum(len(p[0]) for p in parts)
        out = np.empty(n)
        for ids_, vals_ in parts:
            out[ids_] = vals_
        return out

    def advance(self, n):
        for _ in range(int(n)):
            self.step()


class ShardedAdvectionDiffusion(_Sharded):
    """``elements``/``vertex``: the whole mesh (every rank reads it, as every manapy rank
    reads the partition it owns); ``velocity``: f(face_centres) -> (u, v, w) face arrays;
    options as ``AdvectionDiffusionSolver`` (Dxx, Dyy, Dzz, order, cfl)."""

    def __init__(self, elements, vertex, dim, BC, values, velocity, Dxx=0., Dyy=0., Dzz=0., order=1, cfl=0.4,
                 group=None, device=None, store=None, sync_every=0, check_every=1, A=None, overlap=True):
        super().__init__(elements, vertex, dim, group, device, store, sync_every=sync_every, check_every=check_every,
                         A=A, send_first=overlap)
        self.overlap = bool(overlap)
        A = self.A
        self.bc = DeviceBC(A, B.resolve(A, BC, values), self.dev, mesh=self.dm)
        self.params = _lib.MbAdvDiffParams(int(order), int(not (Dxx == Dyy == Dzz == 0)), float(Dxx), float(Dyy),
                                           float(Dzz))
        self.order = int(order)
        nc, nn = self.dm.nbcells, self.dm.nbnodes
        f64 = torch.float64
        self.w = [torch.zeros(nc, dtype=f64, device=self.dev) for _ in range(2)]
        self.cur = 0
        # cell scratch of the fused step: 4 nbcells (2D) or 8 nbcells (3D) doubles
        self.cs = torch.empty((4 if dim == 2 else 8) * nc, dtype=f64, device=self.dev)
        self.ns = torch.empty(nn, dtype=f64, device=self.dev)
        self.sign = torch.empty(4 * nc, dtype=f64, device=self.dev)
        self.dt = torch.zeros(1, dtype=f64, device=self.dev)
        self._set_velocity(velocity, Dxx, Dyy, Dzz, cfl)

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
        self._all_min(self.dt)      # steady velocity: the global dt once

    def set_cells(self, w_global):
        """The state from a whole-mesh cell array (manapy numbering)."""
        self.w[self.cur].copy_(self._local(w_global))

    def step(self):
        self._before_step()
        with self.monitor.guard():
            x, y = self.w[self.cur], self.w[1 - self.cur]
            args = (self.dm.struct, self.bc.struct, self.params, _p(x), _p(y), _p(self.sign), None, _p(self.dt),
                    _p(self.cs), _p(self.ns))
            if self.overlap:
                # the cells peers read, the exchange posted, the other cells while it travels
                _lib.call("mb_advdiff_step_split", *args, 0, self.dm.nfirst, self._stream())
                pending = self.exchanger.start(y)
                _lib.call("mb_advdiff_step_split", *args, 1, self.dm.nfirst, self._stream())
                self.exchanger.finish(pending)
            else:
                _lib.call("mb_advdiff_step", *args, self._stream())
                self.exchanger.exchange(y)
            self.cur = 1 - self.cur

    def owned_values(self):
        """(global cell ids, values) of the cells this rank owns."""
        return self._owned(self.w[self.cur])

    def gather(self):
        """The whole-mesh cell array on every rank (manapy numbering)."""
        return self._gather(self.w[self.cur])


class ShardedShallowWater(_Sharded):
    """First-order shallow water (SRNH flux, bathymetry source) on one sharded triangle
    mesh, as ``ShallowWaterSolver`` with its default Neumann walls (or ``walls=
    "reflective"``).  Per step: dt of the current state over the rank's cells (owned and
    halo, whose values are the owners' after the last exchange) with the fused step's
    formula, min over ranks; the fused step; the exchange of h, hu, hv, hc."""

    def __init__(self, elements, vertex, cfl=0.8, grav=9.81, walls="neumann", group=None, device=None, store=None,
                 sync_every=0, check_every=1, A=None, overlap=True):
        # every shard holds the mesh's last cell: the source term reads it for cellfid padding
        super().__init__(elements, vertex, 2, group, device, store, extra_cells=[len(elements) - 1],
                         sync_every=sync_every, check_every=check_every, A=A, send_first=overlap)
        self.overlap = bool(overlap)
        if walls not in _lib.WALLS:
            raise ValueError("walls must be 'neumann' or 'reflective'")
        self.walls = _lib.WALLS[walls]
        self.cfl, self.grav = float(cfl), float(grav)
        nc, nf = self.dm.nbcells, self.dm.nbfaces
        f64 = torch.float64
        self.q = [[torch.zeros(nc, dtype=f64, device=self.dev) for _ in range(4)] for _ in range(2)]
        self.Z = torch.zeros(nc, dtype=f64, device=self.dev)
        self.cur = 0
        self.ff = torch.empty(4 * nf, dtype=f64, device=self.dev)
        self.dt = torch.zeros(1, dtype=f64, device=self.dev)

    def set_state(self, h, hu, hv, hc, Z):
        """The state from whole-mesh cell arrays (manapy numbering)."""
        for t, a in zip(self.q[self.cur], (h, hu, hv, hc)):
            t.copy_(self._local(a))
        self.Z.copy_(self._local(Z))

    def step(self):
        self._before_step()
        with self.monitor.guard():
            qi, qo = self.q[self.cur], self.q[1 - self.cur]
            st = self._stream()
            _lib.call("mb_sw_dt", self.dm.struct, _p(qi[0]), _p(qi[1]), _p(qi[2]), self.cfl, self.grav, _p(self.dt),
                      st)
            self._all_min(self.dt)
            args = (self.dm.struct, _lib.p5([_p(t) for t in qi] + [_p(self.Z)]),
                    _lib.p5([_p(t) for t in qo] + [_p(self.Z)]), self.cfl, self.grav, 1, self.walls, None,
                    _p(self.ff), _p(self.dt), None)
            if self.overlap:
                # the cells peers read, the exchange posted, the other cells while it travels
                _lib.call("mb_sw_step_split", *args, 0, self.dm.nfirst, st)
                pending = self.exchanger.start(qo)
                _lib.call("mb_sw_step_split", *args, 1, self.dm.nfirst, st)
                self.exchanger.finish(pending)
            else:
                _lib.call("mb_sw_step_ex", *args, st)
                self.exchanger.exchange(qo)
            self.cur = 1 - self.cur

    def gather(self):
        """[h, hu, hv] whole-mesh cell arrays on every rank (manapy numbering)."""
        return [self._gather(t) for t in self.q[self.cur][:3]]
