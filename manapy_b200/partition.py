"""Spatial sharding of one mesh over ranks (manapy's MPI domain decomposition, rebuilt).

manapy partitions the dual graph with METIS and exchanges a one-layer vertex halo
before each gradient, limiter and flux evaluation (``manapy/ast/core.py:415-478``,
``manapy/comms/communication.py:86-145``) plus a dt min-allreduce per step
(``manapy/solvers/advecdiff/system.py:152``).  Here:

* each rank owns a contiguous range of the cells' Morton order (equal counts);
* its submesh is the owned cells plus every cell within two vertex-adjacency
  layers of them (the halo), cells and nodes kept in ascending global order;
* one exchange per step refreshes the halo values from their owners; the halo is
  deep enough that an owned cell's update reads only halo cells whose own
  gradient, limiter and vertex values are complete, so nothing else is
  exchanged (manapy exchanges four more times per step for order 2);
* dt is the min over ranks of the min over each rank's cells.

Because the submesh keeps global order, every per-cell list of an owned cell has
the same members in the same order as on the whole mesh and every number is
computed by the same operations: an owned cell's result is bit-identical to the
single-domain result.  The cut faces at the outer edge of the halo are halo faces
(name 10) with no ghost rule; only outer-halo cells touch them.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import reorder

__all__ = ["partition_cells", "Shard", "build_shards", "HaloExchange", "RankFailure", "FailureMonitor"]


def partition_cells(center, dim, nparts):
    """Owner rank of every cell: equal contiguous ranges of the Morton order."""
    order = reorder.morton_cells(center, dim)
    nc = len(order)
    bounds = np.round(np.linspace(0, nc, nparts + 1)).astype(np.int64)
    owner = np.empty(nc, dtype=np.int32)
    for r in range(nparts):
        owner[order[bounds[r]:bounds[r + 1]]] = r
    return owner


def _neighbours(cellnid_ptr, cellnid_idx, mask):
    rows = np.nonzero(mask)[0]
    cnt = cellnid_ptr[rows + 1] - cellnid_ptr[rows]
    starts = np.repeat(cellnid_ptr[rows], cnt)
    offs = np.arange(int(cnt.sum())) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    out = np.zeros_like(mask)
    out[cellnid_idx[starts + offs]] = True
    return out


@dataclasses.dataclass
class Shard:
    rank: int
    cells: np.ndarray      # global ids of the submesh cells, ascending
    owned: np.ndarray      # bool per submesh cell
    nodes: np.ndarray      # global ids of the submesh nodes, ascending
    elements: np.ndarray   # submesh connectivity (local node ids, count column)
    vertex: np.ndarray     # submesh vertices (global tags kept)
    send: dict             # peer rank -> local indices of owned cells the peer holds as halo
    recv: dict             # peer rank -> local indices of halo cells owned by the peer

    @property
    def nowned(self):
        return int(self.owned.sum())


def build_shards(elements, vertex, dim, nparts, A=None, layers=2, extra_cells=None):
    """The ``nparts`` shards of a mesh.  ``A``: its ``geometry.build`` arrays (built if
    not given; only the cell centres and vertex-neighbour lists are read).  ``extra_cells``:
    global cells every shard also holds (as halo unless it owns them) -- the shallow-water
    source term reads the last cell of the mesh for the padding of ``cells.cellfid``
    (``manapy/solvers/shallowater/fvm_utils.py:95-96``, a negative-index wrap), so those
    shards hold global cell ``nc - 1``, which stays their last cell because shards keep
    global order."""
    from . import geometry
    if A is None:
        A = geometry.build(elements, vertex, dim)
    nc = int(A["nbcells"])
    k = int(elements[0, -1])
    owner = partition_cells(A["cells_center"], dim, nparts)
    shards = []
    for r in range(nparts):
        own = owner == r
        cur = own.copy()
        for _ in range(layers):
            cur |= _neighbours(A["cellnid_ptr"], A["cellnid_idx"], cur)
        if extra_cells is not None:
            cur[np.asarray(extra_cells, dtype=np.int64)] = True
        cells = np.nonzero(cur)[0]
        nodes = np.unique(elements[cells, :k])
        local = np.searchsorted(nodes, elements[cells, :k]).astype(np.int32)
        el = np.empty((len(cells), k + 1), dtype=np.int32)
        el[:, :k] = local
        el[:, k] = k
        shards.append(Shard(rank=r, cells=cells, owned=own[cells], nodes=nodes, elements=el,
                            vertex=np.ascontiguousarray(vertex[nodes]), send={}, recv={}))
    # exchange plan: rank r receives its halo cells from their owners, ordered by global id
    for sh in shards:
        halo = sh.cells[~sh.owned]
        for q in np.unique(owner[halo]):
            g = halo[owner[halo] == q]
            sh.recv[int(q)] = np.searchsorted(sh.cells, g).astype(np.int64)
            shards[q].send[sh.rank] = np.searchsorted(shards[q].cells, g).astype(np.int64)
    assert all(len(s.cells) for s in shards) and nc == sum(s.nowned for s in shards)
    return shards


class HaloExchange:
    """Refresh the halo entries of per-rank cell arrays from their owners.

    Every peer's send list (and receive list) is concatenated, peers in ascending rank
    order; an exchange packs all fields for all peers with one launch
    (``mb_halo_pack``: buffer [entry][field], each peer's entries one contiguous
    message), sends and receives one message per peer
    (``torch.distributed.batch_isend_irecv``), and scatters the received buffer with one
    launch (``mb_halo_unpack``).  With the NCCL backend the buffers stay on the device;
    with gloo they are staged through host memory.  CPU fields (the oracle-driven tests)
    are packed with index operations on the host.
    """

    def __init__(self, shard, group=None, device=None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = shard.rank
        self.device = device
        self.peers = sorted(set(shard.send) | set(shard.recv))
        empty = np.zeros(0, np.int64)
        send = [np.asarray(shard.send.get(q, empty), np.int64) for q in self.peers]
        recv = [np.asarray(shard.recv.get(q, empty), np.int64) for q in self.peers]
        self.send_n = [len(a) for a in send]
        self.recv_n = [len(a) for a in recv]
        to = (lambda a: torch.from_numpy(a).to(device)) if device is not None else torch.from_numpy
        self.send_idx = to(np.concatenate(send) if send else empty)
        self.recv_idx = to(np.concatenate(recv) if recv else empty)
        backend = dist.get_backend(group)
        self.stage = backend == "gloo"

    def exchange(self, fields):
        """In place: fields[halo] = owners' values.  ``fields``: one 1-D float64 tensor over
        the submesh cells, or a list of them (exchanged together)."""
        return self.finish(self.start(fields))

    def start(self, fields):
        """First half of ``exchange``: pack the send entries (ordered on the current stream
        after what it has queued) and post the sends and receives.  Work queued on the
        stream before ``finish`` runs while the messages travel; it must not write the send
        entries.  Returns the handle ``finish`` takes."""
        import torch
        from . import _lib
        dist = self.dist
        single = isinstance(fields, torch.Tensor)
        fl = [fields] if single else list(fields)
        nf = len(fl)
        ns, nr = int(sum(self.send_n)), int(sum(self.recv_n))
        dev = fl[0].device
        cuda = dev.type == "cuda"
        st = torch.cuda.current_stream(dev).cuda_stream if cuda else None
        ptrs = _lib.ptrs([t.data_ptr() for t in fl]) if cuda else None
        if cuda:
            sbuf = torch.empty(ns * nf, dtype=torch.float64, device=dev)
            _lib.call("mb_halo_pack", ptrs, nf, self.send_idx.data_ptr(), ns, sbuf.data_ptr(), st)
        else:
            sbuf = torch.stack([f.index_select(0, self.send_idx) for f in fl], dim=1).reshape(-1)
        rbuf = torch.empty(nr * nf, dtype=torch.float64, device=dev)
        if self.stage and cuda:
            sbuf, rdev, rbuf = sbuf.cpu(), rbuf, rbuf.cpu()
        ops = []
        so = ro = 0
        for q, n_s, n_r in zip(self.peers, self.send_n, self.recv_n):
            if n_s:
                ops.append(dist.P2POp(dist.isend, sbuf[so * nf:(so + n_s) * nf], q, group=self.group))
            if n_r:
                ops.append(dist.P2POp(dist.irecv, rbuf[ro * nf:(ro + n_r) * nf], q, group=self.group))
            so += n_s
            ro += n_r
        works = dist.batch_isend_irecv(ops) if ops else []
        return (fields, fl, nf, nr, cuda, st, ptrs, sbuf, rbuf, rdev if (self.stage and cuda) else None, works)

    def finish(self, handle):
        """Second half of ``exchange``: wait for the messages (NCCL: the current stream
        waits; gloo: the host) and scatter the received values into the halo entries."""
        from . import _lib
        fields, fl, nf, nr, cuda, st, ptrs, sbuf, rbuf, rdev, works = handle
        for w in works:
            w.wait()
        if cuda:
            if rdev is not None:
                rdev.copy_(rbuf)
                rbuf = rdev
            _lib.call("mb_halo_unpack", ptrs, nf, self.recv_idx.data_ptr(), nr, rbuf.data_ptr(), st)
        else:
            r = rbuf.view(nr, nf)
            for j, f in enumerate(fl):
                f.index_copy_(0, self.recv_idx, r[:, j].contiguous())
        return fields


class RankFailure(RuntimeError):
    """Another rank of the sharded run failed (reported through the store)."""


class FailureMonitor:
    """Host-side failure detection of a sharded run (no counterpart in manapy, whose MPI
    ranks abort together).  A rank that fails inside ``guard()`` posts an abort record in
    the process group's key-value store before it leaves; every rank calls ``check()``
    before it launches a step, so the others raise ``RankFailure`` instead of waiting in
    their next exchange.  A rank that dies without posting (killed) is caught by the
    process group's timeout in the next exchange, which raises on the survivors.
    No GPU fault is involved: ranks leave only between steps."""

    KEY = "manapy_b200/abort"
    STEP = "manapy_b200/step/%d"

    def __init__(self, rank, store=None, world=None, timeout=10.0):
        import torch.distributed as dist
        self.rank = rank
        if store is None:
            store = dist.distributed_c10d._get_default_store()
        self.store = store
        self.world = dist.get_world_size() if world is None else int(world)
        self.timeout = float(timeout)

    def check(self):
        """Raise RankFailure if a rank has posted a failure (one store lookup, no wait)."""
        if self.store.check([self.KEY]):
            raise RankFailure(self.store.get(self.KEY).decode())

    def sync(self, step):
        """Heartbeat between steps: post this rank's arrival at ``step`` and wait until every
        rank has arrived; raise RankFailure as soon as a failure is posted, or when a rank has
        not arrived within ``timeout`` seconds (it died without posting)."""
        import time
        key = self.STEP % step
        self.store.add(key, 1)
        deadline = time.monotonic() + self.timeout
        wait = 1e-4
        while True:
            self.check()
            if self.store.add(key, 0) >= self.world:
                break
            if time.monotonic() > deadline:
                raise RankFailure("rank(s) did not reach step %d within %.1f s" % (step, self.timeout))
            time.sleep(wait)
            wait = min(2 * wait, 0.01)
        if step >= 2 and self.rank == 0:
            try:
                self.store.delete_key(self.STEP % (step - 2))   # every rank is past it
            except Exception:
                pass

    def signal(self, reason):
        try:
            self.store.set(self.KEY, "rank %d left: %s" % (self.rank, reason))
        except Exception:      # the store itself may be gone; the timeout still ends the run
            pass

    def guard(self):
        import contextlib

        @contextlib.contextmanager
        def _guard():
            try:
                yield self
            except RankFailure:
                raise
            except BaseException as e:
                self.signal("%s: %s" % (type(e).__name__, e))
                raise
        return _guard()
