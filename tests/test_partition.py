"""Sharding one mesh over ranks: the owned cells of every shard reproduce the
single-domain run bit for bit (two gloo ranks on the CPU, the oracle as the step)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as tmp

from manapy_b200 import boundary as B, geometry as G, partition as P, workloads as W


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_for(A, wl):
    import oracle as O
    o = O.AdvDiffOracle(A, B.resolve(A, wl.bc, wl.bc_values), *wl.diffusion, order=wl.order, cfl=wl.cfl)
    o.set_velocity(*wl.velocity(A["faces_center"]))
    o.w[:] = wl.init(A["cells_center"])
    return o


def _rank_main(rank, world, port, key, n, steps, out_dir):
    import datetime
    import sys
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        wl = W.ALL[key].scaled(n=n)
        el, vx = wl.mesh()
        shard = P.build_shards(el, vx, wl.dim, world)[rank]
        A = G.build(shard.elements, shard.vertex, wl.dim, halo_rim=True)
        o = _oracle_for(A, wl)
        ex = P.HaloExchange(shard)
        for _ in range(steps):
            dt = torch.tensor([o.stepper()], dtype=torch.float64)
            dist.all_reduce(dt, op=dist.ReduceOp.MIN)
            o.dt = float(dt.item())
            o.compute_fluxes()
            o.compute_new_val()
            w = torch.from_numpy(o.w)
            ex.exchange(w)
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), cells=shard.cells[shard.owned],
                 w=o.w[shard.owned], dt=o.dt)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("key,n,steps", [("C2", 24, 12), ("C1", 20, 15), ("C4", 5, 6)])
def test_two_shards_reproduce_the_single_domain_run(tmp_path, key, n, steps):
    wl = W.ALL[key].scaled(n=n)
    el, vx = wl.mesh()
    o = _oracle_for(G.build(el, vx, wl.dim), wl)
    for _ in range(steps):
        o.step()
    port = _free_port()
    tmp.spawn(_rank_main, args=(2, port, key, n, steps, str(tmp_path)), nprocs=2, join=True)
    got = np.full(len(o.w), np.nan)
    for r in range(2):
        d = np.load(tmp_path / ("rank%d.npz" % r))
        got[d["cells"]] = d["w"]
        assert float(d["dt"]) == o.dt
    assert np.array_equal(got, o.w)


def test_shards_cover_the_mesh_once():
    wl = W.C2.scaled(n=30)
    el, vx = wl.mesh()
    shards = P.build_shards(el, vx, 2, 4)
    owned = np.concatenate([s.cells[s.owned] for s in shards])
    assert np.array_equal(np.sort(owned), np.arange(len(el)))
    for s in shards:
        for q, idx in s.recv.items():
            # what q sends to s is what s receives, cell for cell
            assert np.array_equal(shards[q].cells[shards[q].send[s.rank]], s.cells[idx])
            assert not s.owned[idx].any() and shards[q].owned[shards[q].send[s.rank]].all()
