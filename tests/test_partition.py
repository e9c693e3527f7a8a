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


def _sw_rank_main(rank, world, port, n, steps, out_dir):
    """Shallow water on one shard with the oracle as the step: per step the dt of the
    current state over the rank's cells (min over ranks), the step, the exchange of
    h, hu, hv, hc."""
    import datetime
    import sys
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import oracle as O
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        wl = W.C3.scaled(n=n)
        el, vx = wl.mesh()
        # every shard also holds the last cell, which the source term reads for cellfid padding
        shard = P.build_shards(el, vx, 2, world, extra_cells=[len(el) - 1])[rank]
        A = G.build(shard.elements, shard.vertex, 2, halo_rim=True)
        o = O.ShallowWaterOracle(A, order=1, cfl=wl.cfl, grav=wl.grav)
        for k, a in zip(("h", "hu", "hv", "hc", "Z"), wl.init_sw(A["cells_center"])):
            o.state()[k][:] = a
        ex = P.HaloExchange(shard)
        fields = [torch.from_numpy(o.state()[k]) for k in ("h", "hu", "hv", "hc")]
        for _ in range(steps):
            dt = torch.tensor([o.stepper()], dtype=torch.float64)
            dist.all_reduce(dt, op=dist.ReduceOp.MIN)
            o.dt = float(dt.item())
            o.compute_fluxes()
            o.compute_new_val()
            ex.exchange(fields)          # the oracle's arrays, in place
        own = shard.owned
        np.savez(os.path.join(out_dir, "sw%d.npz" % rank), cells=shard.cells[own], h=o.h[own], hu=o.hu[own],
                 hv=o.hv[own])
    finally:
        dist.destroy_process_group()


def test_two_shards_reproduce_the_single_domain_shallow_water_run(tmp_path):
    import oracle as O
    n, steps = 26, 12
    wl = W.C3.scaled(n=n)
    el, vx = wl.mesh()
    o = O.ShallowWaterOracle(G.build(el, vx, 2), order=1, cfl=wl.cfl, grav=wl.grav)
    for k, a in zip(("h", "hu", "hv", "hc", "Z"), wl.init_sw(o.m.A["cells_center"])):
        o.state()[k][:] = a
    for _ in range(steps):
        o.step()
    tmp.spawn(_sw_rank_main, args=(2, _free_port(), n, steps, str(tmp_path)), nprocs=2, join=True)
    for name in ("h", "hu", "hv"):
        got = np.full(o.m.nc, np.nan)
        for r in range(2):
            d = np.load(tmp_path / ("sw%d.npz" % r))
            got[d["cells"]] = d[name]
        assert np.array_equal(got, getattr(o, name)), name


def _failing_rank_main(rank, world, port, mode, out_dir):
    """Rank 1 leaves after two steps -- posting its failure (``mode="signal"``) or silently
    (``"silent"``, a process exit); rank 0 keeps stepping and records what it raised."""
    import datetime
    import json
    import time
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=4))
    wl = W.C2.scaled(n=16)
    el, vx = wl.mesh()
    shard = P.build_shards(el, vx, 2, world)[rank]
    ex = P.HaloExchange(shard)
    mon = P.FailureMonitor(rank, timeout=3.0)
    field = torch.zeros(len(shard.cells), dtype=torch.float64)
    t0 = time.time()
    outcome = {"rank": rank, "raised": None}
    try:
        for step in range(50):
            if rank == 1 and step == 2:          # leave between steps 1 and 2
                if mode == "silent":
                    os._exit(3)
                with mon.guard():
                    raise ValueError("injected failure at step 2")
            mon.sync(step)               # the heartbeat between steps
            with mon.guard():
                field += 1.0
                ex.exchange(field)
    except P.RankFailure as e:
        outcome.update(raised="RankFailure", msg=str(e))
    except ValueError as e:
        outcome.update(raised="ValueError", msg=str(e))
    except Exception as e:       # the exchange's timeout or the closed connection
        outcome.update(raised=type(e).__name__, msg=str(e)[:200])
    outcome["seconds"] = time.time() - t0
    with open(os.path.join(out_dir, "outcome%d.json" % rank), "w") as f:
        json.dump(outcome, f)
    os._exit(0)


@pytest.mark.parametrize("mode", ["signal", "silent"])
def test_a_rank_that_leaves_between_steps_ends_the_others_cleanly(tmp_path, mode):
    import json
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    port = _free_port()
    ps = [ctx.Process(target=_failing_rank_main, args=(r, 2, port, mode, str(tmp_path))) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=60)
    for p in ps:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not end within 60 s")
    with open(tmp_path / "outcome0.json") as f:
        out0 = json.load(f)
    # rank 0 learns of it on the host, before it enters the next exchange
    assert out0["raised"] == "RankFailure", out0
    if mode == "signal":
        assert "rank 1 left" in out0["msg"] and "injected failure" in out0["msg"], out0
        with open(tmp_path / "outcome1.json") as f:
            assert json.load(f)["raised"] == "ValueError"
    else:
        assert "did not reach step 2" in out0["msg"], out0
    assert out0["seconds"] < 30
