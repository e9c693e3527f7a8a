"""One mesh sharded over two ranks on the GPU: the gathered result equals the single-GPU
run of the whole mesh bit for bit.  The two ranks share one GPU (their kernels never wait
on each other; they meet only in host-side gloo exchanges between steps)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as tmp

import manapy_b200 as M
from manapy_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, key, n, steps, out):
    import datetime
    import torch
    import torch.distributed as dist
    from manapy_b200.sharded import ShardedAdvectionDiffusion
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        wl = W.ALL[key].scaled(n=n)
        el, vx = wl.mesh()
        from manapy_b200 import geometry as G
        A = G.build(el, vx, wl.dim)
        S = ShardedAdvectionDiffusion(el, vx, wl.dim, wl.bc, wl.bc_values, wl.velocity, *wl.diffusion,
                                      order=wl.order, cfl=wl.cfl)
        S.set_cells(wl.init(A["cells_center"]))
        S.advance(steps)
        w = S.gather()
        if rank == 0:
            np.save(out, w)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("key,n,steps", [("C2", 40, 10), ("C4", 6, 5)])
def test_sharded_equals_single_gpu(tmp_path, key, n, steps, cuda):
    wl = W.ALL[key].scaled(n=n)
    el, vx = wl.mesh()
    # the shards keep manapy's stencil order; so does the single-domain run compared with them
    dom = M.Domain(dim=wl.dim, mesh=(el, vx), stencil="manapy")
    w = M.Variable(domain=dom, BC=wl.bc, values=wl.bc_values)
    vel = [M.Variable(domain=dom) for _ in range(3)]
    for var, a in zip(vel, wl.velocity(dom.faces.center)):
        var.face = a
        var.interpolate_facetocell()
    w.cell = wl.init(dom.cells.center)
    # the shards gather each cell's whole stencil (no edge sums), as this run does
    S = M.AdvectionDiffusionSolver(w, vel=tuple(vel), conf=M.Struct(Dxx=wl.diffusion[0], Dyy=wl.diffusion[1],
                                                                     Dzz=wl.diffusion[2], order=wl.order, cfl=wl.cfl,
                                                                     lsq_sums=False))
    S.advance(steps)
    out = str(tmp_path / "w.npy")
    tmp.spawn(_rank, args=(2, _free_port(), key, n, steps, out), nprocs=2, join=True)
    assert np.array_equal(np.load(out), w.cell)


def _sw_rank(rank, world, port, n, steps, walls, out):
    import datetime
    import torch
    import torch.distributed as dist
    from manapy_b200.sharded import ShardedShallowWater
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        wl = W.C3.scaled(n=n)
        el, vx = wl.mesh()
        from manapy_b200 import geometry as G
        A = G.build(el, vx, 2)
        S = ShardedShallowWater(el, vx, cfl=wl.cfl, grav=wl.grav, walls=walls, sync_every=4)
        S.set_state(*wl.init_sw(A["cells_center"]))
        S.advance(steps)
        h, hu, hv = S.gather()
        if rank == 0:
            np.savez(out, h=h, hu=hu, hv=hv)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("walls", ["neumann", "reflective"])
def test_sharded_shallow_water_equals_single_gpu(tmp_path, walls, cuda):
    n, steps = 40, 12
    wl = W.C3.scaled(n=n)
    el, vx = wl.mesh()
    dom = M.Domain(dim=2, mesh=(el, vx))
    vs = [M.Variable(domain=dom) for _ in range(5)]
    for var, a in zip(vs, wl.init_sw(dom.cells.center)):
        var.cell = a
    S = M.ShallowWaterSolver(vs[0], hvel=(vs[1], vs[2]), hc=vs[3], Z=vs[4],
                             conf=M.Struct(order=1, cfl=wl.cfl, grav=wl.grav, walls=walls))
    S.advance(steps)
    out = str(tmp_path / "sw.npz")
    tmp.spawn(_sw_rank, args=(2, _free_port(), n, steps, walls, out), nprocs=2, join=True)
    got = np.load(out)
    for name, var in zip(("h", "hu", "hv"), vs[:3]):
        assert np.array_equal(got[name], var.cell), name


def test_bench_sharded_mode_runs_two_ranks(tmp_path, cuda):
    """bench.py under torchrun with two ranks splits one mesh (here both ranks share the one
    GPU and exchange through gloo) and prints one line with strong scaling."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, MANAPY_B200_BENCH_BACKEND="gloo")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), os.path.join(root, "bench.py"), "--gpus", "2",
           "--steps", "3", "--warmup", "3", "--mesh-n", "60", "--min-timed-steps", "3", "--e2e-steps", "2"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=root)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["scaling"] == "strong" and d["config"]["parallelism"] == "sharded2"
    assert d["value"] > 0 and d["e2e"]["value"] > 0
