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
    dom = M.Domain(dim=wl.dim, mesh=(el, vx))
    w = M.Variable(domain=dom, BC=wl.bc, values=wl.bc_values)
    vel = [M.Variable(domain=dom) for _ in range(3)]
    for var, a in zip(vel, wl.velocity(dom.faces.center)):
        var.face = a
        var.interpolate_facetocell()
    w.cell = wl.init(dom.cells.center)
    S = M.AdvectionDiffusionSolver(w, vel=tuple(vel), conf=M.Struct(Dxx=wl.diffusion[0], Dyy=wl.diffusion[1],
                                                                     Dzz=wl.diffusion[2], order=wl.order, cfl=wl.cfl))
    S.advance(steps)
    out = str(tmp_path / "w.npy")
    tmp.spawn(_rank, args=(2, _free_port(), key, n, steps, out), nprocs=2, join=True)
    assert np.array_equal(np.load(out), w.cell)
