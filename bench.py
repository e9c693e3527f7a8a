"""Benchmark of the explicit finite-volume step (cell-updates/s).

Default workload: the 2,000,000-triangle second-order advection-diffusion run
(mesh 1000x1000 squares, LSQ gradient + Barth limiter + diamond diffusion,
rotating velocity, D = 5e-4), FP64, 1000 steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = manapy's ``stepper()`` + ``compute_fluxes()`` + ``compute_new_val()``
on the whole mesh.  ``value`` is timed on the device (CUDA events, inputs
resident, K steps replayed from CUDA graphs); ``e2e`` runs the manapy driver
loop through the public API (per step: the face velocities copied from pinned
host memory, ``interpolate_facetocell``, ``stepper()`` returning dt to the
host, ``compute_fluxes()``, ``compute_new_val()``).  Under torchrun every rank
solves its own copy of the workload (weak scaling, no collective in the step).

``--impl reference`` times the CPU restatement of manapy's kernels (the
oracle, one process per host core, each on its own copy of the mesh).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# compulsory-traffic bytes per cell-update (FP64), per workload
CTM_BYTES = {"C1": 146.6, "C2": 198.8, "C3": 152.4, "C4": 265.9}
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="C2", choices=["C1", "C2", "C3", "C4"])
    ap.add_argument("--e2e-steps", type=int, default=30)
    ap.add_argument("--cpu-steps", type=int, default=5, help="oracle steps of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--n", type=int, default=None, help="mesh resolution override (small profiling cases)")
    return ap.parse_args()


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(workload):
    """DRAM bytes per cell-update of one step, from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(p) as f:
            return json.load(f)[workload]
    except Exception:
        return None


class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        loaded = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def build_advdiff(wl, seed):
    import manapy_b200 as M
    el, vx = wl.scaled(seed=seed).mesh()
    dom = M.Domain(dim=wl.dim, mesh=(el, vx))
    w = M.Variable(domain=dom, BC=wl.bc, values=wl.bc_values)
    u, v, wz = (M.Variable(domain=dom) for _ in range(3))
    uf, vf, wf = wl.velocity(dom.faces.center)
    u.face = uf
    v.face = vf
    wz.face = wf
    for x in (u, v, wz):
        x.interpolate_facetocell()
    w.cell = wl.init(dom.cells.center)
    S = M.AdvectionDiffusionSolver(w, vel=(u, v, wz), conf=M.Struct(
        Dxx=wl.diffusion[0], Dyy=wl.diffusion[1], Dzz=wl.diffusion[2], order=wl.order, cfl=wl.cfl))
    return dom, w, (u, v, wz), S, (uf, vf)


def build_sw(wl, seed):
    import manapy_b200 as M
    el, vx = wl.scaled(seed=seed).mesh()
    dom = M.Domain(dim=2, mesh=(el, vx))
    vs = [M.Variable(domain=dom) for _ in range(5)]
    for var, a in zip(vs, wl.init_sw(dom.cells.center)):
        var.cell = a
    S = M.ShallowWaterSolver(vs[0], hvel=(vs[1], vs[2]), hc=vs[3], Z=vs[4],
                             conf=M.Struct(order=wl.order, cfl=wl.cfl, grav=wl.grav))
    return dom, vs, S


def cpu_baseline(dom, wl, steps):
    """The oracle (serial C port of manapy's kernels) on this host, same mesh."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from manapy_b200 import boundary as B
    A = dom.host_arrays
    m = O.Mesh(A)
    if wl.kind == "advdiff":
        o = O.AdvDiffOracle(A, B.resolve(A, wl.bc, wl.bc_values), *wl.diffusion, order=wl.order,
                            cfl=wl.cfl, mesh=m)
        o.set_velocity(*wl.velocity(A["faces_center"]))
        o.w[:] = wl.init(A["cells_center"])
    else:
        o = O.ShallowWaterOracle(A, order=wl.order, cfl=wl.cfl, grav=wl.grav, mesh=m)
        for k, a in zip(("h", "hu", "hv", "hc", "Z"), wl.init_sw(A["cells_center"])):
            o.state()[k][:] = a
    o.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step()
    el = time.perf_counter() - t0
    return {"value": wl.cells * steps / el, "unit": "cell-updates/s", "cores": 1, "kind": "port",
            "sample": "%d steps of the full %d-cell mesh, serial C restatement of manapy's kernels"
                      % (steps, wl.cells)}


def run_ours(args):
    import torch
    from manapy_b200 import workloads as W
    world, rank, local = dist_setup(args)
    wl = W.ALL[args.workload]
    if args.n:
        wl = wl.scaled(n=args.n)
    K, Wm = args.steps, max(args.warmup, 3)
    if wl.kind == "advdiff":
        dom, w, vel, S, (uf, vf) = build_advdiff(wl, seed=wl.seed + rank)
    else:
        dom, vs, S = build_sw(wl, seed=wl.seed + rank)
    dev = torch.device("cuda", local if world > 1 else 0)
    # warm-up (also captures the CUDA graphs)
    if wl.kind == "advdiff":
        S.advance(Wm, graph=True)
    else:
        S.advance(Wm)
    torch.cuda.synchronize()
    clocks = ClockSampler(local if world > 1 else 0)
    time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    if wl.kind == "advdiff":
        S.advance(K, graph=True)
    else:
        S.advance(K)
    e1.record()
    torch.cuda.synchronize()
    barrier(world)
    ms = e0.elapsed_time(e1)
    ck = clocks.stop()
    ms_max = max_over_ranks(ms, world)
    value = world * wl.cells * K / (ms_max / 1e3)
    ms_step = ms_max / K
    launches_per_step = S.launches_per_step()

    # end to end through the public API, manapy's driver loop
    E = max(args.e2e_steps, 1)
    h2d = d2h = 0
    if wl.kind == "advdiff":
        u, v, _ = vel
        pu = torch.from_numpy(uf).pin_memory()
        pv = torch.from_numpy(vf).pin_memory()
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(E):
            u.face = pu
            v.face = pv
            u.interpolate_facetocell()
            v.interpolate_facetocell()
            S.stepper()
            S.compute_fluxes()
            S.compute_new_val()
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        h2d = pu.numel() * 8 + pv.numel() * 8
        d2h = 8
    else:
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(E):
            S.stepper()
            S.compute_fluxes()
            S.compute_new_val()
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        d2h = 8
    e2e_s = max_over_ranks(e2e_s, world)
    e2e_value = world * wl.cells * E / e2e_s

    peak, peak_kind = measured_peak()
    ctm = CTM_BYTES[args.workload]
    achieved = ctm * wl.cells / (ms_step / 1e3) / 1e9
    traffic = ncu_traffic(args.workload)
    line = {
        "metric": "cell-updates/s (FP64 explicit FV step, %s)" % wl.name,
        "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": K, "warmup": Wm,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic: seeded jittered mesh of the workload, manapy's initial state",
        "config": {"workload": wl.name, "cells": wl.cells, "order": wl.order, "kind": wl.kind,
                   "parallelism": "replicas%d" % world if world > 1 else "single",
                   "l2": "working set %.0f MB > 126 MB L2 (no flush needed)" % (dom.device_mesh.nbytes() / 1e6)},
        "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": E},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": (traffic * wl.cells if traffic else None),
                     "kernel": "fused step (%d launches), compulsory traffic %.1f B/cell-update"
                               % (launches_per_step, ctm)},
        "clocks": ck,
        "gpu_launches": launches_per_step * K,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(dom, wl, args.cpu_steps)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        S.release_graphs()
        dist.destroy_process_group()


def _ref_worker(wk, steps, warmup, q):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from manapy_b200 import boundary as B, geometry as G, workloads as W
    wl = W.ALL[wk]
    el, vx = wl.mesh()
    A = G.build(el, vx, wl.dim)
    m = O.Mesh(A)
    if wl.kind == "advdiff":
        o = O.AdvDiffOracle(A, B.resolve(A, wl.bc, wl.bc_values), *wl.diffusion, order=wl.order, cfl=wl.cfl,
                            mesh=m)
        o.set_velocity(*wl.velocity(A["faces_center"]))
        o.w[:] = wl.init(A["cells_center"])
    else:
        o = O.ShallowWaterOracle(A, order=wl.order, cfl=wl.cfl, grav=wl.grav, mesh=m)
        for k, a in zip(("h", "hu", "hv", "hc", "Z"), wl.init_sw(A["cells_center"])):
            o.state()[k][:] = a
    for _ in range(warmup):
        o.step()
    q.put(("ready", 0.0))
    go = q.get()  # noqa: F841
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step()
    q.put(("done", time.perf_counter() - t0))


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp
    from manapy_b200 import workloads as W
    wl = W.ALL[args.workload]
    ctx = mp.get_context("spawn")
    cores = os.cpu_count() or 1
    # host RAM bounds the number of mesh copies (about 4 GB each at 2M cells)
    try:
        mem_gb = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES") / 1e9
    except Exception:
        mem_gb = 32
    per = max(wl.cells / 2e6 * 4.0, 0.05)
    procs_n = max(1, min(cores, int(mem_gb * 0.5 / per), 32))
    # each timed step of every process is one full oracle step; bound the sample
    steps = max(1, min(args.steps, 3))
    warm = 1
    qs, ps = [], []
    for _ in range(procs_n):
        q = ctx.Queue()
        p = ctx.Process(target=_ref_worker, args=(args.workload, steps, warm, q))
        p.start()
        qs.append(q)
        ps.append(p)
    for q in qs:
        assert q.get()[0] == "ready"
    t0 = time.perf_counter()
    for q in qs:
        q.put("go")
    times = [q.get()[1] for q in qs]
    wall = time.perf_counter() - t0
    for p in ps:
        p.join()
    value = procs_n * wl.cells * steps / wall
    line = {
        "metric": "cell-updates/s (FP64 explicit FV step, %s)" % wl.name, "impl": "reference",
        "value": value, "unit": "cell-updates/s", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * max(times) / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded jittered mesh of the workload, manapy's initial state",
        "config": {"workload": wl.name, "cells": wl.cells, "order": wl.order, "kind": wl.kind},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": procs_n, "kind": "port",
                         "sample": "%d processes x %d full-mesh steps of the serial C restatement of "
                                   "manapy's kernels (manapy itself runs one core per process)"
                                   % (procs_n, steps)},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
