"""Benchmark of the explicit finite-volume step (cell-updates/s).

Default workload: the 2,000,000-triangle second-order advection-diffusion run
(mesh 1000x1000 squares, LSQ gradient + Barth limiter + diamond diffusion,
rotating velocity, D = 5e-4), FP64, 1000 steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = manapy's ``stepper()`` + ``compute_fluxes()`` + ``compute_new_val()``
on the whole mesh.  ``value`` is timed on the device (CUDA events, inputs
resident, K steps replayed from CUDA graphs), as the median of R repeats of
exactly K steps each (R = ceil(500 / K) by default, so that at least 500 steps
are timed; every repeat is bracketed by a barrier and a synchronisation).
``e2e`` runs the manapy driver loop through the public API (per step: the face
velocities copied from pinned host memory, ``interpolate_facetocell``,
``stepper()`` returning dt to the host, ``compute_fluxes()``,
``compute_new_val()``, and the new state copied back into pinned host memory).
Under torchrun every rank solves its own copy of the workload (weak scaling, no
collective in the step); ``--sharded`` instead splits one mesh over the ranks
(halo exchange and dt min-reduction over NCCL).

The single-GPU default run adds the other stated targets to the same line
(``extras``): the 3D workload C4 at full size, a resident batch of uneven meshes
(batched FP32-compensated vs batched FP64 vs the same meshes solved serially in
FP64) and a continuous-batching serving run (p50/p99 latency at a stated arrival
rate).

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
CTM_BYTES = {"C1": 146.6, "C2": 198.8, "C3": 152.4, "C4": 265.9, "E1": 171.0}
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="C2", choices=["C1", "C2", "C3", "C4", "E1"])
    ap.add_argument("--e2e-steps", type=int, default=30)
    ap.add_argument("--cpu-steps", type=int, default=15,
                    help="oracle steps of the CPU baseline sample (about 10-30 s of serial work at 2M cells)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32c", action="store_true", help="skip the FP32-compensated measurement")
    ap.add_argument("--serve", action="store_true", help="continuous-batching serving run instead of one workload")
    ap.add_argument("--batched", action="store_true",
                    help="resident batch of uneven meshes: batched FP32-compensated kernels vs serial FP64 solves")
    ap.add_argument("--meshes", type=int, default=48, help="batched: number of meshes")
    ap.add_argument("--requests", type=int, default=300, help="serving: number of requests")
    ap.add_argument("--rate", type=float, default=15.0, help="serving: Poisson arrival rate (requests/s)")
    ap.add_argument("--serial-sample", type=int, default=60, help="serving: requests timed serially in FP64")
    ap.add_argument("--workers", type=int, default=None, help="serving: mesh-preparation processes")
    ap.add_argument("--n", "--mesh-n", dest="n", type=int, default=None,
                    help="mesh resolution override (small profiling cases; --mesh-n under torchrun, whose own "
                         "options start with --n)")
    ap.add_argument("--launch", type=int, default=None,
                    help="launch-shape variant of the fused phases (0-15; default: tuned per mesh), for "
                         "profiling one shape")
    ap.add_argument("--min-timed-steps", type=int, default=500,
                    help="repeat the K timed steps until at least this many steps are timed (median reported)")
    ap.add_argument("--no-extras", action="store_true",
                    help="single workload only (no C4 / batched / serving sections)")
    ap.add_argument("--extras-requests", type=int, default=1000, help="serving section: requests")
    ap.add_argument("--extras-rate", type=float, default=18.0, help="serving section: arrival rate (requests/s)")
    ap.add_argument("--replicas", action="store_true",
                    help="under torchrun: every rank solves its own copy (weak scaling) instead of one sharded mesh")
    ap.add_argument("--section", default=None, choices=["c4", "batched", "serving"],
                    help="run one extras section alone and print its JSON (the default run starts each "
                         "section in a process of its own)")
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
        # MANAPY_B200_BENCH_BACKEND=gloo runs the ranks' exchanges through host memory, so that
        # the multi-rank path can be exercised with every rank on one GPU (NCCL needs one GPU
        # per rank); the default is NCCL with one GPU per rank
        backend = os.environ.get("MANAPY_B200_BENCH_BACKEND", "nccl")
        local = local % torch.cuda.device_count() if backend == "gloo" else local
        torch.cuda.set_device(local)
        if backend == "gloo":
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
        else:
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


def timed_repeats(run, K, R, world):
    """R repeats of exactly K steps, each bracketed by a barrier and a synchronisation and
    timed with CUDA events on the launching stream; per repeat the max over ranks (ms)."""
    import torch
    out = []
    for _ in range(R):
        barrier(world)
        torch.cuda.synchronize()
        st = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        run(K)
        e1.record(st)
        torch.cuda.synchronize()
        barrier(world)
        out.append(max_over_ranks(e0.elapsed_time(e1), world))
    return out


def repeats_for(K, args):
    return max(1, -(-int(args.min_timed_steps) // max(int(K), 1)))


def build_advdiff(wl, seed, launch="auto"):
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
        Dxx=wl.diffusion[0], Dyy=wl.diffusion[1], Dzz=wl.diffusion[2], order=wl.order, cfl=wl.cfl, launch=launch))
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


def run_fp32c(wl, dom, w64, vel, K, Wm, world, R=1):
    """The FP32-compensated step on the same mesh and initial state: device-timed
    throughput (median of R repeats of K steps), and its L2 / Linf error against the FP64
    state after the same number of steps (Wm + R K)."""
    import torch
    import manapy_b200 as M
    ref = w64.cell.copy()          # FP64 state after Wm + K steps
    w = M.Variable(domain=dom, BC=wl.bc, values=wl.bc_values)
    w.cell = wl.init(dom.cells.center)
    S = M.AdvectionDiffusionSolver(w, vel=vel, conf=M.Struct(
        Dxx=wl.diffusion[0], Dyy=wl.diffusion[1], Dzz=wl.diffusion[2], order=wl.order, cfl=wl.cfl,
        precision="fp32c"))
    S.advance(Wm, graph=True)
    torch.cuda.synchronize()
    ms = statistics.median(timed_repeats(lambda n: S.advance(n, graph=True), K, R, world))
    got = w.cell
    l2 = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    linf = float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
    S.release_graphs()
    return {"value": world * wl.cells * K / (ms / 1e3), "unit": "cell-updates/s", "ms_per_step": ms / K,
            "dtype": "f32 state + compensated sums, f64 geometry and dt",
            "l2_rel_err_vs_fp64": l2, "linf_rel_err_vs_fp64": linf, "steps_compared": Wm + K * R}


def run_fp32c_sw(wl, dom, vs64, S64, K, Wm, world, R=1):
    """FP32-compensated shallow water on the same mesh and initial state: throughput, L2 /
    Linf error of h, hu, hv against the FP64 state after the same steps, FP64 mass drift."""
    import torch
    import manapy_b200 as M
    ref = [v.cell.copy() for v in vs64[:3]]
    m64 = S64.mass()
    vs = [M.Variable(domain=dom) for _ in range(5)]
    for var, a in zip(vs, wl.init_sw(dom.cells.center)):
        var.cell = a
    S = M.ShallowWaterSolver(vs[0], hvel=(vs[1], vs[2]), hc=vs[3], Z=vs[4],
                             conf=M.Struct(order=wl.order, cfl=wl.cfl, grav=wl.grav, precision="fp32c"))
    m0 = S.mass()
    S.advance(Wm)
    torch.cuda.synchronize()
    ms = statistics.median(timed_repeats(S.advance, K, R, world))
    out = {"value": world * wl.cells * K / (ms / 1e3), "unit": "cell-updates/s", "ms_per_step": ms / K,
           "dtype": "f32 state and fluxes + compensated sums, f64 geometry, source and dt",
           "steps_compared": Wm + K * R}
    for name, r, v in zip(("h", "hu", "hv"), ref, vs[:3]):
        got = v.cell
        out["l2_rel_err_vs_fp64_" + name] = float(np.linalg.norm(got - r) / np.linalg.norm(r))
        out["linf_rel_err_vs_fp64_" + name] = float(np.max(np.abs(got - r)) / np.max(np.abs(r)))
    out["mass_fp64_sum"] = {"start": m0, "fp32c_end": S.mass(), "fp64_end": m64}
    return out


def build_euler(wl, seed):
    import manapy_b200 as M
    el, vx = wl.scaled(seed=seed).mesh()
    dom = M.Domain(dim=2, mesh=(el, vx))
    vs = [M.Variable(domain=dom) for _ in range(5)]
    for var, a in zip(vs, wl.init_euler(dom.cells.center, wl.gamma)):
        var.cell = a
    S = M.EulerSolver(*vs, conf=M.Struct(cfl=wl.cfl, gamma=wl.gamma))
    return dom, vs, S


def cpu_baseline_euler(dom, wl, steps):
    """The oracle's Euler step (serial C restatement of manapy's kernels) on this host."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    A = dom.host_arrays
    m = O.Mesh(A)
    q = [np.ascontiguousarray(a, dtype=np.float64) for a in wl.init_euler(A["cells_center"], wl.gamma)]
    O.euler_step_2d(m, q, wl.cfl, wl.gamma)
    t0 = time.perf_counter()
    for _ in range(steps):
        O.euler_step_2d(m, q, wl.cfl, wl.gamma)
    el = time.perf_counter() - t0
    return {"value": wl.cells * steps / el, "unit": "cell-updates/s", "cores": 1, "kind": "port",
            "sample": "%d steps of the full %d-cell mesh, serial C restatement of manapy's euler kernels"
                      % (steps, wl.cells)}


def run_euler(args, wl):
    """The 2D Euler Rusanov step (EulerSolver): two launches per step, dt reduced on the device."""
    import torch
    world, rank, local = dist_setup(args)
    # warm-up long enough to capture the step graph (GRAPH_DEPTH steps, aligned to 6)
    K, Wm = args.steps, max(args.warmup, 3)
    dom, vs, S = build_euler(wl, seed=wl.seed + rank)
    Wm = max(Wm, S.GRAPH_DEPTH + 6)
    S.advance(Wm, graph=True)
    torch.cuda.synchronize()
    clocks = ClockSampler(local if world > 1 else 0)
    time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    S.advance(K, graph=True)
    e1.record()
    torch.cuda.synchronize()
    barrier(world)
    ms = e0.elapsed_time(e1)
    ck = clocks.stop()
    ms_max = max_over_ranks(ms, world)
    value = world * wl.cells * K / (ms_max / 1e3)
    ms_step = ms_max / K
    S.check()
    # end to end, a manapy-style driver loop: dt read back every step
    E = max(args.e2e_steps, 1)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(E):
        S.stepper()
        S.compute_new_val()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    peak, peak_kind = measured_peak()
    ctm = CTM_BYTES["E1"]
    achieved = ctm * wl.cells / (ms_step / 1e3) / 1e9
    traffic = ncu_traffic("E1")
    line = {
        "metric": "cell-updates/s (FP64 Euler Rusanov step, %s)" % wl.name,
        "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": K, "warmup": Wm,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic: seeded jittered mesh, pressure pulse in a sheared flow",
        "config": {"workload": wl.name, "cells": wl.cells, "order": 1, "kind": "euler",
                   "parallelism": "replicas%d" % world if world > 1 else "single",
                   "l2": "working set %.0f MB > 126 MB L2 (no flush needed)" % (dom.device_mesh.nbytes() / 1e6)},
        "e2e": {"value": world * wl.cells * E / e2e_s, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 8, "steps": E},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": (traffic * wl.cells if traffic else None),
                     "kernel": "face flux + cell update (2 launches), compulsory traffic %.1f B/cell-update" % ctm},
        "clocks": ck,
        "gpu_launches": S.launches_per_step() * K,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_euler(dom, wl, args.cpu_steps)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        S.release_graphs()
        dist.destroy_process_group()


def measure_workload(wl, args, world, rank, local, K, fp32c=True, seed_offset=0):
    """Device-timed FP64 step of one workload (median of repeats), its FP32-compensated
    twin, and the objects the end-to-end leg needs."""
    import torch
    Wm = max(args.warmup, 3)
    if wl.kind == "advdiff":
        dom, w, vel, S, (uf, vf) = build_advdiff(wl, seed=wl.seed + seed_offset,
                                                  launch="auto" if args.launch is None else args.launch)
    else:
        dom, vs, S = build_sw(wl, seed=wl.seed + seed_offset)
    # warm-up: also tunes the steps per graph replay and captures the step graph, so that
    # neither happens inside the timed region (the deepest candidate bounds the steps needed)
    if wl.kind == "advdiff":
        from manapy_b200 import autotune
        Wm = Wm + max(autotune.CANDIDATES)
        run = lambda n: S.advance(n, graph=True)  # noqa: E731
    else:
        run = S.advance
    run(Wm)
    torch.cuda.synchronize()
    R = repeats_for(K, args)
    clocks = ClockSampler(local if world > 1 else 0)
    time.sleep(0.3)
    reps = timed_repeats(run, K, R, world)
    ck = clocks.stop()
    ms_med = statistics.median(reps)
    out = {"dom": dom, "S": S, "K": K, "R": R, "Wm": Wm, "reps": reps, "ms_step": ms_med / K, "clocks": ck,
           "value": world * wl.cells * K / (ms_med / 1e3), "launches": S.launches_per_step()}
    if wl.kind == "advdiff":
        out.update(w=w, vel=vel, uf=uf, vf=vf)
    else:
        out.update(vs=vs)
    if fp32c and not args.no_fp32c:
        # the FP32c run takes as many steps as the FP64 run (warm-up + R K) for the comparison
        if wl.kind == "advdiff":
            out["fp32c"] = run_fp32c(wl, dom, w, vel, K, Wm, world, R)
        elif wl.order == 1:
            out["fp32c"] = run_fp32c_sw(wl, dom, vs, S, K, Wm, world, R)
        if "fp32c" in out:
            out["fp32c"]["vs_fp64"] = out["fp32c"]["value"] / out["value"]
    return out


def roofline(wl_key, cells, ms_step, launches):
    peak, peak_kind = measured_peak()
    ctm = CTM_BYTES[wl_key]
    achieved = ctm * cells / (ms_step / 1e3) / 1e9
    traffic = ncu_traffic(wl_key)
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": peak_kind, "traffic": (traffic * cells if traffic else None),
            "kernel": "fused step (%d launches), compulsory traffic %.1f B/cell-update" % (launches, ctm)}


def e2e_advdiff(m, E, world):
    """manapy's driver loop through the public API: per step the face velocities uploaded
    from pinned memory, facetocell, stepper() (dt to the host), compute_fluxes(),
    compute_new_val(), and the new state copied back into pinned memory."""
    import torch
    S, w = m["S"], m["w"]
    u, v, _ = m["vel"]
    pu = torch.from_numpy(m["uf"]).pin_memory()
    pv = torch.from_numpy(m["vf"]).pin_memory()
    out = torch.empty(int(m["dom"].nbcells), dtype=torch.float64, pin_memory=True)
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
        w.fetch("cell", out=out)
    torch.cuda.synchronize()
    sec = max_over_ranks(time.perf_counter() - t0, world)
    return sec, pu.numel() * 8 + pv.numel() * 8, out.numel() * 8 + 8


def e2e_sw(m, E, world):
    import torch
    S, vs = m["S"], m["vs"]
    outs = [torch.empty(int(m["dom"].nbcells), dtype=torch.float64, pin_memory=True) for _ in range(3)]
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(E):
        S.stepper()
        S.compute_fluxes()
        S.compute_new_val()
        for var, o in zip(vs[:3], outs):
            var.fetch("cell", out=o)
    torch.cuda.synchronize()
    sec = max_over_ranks(time.perf_counter() - t0, world)
    return sec, 0, sum(o.numel() * 8 for o in outs) + 8


def extra_c4(args):
    """The 3D workload C4 at full size (1,572,864 tetrahedra): FP64 and FP32-compensated."""
    from manapy_b200 import workloads as W
    wl = W.C4
    m = measure_workload(wl, args, 1, 0, 0, K=50)
    out = {"workload": wl.name, "cells": wl.cells, "value": m["value"], "unit": "cell-updates/s",
           "ms_per_step": m["ms_step"], "steps": m["K"], "repeats": m["R"],
           "roofline": roofline("C4", wl.cells, m["ms_step"], m["launches"]), "clocks": m["clocks"]}
    if "fp32c" in m:
        out["fp32c"] = m["fp32c"]
    m["S"].release_graphs()
    return out


def extra_batched(args):
    """A resident batch of uneven meshes (the serving mix): batched FP32c, batched FP64 and
    the same meshes solved one after another in FP64, all device-timed over the same steps."""
    import torch
    from manapy_b200 import serving as SV
    reqs = SV.make_requests(args.meshes, 0.0, seed=77)
    K = 200
    srv = SV.BatchServer(workers=args.workers)
    srv.start_pool()
    rate32, _ = srv.run_resident(reqs, K)
    srv.stop_pool()
    srv64 = SV.BatchServer(workers=args.workers, precision="fp64")
    srv64.start_pool()
    rate64, _ = srv64.run_resident(reqs, K)
    srv64.stop_pool()
    del srv, srv64
    torch.cuda.empty_cache()
    ser = _serial_fp64(reqs, K)
    cu = sum(r.cells for r in reqs) * K
    serial = cu / ser
    return {"meshes": len(reqs), "cells": sum(r.cells for r in reqs), "steps": K,
            "mix": "70% adv-diff o2 + diffusion, 30% SW o1", "sizes": "log-uniform 2e3-5e5 cells",
            "batched_fp32c": rate32, "batched_fp64": rate64, "serial_fp64": serial, "unit": "cell-updates/s",
            "fp32c_vs_batched_fp64": rate32 / rate64, "batched_fp64_vs_serial_fp64": rate64 / serial,
            "fp32c_vs_serial_fp64": rate32 / serial}


def extra_serving(args):
    """Continuous batching of a seeded request stream (FP32-compensated): sustained rate and
    p50/p99 latency from arrival to the result on the host."""
    import torch
    from manapy_b200 import serving as SV
    reqs = SV.make_requests(args.extras_requests, args.extras_rate, seed=2024)
    total_cu = sum(r.cells * r.steps for r in reqs)
    srv = SV.BatchServer(workers=args.workers)
    srv.start_pool()
    srv.serve(SV.make_requests(8, 0.0, seed=1, cells=(2e3, 2e4), steps=(20, 40)))
    t0 = time.perf_counter()
    recs = srv.serve(reqs)
    wall = time.perf_counter() - t0
    srv.stop_pool()
    lat = np.array([r["latency"] for r in recs])
    torch.cuda.empty_cache()
    return {"requests": len(reqs), "rate_per_s": args.extras_rate, "workers": srv.workers,
            "cells": "log-uniform 2e3-5e5", "steps": "uniform 100-2000", "mix": "70% adv-diff o2, 30% SW o1",
            "precision": "fp32c", "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "makespan_s": wall, "sustained_requests_per_s": len(reqs) / wall,
            "cell_updates_per_s": total_cu / wall,
            "latency": "arrival to result on the host, mesh preparation included"}


SECTIONS = {"c4": extra_c4, "batched": extra_batched, "serving": extra_serving}


def run_section(name, args):
    """One extras section in a process of its own (its GPU memory is returned when it exits,
    and a failure there is reported in the line instead of ending this run)."""
    cmd = [sys.executable, os.path.abspath(__file__), "--section", name, "--warmup", str(args.warmup),
           "--min-timed-steps", str(args.min_timed_steps), "--meshes", str(args.meshes),
           "--extras-requests", str(args.extras_requests), "--extras-rate", str(args.extras_rate)]
    if args.workers is not None:
        cmd += ["--workers", str(args.workers)]
    if args.no_fp32c:
        cmd.append("--no-fp32c")
    t0 = time.perf_counter()
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        out = None
        for ln in reversed(p.stdout.strip().splitlines()):
            if ln.startswith("{"):
                out = json.loads(ln)
                break
        if p.returncode != 0 or out is None:
            out = {"error": "exit %d: %s" % (p.returncode, (p.stderr or p.stdout).strip()[-400:])}
    except subprocess.TimeoutExpired:
        out = {"error": "timed out after 600 s"}
    out["section_seconds"] = round(time.perf_counter() - t0, 1)
    return out


def run_sharded(args, wl, world, rank, local):
    """One advection-diffusion mesh split over the ranks (strong scaling): each rank steps
    its shard (owned cells + two-layer halo) and refreshes the halo over NCCL after every
    step; dt is the min over ranks.  ``value`` counts every cell of the mesh once."""
    import torch
    from manapy_b200.domain import build_host_mesh
    from manapy_b200.sharded import ShardedAdvectionDiffusion
    dev = torch.device("cuda", local)
    el, vx = wl.mesh()
    A, _ = build_host_mesh(el, vx, wl.dim)
    S = ShardedAdvectionDiffusion(el, vx, wl.dim, wl.bc, wl.bc_values, wl.velocity, *wl.diffusion, order=wl.order,
                                  cfl=wl.cfl, device=dev, check_every=0, A=A)
    S.set_cells(wl.init(A["cells_center"]))
    K, Wm = args.steps, max(args.warmup, 3)
    S.advance(Wm)
    torch.cuda.synchronize()
    R = repeats_for(K, args)
    clocks = ClockSampler(local)
    time.sleep(0.3)
    reps = timed_repeats(S.advance, K, R, world)
    ck = clocks.stop()
    ms_step = statistics.median(reps) / K
    # end to end: each step followed by the owned state read back into pinned memory
    E = max(args.e2e_steps, 1)
    # owned cells in the shard's device numbering (device k holds shard cell perm[k])
    own = torch.from_numpy(S.shard.owned).to(dev)[S.dm.perm["cell"]].nonzero().flatten()
    out = torch.empty(own.numel(), dtype=torch.float64, pin_memory=True)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(E):
        S.step()
        out.copy_(S.w[S.cur].index_select(0, own), non_blocking=True)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    peak, peak_kind = measured_peak()
    ctm = CTM_BYTES[args.workload]
    achieved = ctm * wl.cells / (ms_step / 1e3) / 1e9
    halo = int((~S.shard.owned).sum())
    line = {
        "metric": "cell-updates/s (FP64 explicit FV step, %s)" % wl.name,
        "value": wl.cells * K / (statistics.median(reps) / 1e3), "unit": "cell-updates/s", "n_gpus": world,
        "steps": K, "warmup": Wm, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic: seeded jittered mesh of the workload, manapy's initial state",
        "config": {"workload": wl.name, "cells": wl.cells, "order": wl.order, "kind": wl.kind,
                   "parallelism": "sharded%d" % world, "halo_cells_rank0": halo,
                   "exchange": "packed halo, NCCL point-to-point per step; dt min all-reduce",
                   "l2": "per-rank working set > 126 MB L2 at 2M cells over <= 8 ranks"},
        "timing": {"repeats": R, "steps_per_repeat": K, "timed_steps": K * R,
                   "ms_per_step_min": min(reps) / K, "ms_per_step_max": max(reps) / K},
        "e2e": {"value": wl.cells * E / e2e_s, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": out.numel() * 8 * world, "steps": E,
                "copies": "each rank reads its owned state back into pinned memory after every step"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak * world, "unit": "GB/s",
                     "frac": achieved / (peak * world), "peak_source": peak_kind, "traffic": None,
                     "kernel": "fused step (2 launches) + halo pack/unpack (2 launches) per rank"},
        "clocks": ck,
        "gpu_launches": 4 * K * R,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    import torch.distributed as dist
    dist.barrier()
    dist.destroy_process_group()


def run_ours(args):
    from manapy_b200 import workloads as W
    wl = W.ALL[args.workload]
    if args.n:
        wl = wl.scaled(n=args.n)
    if wl.kind == "euler":
        return run_euler(args, wl)
    world, rank, local = dist_setup(args)
    if world > 1 and wl.kind == "advdiff" and not args.replicas:
        return run_sharded(args, wl, world, rank, local)
    K = args.steps
    m = measure_workload(wl, args, world, rank, local, K, seed_offset=rank)
    dom, S = m["dom"], m["S"]
    ms_step, value = m["ms_step"], m["value"]

    # end to end through the public API, manapy's driver loop
    E = max(args.e2e_steps, 1)
    if wl.kind == "advdiff":
        e2e_s, h2d, d2h = e2e_advdiff(m, E, world)
    else:
        e2e_s, h2d, d2h = e2e_sw(m, E, world)
    e2e_value = world * wl.cells * E / e2e_s

    line = {
        "metric": "cell-updates/s (FP64 explicit FV step, %s)" % wl.name,
        "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": K, "warmup": m["Wm"],
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic: seeded jittered mesh of the workload, manapy's initial state",
        "config": {"workload": wl.name, "cells": wl.cells, "order": wl.order, "kind": wl.kind,
                   "parallelism": "replicas%d" % world if world > 1 else "single",
                   "l2": "working set %.0f MB > 126 MB L2 (no flush needed)" % (dom.device_mesh.nbytes() / 1e6)},
        "timing": {"repeats": m["R"], "steps_per_repeat": K, "timed_steps": K * m["R"],
                   "ms_per_step_min": min(m["reps"]) / K, "ms_per_step_median": ms_step,
                   "ms_per_step_max": max(m["reps"]) / K},
        "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": E,
                "copies": ("face velocities u, v uploaded from pinned memory; state w and dt read back"
                           if wl.kind == "advdiff" else "state h, hu, hv and dt read back into pinned memory")},
        "roofline": roofline(args.workload, wl.cells, ms_step, m["launches"]),
        "clocks": m["clocks"],
        "gpu_launches": m["launches"] * K * m["R"],
    }
    if "fp32c" in m:
        line["fp32c"] = m["fp32c"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(dom, wl, args.cpu_steps)
    if world == 1 and not args.no_extras and args.workload == "C2" and not args.n:
        import gc
        import torch
        S.release_graphs()
        del m, S, dom
        gc.collect()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        line["extras"] = {name: run_section(name, args) for name in ("c4", "batched", "serving")}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        S.release_graphs()
        dist.destroy_process_group()


def _ref_worker(wk, steps, warmup, start, out):
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
        step = o.step
    elif wl.kind == "euler":
        q = [np.ascontiguousarray(a, dtype=np.float64) for a in wl.init_euler(A["cells_center"], wl.gamma)]

        def step():
            O.euler_step_2d(m, q, wl.cfl, wl.gamma)
    else:
        o = O.ShallowWaterOracle(A, order=wl.order, cfl=wl.cfl, grav=wl.grav, mesh=m)
        for k, a in zip(("h", "hu", "hv", "hc", "Z"), wl.init_sw(A["cells_center"])):
            o.state()[k][:] = a
        step = o.step
    for _ in range(warmup):
        step()
    start.wait()  # every process starts its timed steps together
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    out.put(time.perf_counter() - t0)


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
    # each timed step of every process is one full oracle step; bound the sample to about
    # 2e7 cell-updates per process (10-20 s of serial work)
    steps = max(2, min(args.steps, int(2e7 // wl.cells)))
    warm = 1
    start = ctx.Barrier(procs_n + 1)
    out = ctx.Queue()
    ps = [ctx.Process(target=_ref_worker, args=(args.workload, steps, warm, start, out), daemon=True)
          for _ in range(procs_n)]
    for p in ps:
        p.start()
    start.wait()
    t0 = time.perf_counter()
    times = [out.get() for _ in ps]
    wall = time.perf_counter() - t0
    for p in ps:
        p.join()
    value = procs_n * wl.cells * steps / wall
    line = {
        "metric": ("cell-updates/s (FP64 Euler Rusanov step, %s)" if wl.kind == "euler"
                   else "cell-updates/s (FP64 explicit FV step, %s)") % wl.name, "impl": "reference",
        "value": value, "unit": "cell-updates/s", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": steps, "steps_requested": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * max(times) / steps,
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


def run_serving(args):
    """Seeded request stream through the continuous-batching server (FP32-compensated,
    batched kernels, graph-replayed steps); beside it, serial plain-FP64 solves of a sample
    of the same requests through the public API, one after another."""
    import torch
    import manapy_b200 as M
    from manapy_b200 import serving as SV
    torch.cuda.set_device(0)
    reqs = SV.make_requests(args.requests, args.rate, seed=2024)
    total_cu = sum(r.cells * r.steps for r in reqs)
    srv = SV.BatchServer(workers=args.workers)
    # warm-up outside the timed run: worker processes started, paths exercised
    srv.start_pool()
    srv.serve(SV.make_requests(8, 0.0, seed=1, cells=(2e3, 2e4), steps=(20, 40)))
    t0 = time.perf_counter()
    recs = srv.serve(reqs)
    wall = time.perf_counter() - t0
    srv.stop_pool()
    lat = np.array([r["latency"] for r in recs])
    # serial plain FP64: host preparation excluded (done beforehand), device solve timed per request
    sample = reqs[:max(1, min(args.serial_sample, len(reqs)))]
    service = []
    from manapy_b200 import meshgen
    for r in sample:
        el, vx = meshgen.square_triangles(r.n, seed=r.seed)
        dom = M.Domain(dim=2, mesh=(el, vx))
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        if r.kind == "advdiff":
            w = M.Variable(domain=dom, BC={k: "dirichlet" for k in SV.SIDES}, values={k: 0.0 for k in SV.SIDES})
            u, v = M.Variable(domain=dom), M.Variable(domain=dom)
            u.face = np.full(dom.nbfaces, r.ux)
            v.face = np.full(dom.nbfaces, r.uy)
            u.cell = np.full(dom.nbcells, r.ux)
            v.cell = np.full(dom.nbcells, r.uy)
            w.cell = SV.initial_state(r, dom.cells.center)[0]
            S = M.AdvectionDiffusionSolver(w, vel=(u, v), conf=M.Struct(Dxx=r.D, Dyy=r.D, order=2, cfl=0.8))
            S.advance(r.steps, graph=True)
            _ = w.cell
        else:
            vs = [M.Variable(domain=dom) for _ in range(5)]
            for var, a in zip(vs, SV.initial_state(r, dom.cells.center)):
                var.cell = a
            S = M.ShallowWaterSolver(vs[0], hvel=(vs[1], vs[2]), hc=vs[3], Z=vs[4],
                                     conf=M.Struct(order=1, cfl=0.5, grav=9.81))
            S.advance(r.steps)
            _ = vs[0].cell
        torch.cuda.synchronize()
        service.append(time.perf_counter() - t1)
    service = np.array(service)
    cu_sample = sum(r.cells * r.steps for r in sample)
    serial_rate = cu_sample / service.sum()
    # FIFO single-server queue over the same arrivals with the measured service times
    # (the sample's times, cycled over the stream in order)
    tq, slat = 0.0, []
    for k, r in enumerate(reqs):
        svc = service[k] if k < len(service) else service[k % len(service)] * (
            (r.cells * r.steps) / max(sample[k % len(service)].cells * sample[k % len(service)].steps, 1))
        tq = max(tq, r.arrival) + svc
        slat.append(tq - r.arrival)
    slat = np.array(slat)
    line = {
        "metric": "served p50/p99 latency at sustained throughput (continuous batching, FP32-compensated)",
        "value": total_cu / wall, "unit": "cell-updates/s", "n_gpus": 1, "higher_is_better": True,
        "dtype": "f32 state + compensated sums, f64 geometry and dt", "data": "synthetic seeded request stream",
        "config": {"workload": "C5-serving", "requests": len(reqs), "rate_per_s": args.rate,
                   "cells": "log-uniform 2e3-5e5", "steps": "uniform 100-2000", "mix": "70% adv-diff o2, 30% SW o1"},
        "serving": {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                    "mean_s": float(lat.mean()), "makespan_s": wall, "requests_per_s": len(reqs) / wall,
                    "cell_updates": total_cu, "host_seconds": {k: round(v, 3) for k, v in srv.stats.items()},
                    "workers": srv.workers},
        "serial_fp64": {"value": serial_rate, "unit": "cell-updates/s", "sample": len(sample),
                        "p50_s": float(np.percentile(slat, 50)), "p99_s": float(np.percentile(slat, 99)),
                        "note": "device solves through the public API, one request at a time; host mesh "
                                "preparation excluded; FIFO latencies over the same arrivals"},
    }
    print(json.dumps(line), flush=True)


def _serial_fp64(reqs, steps, warmup=None):
    """Each request's plain FP64 solve through the public API, one after another (CUDA
    graphs, inputs resident); device time of ``steps`` steps per request, summed.  The
    warm-up runs the same number of steps first (default), so that tuning and the graph
    capture happen before the timed steps."""
    import torch
    import manapy_b200 as M
    from manapy_b200 import meshgen, serving as SV
    total = 0.0
    for r in reqs:
        el, vx = meshgen.square_triangles(r.n, seed=r.seed)
        dom = M.Domain(dim=2, mesh=(el, vx))
        if r.kind == "advdiff":
            w = M.Variable(domain=dom, BC={k: "dirichlet" for k in SV.SIDES}, values={k: 0.0 for k in SV.SIDES})
            u, v = M.Variable(domain=dom), M.Variable(domain=dom)
            u.face, v.face = np.full(dom.nbfaces, r.ux), np.full(dom.nbfaces, r.uy)
            u.cell, v.cell = np.full(dom.nbcells, r.ux), np.full(dom.nbcells, r.uy)
            w.cell = SV.initial_state(r, dom.cells.center)[0]
            S = M.AdvectionDiffusionSolver(w, vel=(u, v), conf=M.Struct(Dxx=r.D, Dyy=r.D, order=2, cfl=0.8))
            run = lambda n: S.advance(n, graph=True)  # noqa: E731
        else:
            vs = [M.Variable(domain=dom) for _ in range(5)]
            for var, a in zip(vs, SV.initial_state(r, dom.cells.center)):
                var.cell = a
            S = M.ShallowWaterSolver(vs[0], hvel=(vs[1], vs[2]), hc=vs[3], Z=vs[4],
                                     conf=M.Struct(order=1, cfl=0.5, grav=9.81))
            run = S.advance
        run(steps if warmup is None else warmup)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run(steps)
        e1.record()
        torch.cuda.synchronize()
        total += e0.elapsed_time(e1) / 1e3
    return total


def run_batched(args):
    """A resident batch of uneven meshes (the serving mix's sizes and kinds): batched
    FP32-compensated and batched FP64 kernels against the same meshes solved one after
    another in plain FP64 through the public API; all device-timed over the same steps."""
    import torch
    torch.cuda.set_device(0)
    b = extra_batched(args)
    line = {"metric": "cell-updates/s, batched FP32-compensated vs batched and serial plain FP64 (resident meshes)",
            "value": b["batched_fp32c"], "unit": "cell-updates/s", "n_gpus": 1, "steps": b["steps"],
            "higher_is_better": True, "dtype": "f32 state + compensated sums, f64 geometry and dt",
            "data": "synthetic seeded meshes",
            "config": {"workload": "C5-batched-resident", "meshes": b["meshes"], "cells": b["cells"],
                       "mix": b["mix"], "sizes": b["sizes"]},
            "batched": b}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.section:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(SECTIONS[args.section](args)), flush=True)
        return
    if args.batched:
        run_batched(args)
        return
    if args.serve:
        run_serving(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
