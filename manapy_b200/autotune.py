"""Measured launch-configuration choices.

``graph_depth(solver)``: how many fused steps one CUDA-graph replay of
``AdvectionDiffusionSolver.advance(graph=True)`` holds.  Small meshes are
launch-bound (a step is two short kernels), so deeper graphs pay; large meshes
are bandwidth-bound and any depth is as fast.

``launch_variant(solver)``: the launch shape (threads per block and resident blocks
per SM, four pre-built instantiations of each) of the two fused phases of the FP64
second-order step with diffusion, chosen per phase: the first phase's variant with
the second at its default, then the second phase's.

Both tuners time the candidates on the solver's own mesh (CUDA events, after a
warm-up replay), keep the fastest, restore the solver's state exactly, and remember
the choice per scheme and mesh-size class for the rest of the process.  Variants
compute the same operations; the compiler may contract multiply-adds differently
in each, so results differ between variants by rounding only.
"""
from __future__ import annotations

import math

import torch

__all__ = ["graph_depth", "launch_variant", "CANDIDATES", "VARIANTS", "clear"]

CANDIDATES = (2, 4, 8, 16, 32, 64)
LARGE = 1 << 20          # cells: bandwidth-bound, no tuning (depth 2)
VARIANTS = (0, 1, 2, 3)
SMALL = 1 << 16          # cells: launch-bound, launch shapes not tuned
_cache = {}


def clear():
    _cache.clear()


def _key(s):
    return (s.precision, int(s.dim), int(s.order), bool(s.diffusion),
            int(round(math.log2(max(int(s._dm.nbcells), 1)))))


def graph_depth(solver, candidates=CANDIDATES, steps=128):
    """The fastest graph depth for ``solver``'s mesh and scheme (see the module doc)."""
    s = solver
    s._setup()
    if s._dm.nbcells >= LARGE:
        return 2
    k = _key(s)
    if k in _cache:
        return _cache[k]
    var = s.var
    saved = var.dev("cell").clone()
    times = {}
    try:
        for d in candidates:
            s.graph_depth = d
            s.release_graphs()
            s.advance(d, graph=True)                       # capture + warm-up replay
            reps = max(1, steps // d)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            s.advance(reps * d, graph=True)
            e1.record()
            e1.synchronize()
            times[d] = e0.elapsed_time(e1) / (reps * d)
    finally:
        s.release_graphs()
        var._s.w("cell").copy_(saved)                      # the state before tuning, exactly
    best = min(times, key=times.get)
    _cache[k] = best
    return best


def _time_steps(s, steps):
    s.advance(2, graph=True)                               # capture + warm-up replay
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    s.advance(steps, graph=True)
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def launch_variant(solver, steps=64):
    """The fastest launch-shape variant (``mb_mesh.variant``: bits 0-1 first phase, 2-3
    second) for ``solver``'s mesh and scheme; 0 where there is nothing to tune."""
    s = solver
    s._setup()
    dm = s._dm
    if not (s.precision == "fp64" and s.order == 2 and s.diffusion and "cell_vtx" in dm.t) or \
            dm.nbcells < SMALL:
        return 0
    k = ("variant",) + _key(s)
    if k in _cache:
        return _cache[k]
    var = s.var
    saved = var.dev("cell").clone()
    try:
        def run(v):
            dm.struct.variant = v
            s.release_graphs()
            return _time_steps(s, steps)
        t1 = {v: run(v) for v in VARIANTS}                  # first phase, second at default
        b1 = min(t1, key=t1.get)
        t2 = {v: run(b1 | (v << 2)) for v in VARIANTS}      # second phase
        best = b1 | (min(t2, key=t2.get) << 2)
    finally:
        s.release_graphs()
        var._s.w("cell").copy_(saved)                      # the state before tuning, exactly
    dm.struct.variant = best
    dm.variant = best
    _cache[k] = best
    return best
