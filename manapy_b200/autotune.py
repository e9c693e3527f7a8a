"""Measured launch-configuration choices.

``graph_depth(solver)``: how many fused steps one CUDA-graph replay of
``AdvectionDiffusionSolver.advance(graph=True)`` holds.  Small meshes are
launch-bound (a step is two short kernels), so deeper graphs pay; large meshes
are bandwidth-bound and any depth is as fast.  The tuner times the candidate
depths on the solver's own mesh (CUDA events, after a warm-up replay), keeps
the fastest, restores the solver's state exactly, and remembers the choice per
scheme and mesh-size class for the rest of the process.
"""
from __future__ import annotations

import math

import torch

__all__ = ["graph_depth", "CANDIDATES", "clear"]

CANDIDATES = (2, 4, 8, 16, 32, 64)
LARGE = 1 << 20          # cells: bandwidth-bound, no tuning (depth 2)
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
