"""Checkpoint and resume of a solver's state (no counterpart in manapy, whose runs restart
from the initial condition).

``save(path, solver, step=0, time=0.0)`` writes one ``.npz`` with the solver's state in
manapy's numbering: the cell fields it advances, the fields its step reads (velocities
of an advection-diffusion solver, the bed of a shallow-water solver), and, in the
FP32-compensated precision, the FP32 state and its rounding errors exactly as the
device holds them.  ``load(path, solver)`` puts that state back into a solver built on
the same mesh with the same options and returns ``(step, time)``; the run then continues
bit for bit as if it had not stopped (the dt of the restored state is recomputed with
the same operations).
"""
from __future__ import annotations

import numpy as np
import torch

__all__ = ["save", "load"]

FORMAT = 1


def _kind(solver):
    from .solvers import AdvectionDiffusionSolver, ShallowWaterSolver
    if isinstance(solver, ShallowWaterSolver):
        return "shallow_water"
    if isinstance(solver, AdvectionDiffusionSolver):
        return "advection_diffusion"
    raise TypeError("checkpoints cover AdvectionDiffusionSolver (and its subclasses) and ShallowWaterSolver")


def _read(var, name):
    """A variable's array in manapy's numbering, read without handing authority to the
    host (the device array stays the one the solver steps)."""
    out = var.fetch(name)
    torch.cuda.synchronize()
    return out.numpy().copy()


def _host_cells(solver, t):
    """A device cell tensor (device numbering) in manapy's numbering, on the host."""
    dm = solver._dm
    return dm.to_host_order("cell", t).cpu().numpy()


def _dev_cells(solver, a, dtype):
    dm = solver._dm
    src = torch.from_numpy(np.ascontiguousarray(a)).to(dm.device)
    out = torch.empty(len(a), dtype=dtype, device=dm.device)
    dm.to_device_order("cell", src, out)
    return out


def save(path, solver, step=0, time=0.0):
    kind = _kind(solver)
    solver._setup()
    out = {"format": FORMAT, "kind": kind, "precision": solver.precision, "step": int(step), "time": float(time),
           "nbcells": int(solver.domain.nbcells), "dim": int(solver.dim)}
    if kind == "advection_diffusion":
        out["cell"] = _read(solver.var, "cell")
        for name, var in (("u", solver.u), ("v", solver.v), ("w", solver.w)):
            out[name + "_face"] = _read(var, "face")
            out[name + "_cell"] = _read(var, "cell")
        if solver.precision == "fp32c" and solver._w32 is not None and \
                solver.var.version("cell") == solver._w32_key:
            k = solver._w32_i
            out["state32"] = _host_cells(solver, solver._w32[k])
            out["lo32"] = _host_cells(solver, solver._lo32[k])
    else:
        for name in ("h", "hu", "hv", "hc", "Z"):
            out[name] = _read(solver.varbs[name], "cell")
        if solver._dt_key is not None and solver._dt_key == solver._state_key():
            # the dt the next step applies (in the FP32-compensated step it comes from the FP32
            # state, so it is carried rather than recomputed)
            out["dt"] = float(solver._dt_buf[solver._cur].item())
        if solver.precision == "fp32c" and solver._q32 is not None and solver._keys() == solver._q32_key:
            k = solver._q32_i
            for c, name in enumerate(("h", "hu", "hv", "hc")):
                out[name + "32"] = _host_cells(solver, solver._q32[k][c])
                out[name + "_lo32"] = _host_cells(solver, solver._lo32[k][c])
            out["Z32"] = _host_cells(solver, solver._q32[2])
    np.savez(path, **out)


def load(path, solver):
    kind = _kind(solver)
    g = np.load(path)
    if int(g["format"]) != FORMAT or str(g["kind"]) != kind:
        raise ValueError("%s is not a %s checkpoint of this format" % (path, kind))
    if int(g["nbcells"]) != int(solver.domain.nbcells) or int(g["dim"]) != int(solver.dim):
        raise ValueError("the checkpoint was written for another mesh")
    if str(g["precision"]) != solver.precision:
        raise ValueError("the checkpoint holds a %s state; the solver runs %s" % (g["precision"], solver.precision))
    solver._setup()
    if kind == "advection_diffusion":
        for name, var in (("u", solver.u), ("v", solver.v), ("w", solver.w)):
            var.face = g[name + "_face"]
            var.cell = g[name + "_cell"]
        solver.var.cell = g["cell"]
        if "state32" in g.files:
            solver._f32_state()                       # buffers allocated, keyed to the new cell array
            k = solver._w32_i
            solver._w32[k].copy_(_dev_cells(solver, g["state32"], torch.float32))
            solver._lo32[k].copy_(_dev_cells(solver, g["lo32"], torch.float32))
    else:
        for name in ("h", "hu", "hv", "hc", "Z"):
            solver.varbs[name].cell = g[name]
        if "h32" in g.files:
            qk, _ = solver._f32_state()
            k = solver._q32_i
            for c, name in enumerate(("h", "hu", "hv", "hc")):
                solver._q32[k][c].copy_(_dev_cells(solver, g[name + "32"], torch.float32))
                solver._lo32[k][c].copy_(_dev_cells(solver, g[name + "_lo32"], torch.float32))
            solver._q32[2].copy_(_dev_cells(solver, g["Z32"], torch.float32))
        if "dt" in g.files:
            solver._dt_buf[solver._cur].fill_(float(g["dt"]))
            solver._dt_key = solver._state_key()
            solver._dt_host = None
    return int(g["step"]), float(g["time"])
