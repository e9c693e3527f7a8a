"""Full-size oracle runs of the large workloads -> compact fixtures ``full_<name>.npz``.

Test infrastructure.  The oracle (``oracle/fv_oracle.c``, the C restatement of
manapy's kernels that ``tests/test_oracle.py`` pins to the reference's own
outputs) runs each configuration at its stated size and length on the host:

* ``C2``: 2,000,000 triangles, order 2 + Barth + diamond diffusion, 1000 steps
  (``manapy/solvers/advecdiff/system.py:149-172``);
* ``C4``: 1,572,864 tetrahedra, order 2 + diffusion, 300 steps;
* ``C3``: 8,000,000 triangles, shallow-water dam break, SRNH order 1, 500 steps
  with a checkpoint after 100 (``manapy/solvers/shallowater/system.py:186-281``).

A full final state is too large to commit (16-192 MB), so each checkpoint keeps
what a size-independent comparison needs:

* ``dts``: every step's dt;
* ``mass``: the FP64 sum of volume x state after every step (h for shallow water);
* per field: L2 norm, Linf norm, plain sum, four projections onto fixed integer-hash
  weight vectors (``weights``: the same on every machine, no RNG stream involved),
  and the values of a seeded sample of cells (``sample_idx``, manapy numbering).

Usage: ``python tests/golden/make_fullsize.py C2 [C3 C4 ...]`` (one process per
workload; C2 takes about 15 minutes on one core, C4 about 8, C3 about 45).
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

NPROJ = 4
SAMPLE = {"C2": 20000, "C4": 16000, "C3": 16000}
CHECKPOINTS = {"C2": (1000,), "C4": (300,), "C3": (100, 500)}


def weights(n, k):
    """Projection weight vector k over n cells: an integer hash of the cell id mapped to
    [-0.5, 0.5) exactly (Knuth's multiplicative hash, 32-bit)."""
    i = np.arange(n, dtype=np.uint64)
    h = ((i + np.uint64(0x9E3779B9 * (k + 1) & 0xFFFFFFFF)) * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)
    return h.astype(np.float64) / 4294967296.0 - 0.5


def summary(a, sample_idx):
    a = np.asarray(a, dtype=np.float64)
    n = len(a)
    return {
        "l2": float(np.sqrt(np.dot(a, a))),
        "linf": float(np.max(np.abs(a))),
        "sum": float(np.sum(a)),
        "proj": np.array([float(np.dot(weights(n, k), a)) for k in range(NPROJ)]),
        "projabs": np.array([float(np.dot(np.abs(weights(n, k)), np.abs(a))) for k in range(NPROJ)]),
        "sample": a[sample_idx].copy(),
    }


def sample_indices(n, k, seed):
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n, size=min(k, n), replace=False)).astype(np.int32)


def run_advdiff(name, wl):
    from manapy_b200 import boundary as B
    from manapy_b200.domain import build_host_mesh
    import oracle as O
    t0 = time.time()
    el, vx = wl.mesh()
    A, _ = build_host_mesh(el, vx, wl.dim)
    print(name, "mesh", len(el), "cells, built in %.1f s" % (time.time() - t0), flush=True)
    o = O.AdvDiffOracle(A, B.resolve(A, wl.bc, wl.bc_values), *wl.diffusion, order=wl.order, cfl=wl.cfl)
    o.set_velocity(*wl.velocity(A["faces_center"]))
    o.w[:] = wl.init(A["cells_center"])
    vol = np.asarray(A["cells_volume"], dtype=np.float64)
    sidx = sample_indices(o.m.nc, SAMPLE[name], 2024)
    out = {"nbcells": o.m.nc, "sample_idx": sidx, "mass0": float(np.dot(vol, o.w))}
    dts, mass = [], []
    t0 = time.time()
    for it in range(1, wl.steps + 1):
        dts.append(o.step())
        mass.append(float(np.dot(vol, o.w)))
        if it in CHECKPOINTS[name]:
            s = summary(o.w, sidx)
            for k, v in s.items():
                out["s%d_w_%s" % (it, k)] = v
        if it % 50 == 0:
            print(name, "step", it, "%.1f s" % (time.time() - t0), flush=True)
    out["dts"] = np.array(dts)
    out["mass"] = np.array(mass)
    out["oracle_seconds"] = time.time() - t0
    return out


def run_sw(name, wl):
    from manapy_b200.domain import build_host_mesh
    import oracle as O
    t0 = time.time()
    el, vx = wl.mesh()
    A, _ = build_host_mesh(el, vx, 2)
    print(name, "mesh", len(el), "cells, built in %.1f s" % (time.time() - t0), flush=True)
    so = O.ShallowWaterOracle(A, order=wl.order, cfl=wl.cfl, grav=wl.grav)
    for k, a in zip(("h", "hu", "hv", "hc", "Z"), wl.init_sw(A["cells_center"])):
        so.state()[k][:] = a
    vol = np.asarray(A["cells_volume"], dtype=np.float64)
    sidx = sample_indices(so.m.nc, SAMPLE[name], 2025)
    out = {"nbcells": so.m.nc, "sample_idx": sidx, "mass0": float(np.dot(vol, so.h))}
    dts, mass = [], []
    t0 = time.time()
    for it in range(1, wl.steps + 1):
        dts.append(so.step())
        mass.append(float(np.dot(vol, so.h)))
        if it in CHECKPOINTS[name]:
            for f in ("h", "hu", "hv"):
                for k, v in summary(so.state()[f], sidx).items():
                    out["s%d_%s_%s" % (it, f, k)] = v
        if it % 10 == 0:
            print(name, "step", it, "%.1f s" % (time.time() - t0), flush=True)
    out["dts"] = np.array(dts)
    out["mass"] = np.array(mass)
    out["oracle_seconds"] = time.time() - t0
    return out


def main(names):
    from manapy_b200 import workloads as W
    for name in names:
        wl = W.ALL[name]
        out = run_sw(name, wl) if wl.kind == "sw" else run_advdiff(name, wl)
        out["checkpoints"] = np.array(CHECKPOINTS[name])
        path = os.path.join(HERE, "full_%s.npz" % name.lower())
        np.savez_compressed(path, **out)
        print("wrote", path, "(%.1f s of oracle steps)" % out["oracle_seconds"], flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or ["C2", "C4", "C3"])
