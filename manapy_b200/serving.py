"""Continuous-batching server for explicit finite-volume solves (no counterpart in manapy).

Each request is a whole solve on its own mesh: an advection-diffusion run (second
order, Barth limiter, diamond diffusion, Dirichlet 0 boundaries) or a
shallow-water dam break (first order, Neumann walls), for a given number of
steps, in the FP32-compensated precision.  The server keeps every admitted
request's mesh tables and fields resident on the GPU and advances all of them
together: per step, one batched launch pair per family (the block -> mesh maps
of ``mb_advdiff_batch_step_f32c`` / ``mb_sw_batch_step_f32c``) over all active
meshes, so requests of very different sizes share the device.  Requests that
arrive while others run are admitted between steps, as soon as a slot and the
HBM budget allow; finished ones retire between steps and free their memory.

Mesh preparation (generation, geometry, locality numbering, compact tables) is
host work; it runs in a pool of worker processes that overlaps the GPU.  The
step loop is replayed from CUDA graphs, re-captured whenever the set of active
requests changes.

Results are independent of the mix: every request computes exactly what its
own solve computes alone (no cross-request sums; each dt reduction is an exact
min over the request's own cells), so a request's result is bit-for-bit the same
alone and in any batch.
"""
from __future__ import annotations

import concurrent.futures as cf
import dataclasses
import functools
import math
import multiprocessing as mp
import os
import pickle
import queue
import tempfile
import threading
import time

import numpy as np
import torch

from . import _lib

__all__ = ["Request", "make_requests", "prepare", "BatchServer"]


@dataclasses.dataclass
class Request:
    rid: int
    kind: str            # "advdiff" or "sw"
    n: int               # mesh: n x n squares, 2 n^2 triangles
    seed: int
    steps: int
    arrival: float = 0.0  # seconds after the start of the run
    ux: float = 0.0
    uy: float = 0.0
    D: float = 0.0
    ratio: float = 2.0    # dam-break height ratio (left / right)
    prep_window: tuple = None  # (start, end) of its preparation, time.perf_counter() of the worker

    @property
    def cells(self):
        return 2 * self.n * self.n


def make_requests(count, rate, seed=0, cells=(2e3, 5e5), frac_advdiff=0.7, steps=(100, 2000)):
    """Seeded request stream: Poisson arrivals at ``rate`` per second, mesh sizes
    log-uniform in ``cells``, 70 % advection-diffusion (speed U[0.2, 1.5], random
    direction, D log-uniform in [1e-4, 1e-2]), 30 % dam breaks (height ratio U[1.2, 3]),
    steps uniform in ``steps``."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=count)) if rate > 0 else np.zeros(count)
    out = []
    for k in range(count):
        nc = math.exp(rng.uniform(math.log(cells[0]), math.log(cells[1])))
        n = max(2, int(round(math.sqrt(nc / 2))))
        kind = "advdiff" if rng.uniform() < frac_advdiff else "sw"
        st = int(rng.integers(steps[0], steps[1] + 1))
        r = Request(rid=k, kind=kind, n=n, seed=int(rng.integers(1 << 30)), steps=st, arrival=float(t[k]))
        if kind == "advdiff":
            sp, th = rng.uniform(0.2, 1.5), rng.uniform(0, 2 * math.pi)
            r.ux, r.uy = sp * math.cos(th), sp * math.sin(th)
            r.D = math.exp(rng.uniform(math.log(1e-4), math.log(1e-2)))
        else:
            r.ratio = rng.uniform(1.2, 3.0)
        out.append(r)
    return out


# ------------------------------------------------------------------ host preparation

SIDES = ("in", "out", "upper", "bottom")


def initial_state(req, centers):
    """Initial cell fields (device numbering is applied by the caller)."""
    x, y = centers[:, 0], centers[:, 1]
    if req.kind == "advdiff":
        return [np.exp(-((x - 0.5) ** 2 + (y - 0.5) ** 2) / 0.01)]
    h = np.where(x < 0.5, req.ratio, 1.0)
    Z = 0.1 * np.exp(-((x - 0.7) ** 2 + (y - 0.5) ** 2) / 0.02)
    zero = np.zeros_like(x)
    return [h, zero, zero.copy(), zero.copy(), Z]


# tables the FP64 batched steps read beyond the FP32-compensated ones (the FP64
# centre -> vertex weights)
FP64_EXTRA_TABLES = ("n2c_sell_alpha",)

# mesh tables each batched step dereferences, checked on the host before an item table
# goes to the device (the kernels cannot check pointers that live in device memory)
_NEEDS = {
    ("advdiff", "fp32c"): ("cell_volume", "cell_order", "cell_vtx", "cell_nbr", "cell_flags", "node_coord", "cell_xy",
                           "lsq_sell_ptr", "lsq_sell_idx", "n2c_sell_ptr", "n2c_sell_idx", "n2c_sell_alpha_f32",
                           "ghostnid_ptr", "ghostnid_idx", "face_ghostcenter", "n2g_ptr", "n2g_idx", "n2g_alpha",
                           "face_cellid", "face_dist"),
    ("advdiff", "fp64"): ("cell_volume", "cell_order", "cell_vtx", "cell_nbr", "cell_flags", "node_coord", "cell_xy",
                          "lsq_sell_ptr", "lsq_sell_idx", "n2c_sell_ptr", "n2c_sell_idx", "n2c_sell_alpha",
                          "ghostnid_ptr", "ghostnid_idx", "face_ghostcenter", "n2g_ptr", "n2g_idx", "n2g_alpha",
                          "face_cellid", "face_dist"),
    ("sw", "fp32c"): ("cell_volume", "cell_order", "cell_faces", "cell_vtx", "cell_nbr", "cell_flags", "node_coord",
                      "cell_xy", "cell_cellfid", "face_cellid", "face_nm_f32"),
    ("sw", "fp64"): ("cell_volume", "cell_order", "cell_faces", "cell_vtx", "cell_nbr", "cell_flags", "node_coord",
                     "cell_xy", "cell_cellfid", "face_cellid", "face_normal", "face_mesure"),
}


def check_item_tables(kind, precision, mesh_struct):
    """Raise ValueError if a table the batched step of (kind, precision) reads is missing
    from the mesh struct (a NULL pointer)."""
    missing = [n for n in _NEEDS[(kind, precision)] if not getattr(mesh_struct, n)]
    if missing:
        raise ValueError("mesh tables missing for the %s %s batched step: %s" % (precision, kind, ", ".join(missing)))


def prepare(req, precision="fp32c"):
    """Host work of one request (runs in a worker process): mesh, geometry, device tables
    (as host arrays), boundary rules and the initial state in the device numbering."""
    from . import boundary as B, meshgen
    from .device import DeviceBC, DeviceMesh
    t_start = time.perf_counter()
    el, vx = meshgen.square_triangles(req.n, seed=req.seed)
    dm = DeviceMesh.from_native(el, vx)       # the native host builder (C++)
    A = dm.A
    dm.keep_only(DeviceMesh.SERVE_TABLES + (FP64_EXTRA_TABLES if precision == "fp64" else ()))
    bc = None
    if req.kind == "advdiff":
        res = B.resolve(A, {s: "dirichlet" for s in SIDES}, {s: 0.0 for s in SIDES})
        bc = DeviceBC(A, res, device=None, mesh=dm)
        bc.resolved = None
    init = [a[dm.R.cperm] for a in initial_state(req, A["cells_center"])]
    dm.strip()
    req = dataclasses.replace(req, prep_window=(t_start, time.perf_counter()))
    return req, dm, bc, init


# Prepared requests cross from the workers in shared memory: the pickle stream of the
# (req, mesh, bc, init) tuple keeps only a header of each numpy array (protocol 5, buffers
# out of band), the buffers go to one file on a tmpfs, and the serving process reads the file
# back in one read.  Through the pool's result pipe a 500k-cell mesh's ~200 MB took about a
# quarter of a second and held up every other result behind it.
_SHM_DIR = "/dev/shm"
_ALIGN = 64


@dataclasses.dataclass
class _Shipped:
    path: str
    head: bytes
    sizes: list


def _ship(obj):
    """Worker side: ``obj`` with its array buffers moved to a file in shared memory, or
    ``obj`` itself when no tmpfs with room for them is there."""
    bufs = []
    head = pickle.dumps(obj, protocol=5, buffer_callback=bufs.append)
    raws = [b.raw() for b in bufs]
    sizes = [r.nbytes for r in raws]
    total = sum(-(-n // _ALIGN) * _ALIGN for n in sizes)
    path = None
    try:
        st = os.statvfs(_SHM_DIR)
        if st.f_bavail * st.f_frsize < 2 * total + (256 << 20):
            return obj
        fd, path = tempfile.mkstemp(prefix="manapy_b200_prep_", dir=_SHM_DIR)
        with os.fdopen(fd, "wb") as f:
            for r in raws:
                f.write(r)
                pad = -r.nbytes % _ALIGN
                if pad:
                    f.write(bytes(pad))
    except OSError:
        if path is not None and os.path.exists(path):
            os.unlink(path)
        return obj
    return _Shipped(path, head, sizes)


def _receive(x):
    """Serving side of ``_ship``: the object rebuilt on one read of its buffer file (the
    arrays are views of that read, each 64-byte aligned), the file removed."""
    if not isinstance(x, _Shipped):
        return x
    total = sum(-(-n // _ALIGN) * _ALIGN for n in x.sizes)
    raw = np.empty(total + _ALIGN, dtype=np.uint8)
    start = -raw.ctypes.data % _ALIGN
    data = raw[start:start + total]
    try:
        with open(x.path, "rb", buffering=0) as f:
            got = f.readinto(memoryview(data))
    finally:
        os.unlink(x.path)
    if got != total:
        raise RuntimeError("prepared request %s: short read (%d of %d bytes)" % (x.path, got, total))
    views, off = [], 0
    for n in x.sizes:
        views.append(memoryview(data[off:off + n]))
        off += -(-n // _ALIGN) * _ALIGN
    return pickle.loads(x.head, buffers=views)


def _discard(fut):
    """Done-callback of a preparation nobody will admit: its shared-memory file removed."""
    try:
        _receive(fut.result())
    except BaseException:  # a failed or cancelled preparation left no file
        pass


def prepare_shipped(req, precision="fp32c", host_threads=None):
    """``prepare`` in a worker process (its native builder on ``host_threads`` threads when
    given), its result handed back through shared memory."""
    if host_threads is not None:
        os.environ["MANAPY_B200_HOST_THREADS"] = str(max(1, int(host_threads)))
    return _ship(prepare(req, precision))


def admission_order(waiting, used, budget, slots, active, now, max_skip_wait=1.0):
    """Which prepared requests to admit now, as indices into ``waiting`` in the order to admit
    them.  ``waiting``: (ready time, estimated device bytes) of the prepared requests in
    arrival order; ``used``: bytes the admitted requests hold; ``slots``: free slots;
    ``active``: admitted requests.  Arrival order, except that a request that does not fit
    in the budget lets later ones that fit pass it until it has been ready for
    ``max_skip_wait`` seconds; from then on nothing passes it (0: strict arrival order).
    With nothing admitted, the first request goes in even if it alone exceeds the budget."""
    out = []
    for k, (ready, est) in enumerate(waiting):
        if len(out) >= slots:
            break
        if used + est <= budget or (active == 0 and not out):
            out.append(k)
            used += est
        elif now - ready >= max_skip_wait:
            break
    return out


def _init_worker(host_threads):
    """Worker initialiser: the thread count of the native builder in this process."""
    os.environ["MANAPY_B200_HOST_THREADS"] = str(int(host_threads))


def _warm(_):
    """Worker start-up: load the modules and the native builder."""
    from . import device, meshgen, native  # noqa: F401
    native.lib()
    return os.getpid()


# ------------------------------------------------------------------ device side

def _p(t):
    return t.data_ptr() if t is not None else None


class _Slot:
    """One admitted request: its device tables, fields and batch item."""

    def __init__(self, req, dm, bc, init, dev, stream, staging, stats=None, precision="fp32c"):
        stats = stats if stats is not None else {}
        self.precision = precision
        t0 = time.perf_counter()
        self.req = req
        extra = {"init%d" % k: np.ascontiguousarray(a, dtype=np.float64) for k, a in enumerate(init)}
        if bc is not None:
            extra.update(bc_kind=bc.kind, bc_value=bc.value, bc_grad=bc.face_grad_on)
        views = dm.upload_staged(dev, stream, staging, extra)   # tables, rules and state: one copy
        self.dm = dm
        t1 = time.perf_counter()
        if bc is not None:
            bc.kind, bc.value, bc.face_grad_on = views["bc_kind"], views["bc_value"], views["bc_grad"]
            bc.struct = bc._make_struct()
        self.bc = bc
        t2 = time.perf_counter()
        stats["admit_tables"] = stats.get("admit_tables", 0.0) + t1 - t0
        stats["admit_bc"] = stats.get("admit_bc", 0.0) + t2 - t1
        nc, nf = dm.nbcells, dm.nbfaces
        f32 = torch.float32
        f64 = torch.float64
        with torch.cuda.stream(stream):
            up = [views["init%d" % k] for k in range(len(init))]
            if precision == "fp64":
                self._setup_fp64(req, up, dev, stream, nc, nf, f64)
            elif req.kind == "advdiff":
                self.w = [up[0].float(), torch.empty(nc, dtype=f32, device=dev)]
                self.lo = [(up[0] - self.w[0].double()).float(), torch.empty(nc, dtype=f32, device=dev)]
                uf = torch.full((nf,), req.ux, dtype=torch.float64, device=dev)
                vf = torch.full((nf,), req.uy, dtype=torch.float64, device=dev)
                zf = torch.zeros(nf, dtype=torch.float64, device=dev)
                sign = torch.empty(4 * nc, dtype=torch.float64, device=dev)
                st = stream.cuda_stream
                _lib.call("mb_cell_face_sign", self.dm.struct, _p(uf), _p(vf), _p(zf), _p(sign), st)
                self.sign = torch.empty(4 * nc, dtype=f32, device=dev)
                _lib.call("mb_cell_face_sign_f32c", self.dm.struct, _p(sign), _p(self.sign), st)
                uc = torch.full((nc,), req.ux, dtype=torch.float64, device=dev)
                vc = torch.full((nc,), req.uy, dtype=torch.float64, device=dev)
                zc = torch.zeros(nc, dtype=torch.float64, device=dev)
                self.dt = torch.empty(1, dtype=torch.float64, device=dev)
                _lib.call("mb_time_step", self.dm.struct, _p(uc), _p(vc), _p(zc), 0.8, req.D, req.D, 0.0,
                          _p(self.dt), st)
                self.cs = torch.empty(4 * nc, dtype=f32, device=dev)
                self.ns = torch.empty(dm.nbnodes, dtype=f32, device=dev)
                self.params = _lib.MbAdvDiffParams(2, 1, req.D, req.D, 0.0)
            else:
                q = [up[k].float() for k in range(4)]
                self.q = [q, [torch.empty(nc, dtype=f32, device=dev) for _ in range(4)]]
                self.lo = [[(up[k] - q[k].double()).float() for k in range(4)],
                           [torch.empty(nc, dtype=f32, device=dev) for _ in range(4)]]
                self.Z = up[4].float()
                self.ff = torch.empty(4 * nf, dtype=f32, device=dev)
                self.dt = torch.empty(2, dtype=torch.float64, device=dev)
                _lib.call("mb_time_step_sw", self.dm.struct, _p(up[0]), _p(up[1]), _p(up[2]), 0.5, 9.81, 0.0, 0.0,
                          _p(self.dt), stream.cuda_stream)
            self.ready = torch.cuda.Event()
            self.ready.record(stream)
        stats["admit_setup"] = stats.get("admit_setup", 0.0) + time.perf_counter() - t2
        self._keep = up  # the uploads stay alive until the copies have run
        self.start = self.end = None
        self.fam = None
        self.nbytes = self.dm.nbytes() + sum(t.numel() * t.element_size() for t in self._tensors())

    def _setup_fp64(self, req, up, dev, stream, nc, nf, f64):
        """Plain FP64 buffers of the request (the batched FP64 steps)."""
        st = stream.cuda_stream
        if req.kind == "advdiff":
            self.w = [up[0].clone(), torch.empty(nc, dtype=f64, device=dev)]
            self.lo = []
            uf = torch.full((nf,), req.ux, dtype=f64, device=dev)
            vf = torch.full((nf,), req.uy, dtype=f64, device=dev)
            zf = torch.zeros(nf, dtype=f64, device=dev)
            self.sign = torch.empty(4 * nc, dtype=f64, device=dev)
            _lib.call("mb_cell_face_sign", self.dm.struct, _p(uf), _p(vf), _p(zf), _p(self.sign), st)
            uc = torch.full((nc,), req.ux, dtype=f64, device=dev)
            vc = torch.full((nc,), req.uy, dtype=f64, device=dev)
            zc = torch.zeros(nc, dtype=f64, device=dev)
            self.dt = torch.empty(1, dtype=f64, device=dev)
            _lib.call("mb_time_step", self.dm.struct, _p(uc), _p(vc), _p(zc), 0.8, req.D, req.D, 0.0, _p(self.dt), st)
            self.cs = torch.empty(4 * nc, dtype=f64, device=dev)
            self.ns = torch.empty(self.dm.nbnodes, dtype=f64, device=dev)
            self.params = _lib.MbAdvDiffParams(2, 1, req.D, req.D, 0.0)
        else:
            q = [up[k].clone() for k in range(4)]
            self.q = [q, [torch.empty(nc, dtype=f64, device=dev) for _ in range(4)]]
            self.lo = [[], []]
            self.Z = up[4].clone()
            self.ff = torch.empty(4 * nf, dtype=f64, device=dev)
            self.dt = torch.empty(2, dtype=f64, device=dev)
            _lib.call("mb_time_step_sw", self.dm.struct, _p(q[0]), _p(q[1]), _p(q[2]), 0.5, 9.81, 0.0, 0.0,
                      _p(self.dt), st)

    def _tensors(self):
        if self.req.kind == "advdiff":
            return self.w + self.lo + [self.sign, self.dt, self.cs, self.ns]
        return self.q[0] + self.q[1] + self.lo[0] + self.lo[1] + [self.Z, self.ff, self.dt]

    def blocks(self):
        nc = self.dm.nbcells
        cb = -(-nc // 256)
        if self.req.kind == "advdiff":
            return cb + -(-self.dm.nbnodes // 256), cb, cb   # phase-1 blocks, of which cells, phase-2
        return -(-self.dm.nbfaces // 256), cb              # face blocks, cell blocks

    def result(self):
        """Final state (device tensors, device numbering): [w] or [h, hu, hv]."""
        par = (self.end - self.start) & 1
        if self.precision == "fp64":
            if self.req.kind == "advdiff":
                return [self.w[par].clone()]
            return [self.q[par][c].clone() for c in range(3)]
        if self.req.kind == "advdiff":
            return [self.w[par].double() + self.lo[par].double()]
        return [self.q[par][c].double() + self.lo[par][c].double() for c in range(3)]


class BatchServer:
    """Continuous-batching server on one GPU.

    ``hbm_budget``: bytes of device memory the admitted requests may hold;
    ``max_active``: slots; ``chunk``: steps per graph replay between admission points;
    ``workers``: host processes preparing meshes (0: prepare in this process);
    ``precision``: "fp32c" (FP32 state with compensated sums, the serving default) or "fp64"
    (manapy's plain arithmetic, each result bit-identical to the single-mesh FP64 solver);
    ``host_threads``: native-builder threads per worker; default: with ``poll``, the host cores
    shared among the preparations in flight when a request is handed over (one when many
    are), else host cores / workers;
    ``max_skip_wait``: seconds a prepared request that does not fit in the HBM budget lets
    later ones that fit pass it (``admission_order``; 0: strict arrival order);
    ``poll``: a dispatcher thread hands each request to the workers at its arrival, and the
    serving loop polls the device while two chunks are queued instead of blocking on the
    older one, so that meshes prepared meanwhile are admitted at once (False: requests are
    handed over and admitted only between chunks).
    """

    def __init__(self, device="cuda:0", hbm_budget=40e9, max_active=256, chunk=16, workers=None,
                 graphs=True, precision="fp32c", host_threads=None, poll=True, max_skip_wait=1.0):
        if precision not in ("fp32c", "fp64"):
            raise ValueError("precision must be 'fp32c' or 'fp64'")
        self.precision = precision
        self.dev = torch.device(device)
        self.budget = float(hbm_budget)
        self.max_active = int(max_active)
        self.chunk = int(chunk)
        self.graphs = bool(graphs)
        self.poll = bool(poll)
        self.max_skip_wait = float(max_skip_wait)
        self.workers = (os.cpu_count() or 1) if workers is None else int(workers)
        # native-builder threads per preparation process: the host cores shared out
        self.cores = os.cpu_count() or 1
        self.adaptive_threads = host_threads is None
        self.host_threads = (max(1, self.cores // max(1, self.workers)) if host_threads is None
                             else int(host_threads))
        self.stream = torch.cuda.Stream(device=self.dev)
        self.upload_stream = torch.cuda.Stream(device=self.dev)
        # one step counter per family: [advection-diffusion, shallow water]
        self.clock = torch.zeros(2, dtype=torch.int32, device=self.dev)
        self.clock_host = [0, 0]
        self.active = {}
        self._graph = None
        self._tables = None
        self._old = []
        self._staging = None
        self._staging_ev = None
        self.pool = None
        self.stats = {}

    def start_pool(self):
        """Start the mesh-preparation worker processes (and load their modules) ahead of a run."""
        if self.workers > 0 and self.pool is None:
            self.pool = cf.ProcessPoolExecutor(max_workers=self.workers, mp_context=mp.get_context("spawn"),
                                               initializer=_init_worker, initargs=(self.host_threads,))
            list(self.pool.map(_warm, range(self.workers)))
        return self

    def stop_pool(self):
        if self.pool is not None:
            self.pool.shutdown(cancel_futures=True)
            self.pool = None

    def _stage(self, nbytes):
        """The pinned staging buffer of mesh uploads, free for reuse (its last copy has run)."""
        if self._staging_ev is not None:
            self._staging_ev.synchronize()
        if self._staging is None or self._staging.numel() < nbytes:
            self._staging = torch.empty(int(nbytes * 1.25) + (1 << 20), dtype=torch.uint8, pin_memory=True)
        return self._staging

    def _admit(self, req, dm, bc, init):
        from .device import staged_nbytes
        need = staged_nbytes(dm.t) + sum(int(np.asarray(a).nbytes) + 512 for a in init) + (
            0 if bc is None else staged_nbytes({"k": bc.kind, "v": bc.value, "g": bc.face_grad_on}))
        t0 = time.perf_counter()
        staging = self._stage(need)
        self.stats["admit_stage_wait"] = self.stats.get("admit_stage_wait", 0.0) + time.perf_counter() - t0
        slot = _Slot(req, dm, bc, init, self.dev, self.upload_stream, staging, self.stats, self.precision)
        self._staging_ev = torch.cuda.Event()
        self._staging_ev.record(self.upload_stream)
        self.stream.wait_event(slot.ready)
        return slot

    # -------------------------------------------------------------- batch tables
    def _build_tables(self):
        """Item arrays and block maps of the active slots, uploaded on the compute stream."""
        ad = [s for s in self.active.values() if s.req.kind == "advdiff"]
        sw = [s for s in self.active.values() if s.req.kind == "sw"]
        tabs = {}
        fp64 = self.precision == "fp64"
        with torch.cuda.stream(self.stream):
            if ad:
                items = ((_lib.MbAdvDiffItemF64 if fp64 else _lib.MbAdvDiffItem) * len(ad))()
                p1, p2 = [], []
                b1 = b2 = 0
                for k, s in enumerate(ad):
                    n1, ncb, n2 = s.blocks()
                    it = items[k]
                    check_item_tables("advdiff", self.precision, s.dm.struct)
                    it.m, it.bc, it.p = s.dm.struct, s.bc.struct, s.params
                    it.w[0], it.w[1] = _p(s.w[0]), _p(s.w[1])
                    if not fp64:
                        it.lo[0], it.lo[1] = _p(s.lo[0]), _p(s.lo[1])
                    it.sign_cf, it.src, it.dt_dev = _p(s.sign), None, _p(s.dt)
                    it.cell_scratch, it.node_scratch = _p(s.cs), _p(s.ns)
                    it.start_step, it.end_step = s.start, s.end
                    it.p1_begin, it.p1_cell_blocks, it.p2_begin = b1, ncb, b2
                    p1.append(np.full(n1, k, np.int32))
                    p2.append(np.full(n2, k, np.int32))
                    b1 += n1
                    b2 += n2
                tabs["ad"] = (self._dev_bytes(items), self._dev_i32(np.concatenate(p1)), b1,
                              self._dev_i32(np.concatenate(p2)), b2)
            if sw:
                items = ((_lib.MbSwItemF64 if fp64 else _lib.MbSwItem) * len(sw))()
                fm, cm = [], []
                bf = bc = 0
                for k, s in enumerate(sw):
                    nfb, ncb = s.blocks()
                    it = items[k]
                    check_item_tables("sw", self.precision, s.dm.struct)
                    it.m = s.dm.struct
                    for par in range(2):
                        for c in range(4):
                            it.q[par][c] = _p(s.q[par][c])
                            if not fp64:
                                it.lo[par][c] = _p(s.lo[par][c])
                        if fp64:
                            it.q[par][4] = _p(s.Z)   # the bed does not change: one array for both
                    if not fp64:
                        it.Z = _p(s.Z)
                    it.face_flux, it.dt = _p(s.ff), _p(s.dt)
                    it.cfl, it.grav = 0.5, 9.81
                    it.start_step, it.end_step = s.start, s.end
                    it.f_begin, it.c_begin = bf, bc
                    fm.append(np.full(nfb, k, np.int32))
                    cm.append(np.full(ncb, k, np.int32))
                    bf += nfb
                    bc += ncb
                tabs["sw"] = (self._dev_bytes(items), self._dev_i32(np.concatenate(fm)), bf,
                              self._dev_i32(np.concatenate(cm)), bc)
        return tabs

    def _dev_bytes(self, cstruct_array):
        raw = np.frombuffer(bytes(cstruct_array), dtype=np.uint8)
        return torch.from_numpy(raw.copy()).pin_memory().to(self.dev, non_blocking=True)

    def _dev_i32(self, a):
        return torch.from_numpy(a).pin_memory().to(self.dev, non_blocking=True)

    def _launch_step(self, tabs, st):
        fp64 = self.precision == "fp64"
        if "ad" in tabs:
            items, m1, b1, m2, b2 = tabs["ad"]
            _lib.call("mb_advdiff_batch_step" if fp64 else "mb_advdiff_batch_step_f32c", _p(items), _p(m1), b1,
                      _p(m2), b2, 2, 1, _p(self.clock[0:1]), st)
        if "sw" in tabs:
            items, m1, b1, m2, b2 = tabs["sw"]
            _lib.call("mb_sw_batch_step" if fp64 else "mb_sw_batch_step_f32c", _p(items), _p(m1), b1, _p(m2), b2,
                      _p(self.clock[1:2]), st)

    def _run_chunk(self, nsteps):
        """``nsteps`` batch steps on the compute stream (each family ticks its own clock)."""
        tabs = self._tables
        if self.graphs and nsteps == self.chunk:
            if self._graph is None:
                # captured without the device-wide synchronisation of torch.cuda.graph()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.stream(self.stream):
                    g.capture_begin()
                    try:
                        for _ in range(nsteps):
                            self._launch_step(tabs, self.stream.cuda_stream)
                    finally:
                        g.capture_end()
                self._graph = g
            with torch.cuda.stream(self.stream):
                self._graph.replay()
        else:
            for _ in range(nsteps):
                self._launch_step(tabs, self.stream.cuda_stream)

    # -------------------------------------------------------------- resident batch
    def run_resident(self, requests, steps, warmup=3):
        """Admit all ``requests`` at once (prepared beforehand), then time ``steps`` batch
        steps on the device with CUDA events.  Returns (cell-updates per second, seconds)."""
        if self.workers > 0:
            own = self.pool is None
            self.start_pool()
            prepared = [_receive(x) for x in
                        self.pool.map(prepare_shipped, requests, [self.precision] * len(requests))]
            if own:
                self.stop_pool()
        else:
            prepared = [prepare(r, self.precision) for r in requests]
        for req, dm, bc, init in prepared:
            slot = self._admit(req, dm, bc, init)
            slot.fam = 0 if req.kind == "advdiff" else 1
            slot.start, slot.end = self.clock_host[slot.fam], 1 << 30
            slot.admitted = 0.0
            self.active[req.rid] = slot
        self._retable()
        self._run_chunk(warmup)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        for _ in range(steps // self.chunk):
            self._run_chunk(self.chunk)
        if steps % self.chunk:
            self._run_chunk(steps % self.chunk)
        e1.record(self.stream)
        torch.cuda.synchronize(self.dev)
        sec = e0.elapsed_time(e1) / 1e3
        cu = sum(s.dm.nbcells for s in self.active.values()) * steps
        return cu / sec, sec

    # -------------------------------------------------------------- serving loop
    def serve(self, requests, keep_results=False, log=None):
        """Run ``requests`` (their ``arrival`` times are honoured) to completion.  Returns a
        list of per-request records: arrival, admission, completion, latency (seconds from
        arrival to the result on the host), cells, steps, and the result arrays if asked."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        own_pool = self.workers > 0 and self.pool is None
        if own_pool:
            self.start_pool()
        pool = self.pool if self.workers > 0 else None
        st = self.stats = {k: 0.0 for k in ("receive", "admit", "retable", "launch", "throttle", "complete", "idle")}
        for k in ("admit_stage_wait", "admit_tables", "admit_bc", "admit_setup"):
            st[k] = 0.0
        inflight = []          # events of the chunks on the device, oldest first
        futures = {}
        prepared = []          # (req, dm, bc, init), in arrival order
        nxt = 0
        done = []
        pending_done = []      # (event, slots)
        t0 = time.perf_counter()
        self._t0, self._t_sub, self._t_recv = t0, {}, {}
        used = 0.0
        arrived = queue.SimpleQueue()   # (rid, future) of finished preparations
        n_recv = 0
        stop = threading.Event()
        dispatcher = None
        if pool is not None and self.poll:
            def dispatch():
                for r in reqs:
                    while (wait := r.arrival - (time.perf_counter() - t0)) > 0:
                        if stop.wait(wait):
                            return
                    threads = None
                    if self.adaptive_threads:
                        busy = len(self._t_sub) - n_recv + 1    # preparations in flight, this one included
                        threads = max(1, self.cores // busy)
                    self._t_sub[r.rid] = time.perf_counter() - t0
                    fut = pool.submit(prepare_shipped, r, self.precision, threads)
                    fut.add_done_callback(functools.partial(self._arrived, arrived, r.rid))
            dispatcher = threading.Thread(target=dispatch, daemon=True)
            dispatcher.start()
            nxt = len(reqs)
        try:
            while len(done) < len(reqs):
                now = time.perf_counter() - t0
                # hand arrived requests to the preparation pool
                while nxt < len(reqs) and reqs[nxt].arrival <= now:
                    r = reqs[nxt]
                    self._t_sub[r.rid] = time.perf_counter() - t0
                    if pool is not None:
                        futures[r.rid] = pool.submit(prepare_shipped, r, self.precision)
                    else:
                        prepared.append(prepare(r, self.precision))
                    nxt += 1
                ta = time.perf_counter()
                for rid in [k for k, f in futures.items() if f.done()]:
                    prepared.append(_receive(futures.pop(rid).result()))
                    self._t_recv[rid] = time.perf_counter() - t0
                while not arrived.empty():
                    rid, item, err = arrived.get()
                    if err is not None:
                        raise err
                    prepared.append(item)
                    self._t_recv[rid] = time.perf_counter() - t0
                    n_recv += 1
                prepared.sort(key=lambda x: x[0].arrival)
                tb = time.perf_counter()
                st["receive"] += tb - ta
                # admission (between steps): arrival order while a slot and the budget
                # allow, smaller requests passing one that does not fit for a while
                changed = False
                picks = []
                if prepared and len(self.active) < self.max_active:
                    waiting = [(self._t_recv.get(x[0].rid, x[0].arrival),
                                x[1].nbytes() + 48.0 * x[1].nbcells + 16.0 * x[1].nbfaces) for x in prepared]
                    picks = admission_order(waiting, used, self.budget, self.max_active - len(self.active),
                                            len(self.active), time.perf_counter() - t0, self.max_skip_wait)
                chosen = [prepared[k] for k in picks]
                if picks:
                    taken = set(picks)
                    prepared = [x for k, x in enumerate(prepared) if k not in taken]
                for req, dm, bc, init in chosen:
                    slot = self._admit(req, dm, bc, init)
                    slot.admitted = time.perf_counter() - t0
                    slot.fam = 0 if req.kind == "advdiff" else 1
                    slot.start = self.clock_host[slot.fam]
                    slot.end = slot.start + req.steps
                    used += slot.nbytes
                    self.active[req.rid] = slot
                    changed = True
                tc = time.perf_counter()
                st["admit"] += tc - tb
                if changed:
                    self._retable()
                td = time.perf_counter()
                st["retable"] += td - tc
                if not self.active:
                    if (nxt >= len(reqs) and not futures and not prepared and not pending_done
                            and (dispatcher is None or n_recv == len(reqs))):
                        break
                    used -= self._complete(pending_done, done, t0, keep_results, log)
                    time.sleep(0.002)
                    st["idle"] += time.perf_counter() - td
                    continue
                # keep at most two chunks queued on the device, so that admissions and
                # retirements take effect within about one chunk
                if self.poll:
                    while inflight and inflight[0].query():
                        inflight.pop(0)
                    if len(inflight) >= 2:
                        used -= self._complete(pending_done, done, t0, keep_results, log)
                        time.sleep(0.0002)
                        st["throttle"] += time.perf_counter() - td
                        continue
                while len(inflight) >= 2:
                    inflight.pop(0).synchronize()
                te = time.perf_counter()
                st["throttle"] += te - td
                # advance to the next finishing request or one chunk, whichever is first
                remaining = min(s.end - self.clock_host[s.fam] for s in self.active.values())
                nsteps = max(1, min(self.chunk, remaining))
                self._run_chunk(nsteps)
                ev_chunk = torch.cuda.Event()
                ev_chunk.record(self.stream)
                inflight.append(ev_chunk)
                tf = time.perf_counter()
                st["launch"] += tf - te
                fams = {s.fam for s in self.active.values()}
                for f in fams:
                    self.clock_host[f] += nsteps
                fin = [s for s in self.active.values() if s.end <= self.clock_host[s.fam]]
                if fin:
                    for s in fin:
                        del self.active[s.req.rid]
                    with torch.cuda.stream(self.stream):
                        outs = [[t.to("cpu", non_blocking=True) for t in s.result()] for s in fin]
                    ev = torch.cuda.Event()
                    ev.record(self.stream)
                    pending_done.append((ev, fin, outs))
                    self._retable()
                tg = time.perf_counter()
                used -= self._complete(pending_done, done, t0, keep_results, log)
                st["complete"] += time.perf_counter() - tg
            torch.cuda.synchronize(self.dev)
            used -= self._complete(pending_done, done, t0, keep_results, log)
        finally:
            stop.set()
            if dispatcher is not None:
                dispatcher.join()
            # preparations that were never received (an error ended the loop): their
            # shared-memory files are removed as they finish
            for f in futures.values():
                if not f.cancel():
                    f.add_done_callback(_discard)
            if own_pool:
                self.stop_pool()
        return done

    @staticmethod
    def _arrived(out, rid, fut):
        """Done-callback of a preparation (on the pool's thread): the request read back from
        shared memory, or the error, queued for the serving loop."""
        try:
            out.put((rid, _receive(fut.result()), None))
        except BaseException as e:  # handed to the serving loop, which raises it
            out.put((rid, None, e))

    def _retable(self):
        """New item tables and block maps for the current active set (the old ones stay
        alive until later steps have certainly finished with them)."""
        if self._tables is not None:
            self._old.append((self._tables, self._graph))
            self._old = self._old[-8:]
        self._tables = self._build_tables() if self.active else None
        self._graph = None

    def _complete(self, pending_done, done, t0, keep_results, log):
        """Record requests whose results reached the host; returns the bytes they release."""
        freed = 0
        still = []
        for ev, fin, outs in pending_done:
            if not ev.query():
                still.append((ev, fin, outs))
                continue
            tdone = time.perf_counter() - t0
            for s, o in zip(fin, outs):
                rec = {"rid": s.req.rid, "kind": s.req.kind, "cells": s.dm.nbcells, "steps": s.req.steps,
                       "arrival": s.req.arrival, "admitted": s.admitted, "done": tdone,
                       "latency": tdone - s.req.arrival}
                # the preparation's course: handed to the pool, run in a worker, back in this process
                rec["submitted"] = self._t_sub.get(s.req.rid)
                if s.req.prep_window is not None:
                    rec["prep_start"], rec["prep_end"] = (x - self._t0 for x in s.req.prep_window)
                rec["received"] = self._t_recv.get(s.req.rid, rec["submitted"])
                if keep_results:
                    inv = np.asarray(s.dm.inv["cell"])
                    rec["result"] = [x.numpy()[inv] for x in o]
                done.append(rec)
                freed += s.nbytes
            if log:
                log(len(done))
        pending_done[:] = still
        return freed
