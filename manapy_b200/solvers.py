"""Explicit solvers with manapy's call surface, running the fused CUDA steps.

``AdvectionDiffusionSolver`` mirrors ``manapy/solvers/advecdiff/system.py:21-172``
and ``ShallowWaterSolver`` mirrors ``manapy/solvers/shallowater/system.py:23-281``:
same options, same validation errors, same ``stepper()`` /
``compute_fluxes()`` / ``compute_new_val()`` sequence.

Execution: ``compute_new_val()`` runs one fused step (two kernel launches for
advection-diffusion, three for shallow water) that recomputes what
``compute_fluxes()`` would have produced on the fly.  The intermediate arrays
manapy leaves behind (``var.ghost``, ``var.convective``, ``var.dissipative``,
``var.gradfacex/y/z``) are still available: reading one runs the matching
single kernel on the step's input state.  Editing ``var.convective``,
``var.dissipative`` or ``var.source`` between ``compute_fluxes()`` and
``compute_new_val()`` switches that step to the unfused update, so the edit
is honoured exactly as in manapy.

``advance(n)`` runs ``n`` whole steps (``stepper`` + ``compute_fluxes`` +
``compute_new_val``) on the device without host round trips, optionally
replayed from a CUDA graph.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .base import Struct, make_get_conf, process_conf
from .variable import Variable

__all__ = ["AdvectionDiffusionSolver", "AdvectionSolver", "DiffusionSolver", "ShallowWaterSolver", "EulerSolver"]


def _p(t):
    return t.data_ptr() if t is not None else None


def check_state(arrays, nonneg=(), names=None):
    """Raise ``FloatingPointError`` if a device array holds NaN or infinity, ``ValueError``
    if an array listed in ``nonneg`` (by position) holds a negative value (the statuses
    MB_ENONFINITE / MB_ENEGATIVE of ``mb_check_state``)."""
    for k, t in enumerate(arrays):
        flags = torch.zeros(1, dtype=torch.int32, device=t.device)
        f64 = t if t.dtype == torch.float64 else None
        f32 = t if t.dtype == torch.float32 else None
        _lib.call("mb_check_state", _p(f64), _p(f32), t.numel(), int(k in nonneg), _p(flags),
                  torch.cuda.current_stream(t.device).cuda_stream)
        f = int(flags.item())
        name = names[k] if names else "array %d" % k
        if f & 1:
            raise FloatingPointError("non-finite values in %s" % name)
        if f & 2:
            raise ValueError("negative values in %s" % name)


class AdvectionDiffusionSolver:
    _parameters = [("Dxx", float, 0., 0., "Diffusion in x direction"),
                   ("Dyy", float, 0., 0., "Diffusion in y direction"),
                   ("Dzz", float, 0., 0., "Diffusion in z direction"),
                   ("dt", float, 0., 0., "time step"),
                   ("order", int, 1, 1, "order of the convective scheme"),
                   ("cfl", float, .4, 0, "cfl of the explicit scheme"),
                   ("precision", str, "fp64", 0, "fp64 (manapy's arithmetic) or fp32c: FP32 state and "
                                                 "fluxes with compensated per-cell sums, FP64 geometry and dt "
                                                 "(no counterpart in manapy)"),
                   ("graph_depth", object, "auto", 0, "steps per CUDA-graph replay in advance(graph=True): an "
                                                      "even number, or 'auto' (measured by manapy_b200.autotune)"),
                   ("launch", object, "auto", 0, "launch shapes of the fused phases: 'auto' (measured by "
                                                 "manapy_b200.autotune at the first graph advance), or a variant "
                                                 "number (bits 0-1 first phase, 2-3 second; 0 = defaults)"),
                   ("lsq_sums", bool, True, 0, "tetrahedra, second order: least-squares sums by inclusion-"
                                               "exclusion over vertex and edge sums instead of gathering each "
                                               "cell's stencil (equal up to rounding; no counterpart in manapy)")]

    @classmethod
    def process_conf(cls, conf, kwargs):
        return process_conf(cls._parameters, conf, kwargs)

    def __init__(self, var=None, vel=(None, None, None), conf=None, **kwargs):
        if conf is None:
            conf = Struct()
        self.conf = self.process_conf(conf, kwargs)
        get = make_get_conf(self.conf, kwargs)
        if not isinstance(var, Variable):
            raise ValueError("primal var must be a Variable type")
        if not isinstance(vel[0], Variable):
            raise ValueError("u must be a Variable type")
        if not isinstance(vel[1], Variable):
            raise ValueError("v must be a Variable type")
        self.var = var
        self.comm = var.comm
        self.domain = var.domain
        self.dim = var.dim
        self.float_precision = self.domain.float_precision
        self.u, self.v = vel[0], vel[1]
        if len(vel) == 3:
            if not isinstance(vel[2], Variable):
                raise ValueError("w must be a Variable type")
            self.w = vel[2]
        else:
            self.w = Variable(domain=self.domain)
        self.Dxx = np.float64(get("Dxx"))
        self.Dyy = np.float64(get("Dyy"))
        self.Dzz = np.float64(get("Dzz"))
        self.dt = np.float64(get("dt"))
        self.order = np.int32(get("order"))
        self.cfl = np.float64(get("cfl"))
        if self.order not in (1, 2):
            raise ValueError("order must be 1 or 2")
        self.precision = str(get("precision"))
        if self.precision not in ("fp64", "fp32c"):
            raise ValueError("precision must be 'fp64' or 'fp32c'")
        depth = get("graph_depth")
        if depth != "auto" and (int(depth) < 2 or int(depth) % 2):
            raise ValueError("graph_depth must be 'auto' or an even number >= 2")
        self.graph_depth = depth if depth == "auto" else int(depth)
        launch = get("launch")
        if launch != "auto" and int(launch) not in range(16):
            raise ValueError("launch must be 'auto' or a variant number 0-15")
        self.launch = launch if launch == "auto" else int(launch)
        self.launch_variant = 0 if launch == "auto" else int(launch)
        self.lsq_sums = bool(get("lsq_sums"))
        self.diffusion = not (self.Dxx == self.Dyy == self.Dzz == 0)
        self.backend = self.domain.backend
        self.signature = self.domain.signature
        for t in ("convective", "dissipative", "source"):
            var.add_term(t)
        self._dm = None
        self._dt_dev = None
        self._dt_key = None
        self._sign = None
        self._sign_key = None
        self._pending = False
        self._spare = None
        self._graph = None
        self._dt_host = None
        self._w32 = None       # FP32 ping-pong state of the fp32c mode
        self._w32_i = 0
        self._w32_key = None   # var.version("cell") the FP32 state corresponds to
        self._sign32 = None
        self._sign32_key = None
        self._src32 = None
        self._src32_key = None
        self._graph_src = None

    # ------------------------------------------------------------ device helpers
    def _setup(self):
        if self._dm is None:
            self._dm = self.domain.device_mesh
            if self.order == 2:
                self._dm.ensure_lsq_matrix(self._stream())
                if self.lsq_sums:
                    self._dm.use_edge_sums()
            if self.launch != "auto":
                self._dm.struct.variant = int(self.launch)
            dev = self._dm.device
            self._dt_dev = torch.zeros(1, dtype=torch.float64, device=dev)
            self._sign = torch.zeros(4 * self._dm.nbcells, dtype=torch.float64, device=dev)
            self._params = _lib.MbAdvDiffParams(int(self.order), int(self.diffusion), float(self.Dxx),
                                                float(self.Dyy), float(self.Dzz))
        return self._dm

    def _stream(self):
        return torch.cuda.current_stream(self._dm.device).cuda_stream

    def _update_sign(self):
        key = (self.u.version("face"), self.v.version("face"), self.w.version("face"))
        if key != self._sign_key:
            _lib.call("mb_cell_face_sign", self._dm.struct, _p(self.u.dev("face")), _p(self.v.dev("face")),
                      _p(self.w.dev("face")), _p(self._sign), self._stream())
            self._sign_key = (self.u.version("face"), self.v.version("face"), self.w.version("face"))

    def _time_step_dev(self):
        """dt on the device; recomputed only when the cell velocity or options change
        (manapy recomputes the same value every step from the same inputs)."""
        key = (self.u.version("cell"), self.v.version("cell"), self.w.version("cell"),
               float(self.cfl), float(self.Dxx), float(self.Dyy), float(self.Dzz))
        if key != self._dt_key:
            _lib.call("mb_time_step", self._dm.struct, _p(self.u.dev("cell")), _p(self.v.dev("cell")),
                      _p(self.w.dev("cell")), float(self.cfl), float(self.Dxx), float(self.Dyy),
                      float(self.Dzz), _p(self._dt_dev), self._stream())
            self._dt_key = (self.u.version("cell"), self.v.version("cell"), self.w.version("cell"),
                            float(self.cfl), float(self.Dxx), float(self.Dyy), float(self.Dzz))
            self._dt_host = None
        return self._dt_dev

    # ------------------------------------------------------------ manapy API
    def stepper(self):
        """manapy/solvers/advecdiff/system.py:149-153: the CFL time step."""
        self._setup()
        self._time_step_dev()
        if self._dt_host is None:
            self._dt_host = float(self._dt_dev.item())
        self.dt = np.float64(self._dt_host)
        return self.dt

    def explicit_convective(self):
        """manapy/solvers/advecdiff/system.py:131-141 (unfused: gradient, limiter, upwind flux)."""
        self._setup()
        var = self.var
        if self.order == 2:
            var.compute_cell_gradient()
        _lib.call("mb_explicitscheme_convective", self._dm.struct, _p(var.dev_out("convective")),
                  _p(var.dev("cell")), _p(var.dev("ghost")), _p(self.u.dev("face")), _p(self.v.dev("face")),
                  _p(self.w.dev("face")), _p(var.dev("gradcellx")), _p(var.dev("gradcelly")),
                  _p(var.dev("gradcellz")), _p(var.dev("psi")), int(self.order), self._stream())

    def explicit_dissipative(self):
        """manapy/solvers/advecdiff/system.py:143-146 (unfused)."""
        self._setup()
        var = self.var
        var.compute_face_gradient()
        _lib.call("mb_explicitscheme_dissipative", self._dm.struct, _p(var.dev("gradfacex")),
                  _p(var.dev("gradfacey")), _p(var.dev("gradfacez")), _p(var.dev_out("dissipative")),
                  float(self.Dxx), float(self.Dyy), float(self.Dzz), self._stream())

    def _materialise(self, w_in):
        """Run the unfused kernels on state ``w_in`` to fill ghost, convective, dissipative
        (and face gradients, nodes) exactly as manapy's compute_fluxes leaves them."""
        var = self.var
        cur = var.swap_cell(w_in)
        try:
            var.update_ghost_value()
            self.explicit_convective()
            if self.diffusion:
                var.interpolate_celltonode()
                self.explicit_dissipative()
        finally:
            var.swap_cell(cur)

    def _install_lazies(self, w_in):
        """``w_in``: the step's FP64 input state, or a callable returning it."""
        var = self.var
        done = {"v": False}

        def run():
            if not done["v"]:
                done["v"] = True
                for n in names:
                    var._s.lazy.pop(n, None)
                self._materialise(w_in() if callable(w_in) else w_in)

        names = ["ghost", "convective"]
        if self.order == 2:
            names += ["gradcellx", "gradcelly", "gradcellz", "psi"]
        if self.diffusion:
            names += ["node", "dissipative", "gradfacex", "gradfacey", "gradfacez"]
        for n in names:
            var.set_lazy(n, run)

    def compute_fluxes(self):
        """manapy/solvers/advecdiff/system.py:156-168; fused into compute_new_val()."""
        self._setup()
        var = self.var
        self._pending = True
        self._res_versions = tuple(var.version(n) for n in ("convective", "dissipative"))
        self._install_lazies(var.dev("cell"))

    def compute_new_val(self):
        """manapy/solvers/advecdiff/system.py:171-172: w += dt((rez + dissip)/V + src)."""
        self._setup()
        var = self.var
        if self._dt_host is None or float(self.dt) != self._dt_host:
            # stepper() not called, or S.dt set by hand: use S.dt as manapy does
            self._dt_dev.fill_(float(self.dt))
            self._dt_key = None
            self._dt_host = float(self.dt)
        edited = (not self._pending or
                  tuple(var.version(n) for n in ("convective", "dissipative")) != self._res_versions)
        if edited:
            for n in ("ghost", "convective", "dissipative", "gradfacex", "gradfacey", "gradfacez"):
                if n in var._s.lazy:
                    var._s.d(n)
            _lib.call("mb_update_new_value", self._dm.struct, _p(var.dev("cell")),
                      _p(var.dev("convective")), _p(var.dev("dissipative")), _p(var.dev("source")),
                      _p(self._dt_dev), self._stream())
            var._s.version["cell"] += 1
        else:
            self._fused_step()
        self._pending = False

    def _source_ptr(self):
        var = self.var
        return None if var.version("source") == 0 else _p(var.dev("source"))

    def _scratch(self):
        dm = self._dm
        if getattr(self, "_cs", None) is None or self._cs.numel() < dm.cell_scratch_size():
            # 4 nbcells (2D: records) or 8 nbcells (3D: records, rows), plus the vertex and edge
            # records when the 3D step uses the edge sums (grown if another solver on this mesh
            # opted the struct into them since)
            self._cs = torch.empty(dm.cell_scratch_size(), dtype=torch.float64, device=dm.device)
            self._ns = torch.empty(dm.nbnodes, dtype=torch.float64, device=dm.device)
        return self._cs, self._ns

    # rows {centre, value} carried from step to step (second order): each cell buffer has a
    # rows buffer; _rows_version is the cell version whose rows are current
    def _use_rows(self):
        # tetrahedra only: a triangle's 16-byte centre row shares its 32-byte sector with its
        # Morton neighbour's, so 32-byte rows would double the gathered sectors (measured slower)
        return self.order == 2 and self.dim == 3 and "cell_vtx" in self._dm.t

    def _rows_of(self, buf):
        if getattr(self, "_rowbufs", None) is None:
            self._rowbufs = {}
        r = self._rowbufs.get(buf.data_ptr())
        if r is None:
            r = torch.empty(4 * self._dm.nbcells, dtype=torch.float64, device=self._dm.device)
            self._rowbufs[buf.data_ptr()] = r
        return r

    def _ensure_rows(self, buf):
        """Rows of ``buf`` (the current cell array), packed if the state changed since a step
        wrote them."""
        if getattr(self, "_rows_version", None) != self.var.version("cell"):
            _lib.call("mb_pack_rows", self._dm.struct, _p(buf), _p(self._rows_of(buf)), self._stream())
            self._rows_version = self.var.version("cell")
        return self._rows_of(buf)

    def _fused_step(self):
        if self.precision == "fp32c":
            return self._fused_step_f32c()
        var = self.var
        dm = self._dm
        self._update_sign()
        w_in = var.dev("cell")
        if self._spare is None or self._spare.numel() != w_in.numel():
            self._spare = torch.empty_like(w_in)
        w_out = self._spare
        cs, ns = self._scratch()
        if self._use_rows():
            rin = self._ensure_rows(w_in)
            _lib.call("mb_advdiff_step_rows", dm.struct, var.device_bc.struct, self._params, _p(w_in), _p(w_out),
                      _p(rin), _p(self._rows_of(w_out)), _p(self._sign), self._source_ptr(), _p(self._dt_dev), _p(cs),
                      _p(ns), self._stream())
        else:
            _lib.call("mb_advdiff_step", dm.struct, var.device_bc.struct, self._params, _p(w_in), _p(w_out),
                      _p(self._sign), self._source_ptr(), _p(self._dt_dev), _p(cs), _p(ns), self._stream())
        self._spare = var.swap_cell(w_out)
        self._install_lazies(self._spare)
        self._rows_version = var.version("cell")

    # ------------------------------------------------------------ fp32c mode
    def _f32_state(self):
        """The FP32 state, reloaded from the cell array when that changed since the last step."""
        var = self.var
        dm = self._dm
        if self._w32 is None:
            self._w32 = [torch.empty(dm.nbcells, dtype=torch.float32, device=dm.device) for _ in range(2)]
            # rounding errors of the FP32 state (w + lo carries the state to ~48 bits)
            self._lo32 = [torch.empty(dm.nbcells, dtype=torch.float32, device=dm.device) for _ in range(2)]
            self._cs32 = torch.empty(dm.cell_scratch_size_f32c(), dtype=torch.float32, device=dm.device)
            self._ns32 = torch.empty(dm.nbnodes, dtype=torch.float32, device=dm.device)
            self._sign32 = torch.empty((4 if dm.dim == 2 else 5) * dm.nbcells, dtype=torch.float32,
                                       device=dm.device)
        if var.version("cell") != self._w32_key:
            w64 = var.dev("cell")
            hi = self._w32[self._w32_i]
            hi.copy_(w64)
            self._lo32[self._w32_i].copy_(w64 - hi.double())
            self._w32_key = var.version("cell")
        return self._w32[self._w32_i]

    def _f64_of(self, k):
        """FP64 value of FP32 state buffer ``k`` (w + lo)."""
        return self._w32[k].double() + self._lo32[k].double()

    def _f32_inputs(self):
        self._update_sign()
        if self._sign32_key != self._sign_key:
            _lib.call("mb_cell_face_sign_f32c", self._dm.struct, _p(self._sign), _p(self._sign32), self._stream())
            self._sign32_key = self._sign_key
        var = self.var
        if var.version("source") == 0:
            return None
        if self._src32_key != var.version("source"):
            self._src32 = var.dev("source").float()
            self._src32_key = var.version("source")
        return self._src32

    def _f32_publish(self, prev):
        """Make the FP32 result the variable's cell array (converted on first read);
        ``prev``: the buffer index holding the step's input."""
        var = self.var
        cur = self._w32_i

        def materialise(k=cur):
            var._s.dev["cell"].copy_(self._f64_of(k))

        var._s.lazy.pop("cell", None)  # the previous result, superseded
        var._s.version["cell"] += 1
        var.set_lazy("cell", materialise)
        self._w32_key = var.version("cell")
        self._install_lazies(lambda k=prev: self._f64_of(k))

    def _call_f32c(self, k, src, st):
        """One step from buffer k into buffer 1 - k."""
        w, lo = self._w32, self._lo32
        if self._cs32.numel() < self._dm.cell_scratch_size_f32c():
            # another solver on this mesh opted its struct into the edge sums since the
            # scratch was sized
            self._cs32 = torch.empty(self._dm.cell_scratch_size_f32c(), dtype=torch.float32, device=self._dm.device)
        _lib.call("mb_advdiff_step_f32c", self._dm.struct, self.var.device_bc.struct, self._params, _p(w[k]),
                  _p(w[1 - k]), _p(lo[k]), _p(lo[1 - k]), _p(self._sign32), _p(src), _p(self._dt_dev),
                  _p(self._cs32), _p(self._ns32), st)

    def _fused_step_f32c(self):
        self._f32_state()
        src = self._f32_inputs()
        k = self._w32_i
        self._call_f32c(k, src, self._stream())
        self._w32_i = 1 - k
        self._f32_publish(k)

    def check(self):
        """Raise if the state holds NaN or infinity (manapy lets them propagate)."""
        self._setup()
        if self.precision == "fp32c" and self._w32 is not None and self.var.version("cell") == self._w32_key:
            check_state([self._w32[self._w32_i]], names=["the FP32 state"])
        else:
            check_state([self.var.dev("cell")], names=["the cell values"])

    def launches_per_step(self):
        """Kernel launches of one fused step."""
        # (tetrahedra at order 2 through mb_advdiff_step pack rows first; the solver's steps
        # carry them from one step to the next instead; with the edge sums the first phase is
        # two launches: vertex and edge sums, then the cells)
        dm = self._dm
        sums = dm is not None and self.order == 2 and dm.struct is not None and bool(dm.struct.cell_edges)
        return 1 + int(self.order == 2 or bool(self.diffusion)) + int(sums)

    def release_graphs(self):
        self._graph = None

    # ------------------------------------------------------------ device loop
    def advance(self, nsteps, graph=False):
        """Run ``nsteps`` full steps on the device (dt, fluxes, update) without host
        synchronisation.  Returns the simulated time span (dt is constant while the
        velocity does not change).  ``graph=True`` replays two-step CUDA graphs."""
        self._setup()
        var = self.var
        self._time_step_dev()
        self._update_sign()
        n = int(nsteps)
        if self.precision == "fp32c":
            self._advance_f32c(n, graph)
            if self._dt_host is None:
                self._dt_host = float(self._dt_dev.item())
            self.dt = np.float64(self._dt_host)
            return n * self._dt_host
        var.dev("cell")
        if self._spare is None:
            self._spare = torch.empty_like(var.dev("cell"))
        depth = self._depth() if graph else 2
        if not graph or n < depth:
            for _ in range(n):
                self._fused_step()
        else:
            g = self._get_graph()
            a, b = self._graph_bufs
            cur = var.dev("cell")
            if cur is b:      # after an odd number of steps: one step brings the state back to a
                self._fused_step()
                n -= 1
            elif cur is not a:  # a cell array installed since the capture
                a.copy_(cur)
                var.swap_cell(a)
                self._spare = b
            if self._use_rows() and n // depth:
                self._ensure_rows(a)         # the captured steps start from a's rows
            for _ in range(n // depth):
                g.replay()
            if n // depth:
                var._s.version["cell"] += 1
                self._install_lazies(self._spare)
                self._rows_version = var.version("cell")
            for _ in range(n % depth):
                self._fused_step()
        if self._dt_host is None:
            self._dt_host = float(self._dt_dev.item())
        self.dt = np.float64(self._dt_host)
        return n * self._dt_host

    def _advance_f32c(self, n, graph):
        depth = self._depth() if graph else 2
        if not graph or n < depth:
            for _ in range(n):
                self._fused_step_f32c()
            return
        self._f32_state()
        if self._w32_i != 0:  # the captured pair starts from buffer 0
            self._fused_step_f32c()
            n -= 1
        src = self._f32_inputs()
        self.var.device_bc  # built (and uploaded) before any capture
        if self._graph is None or self._graph_src != _p(src):
            s = torch.cuda.Stream(device=self._dm.device)
            s.wait_stream(torch.cuda.current_stream(self._dm.device))
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    st = torch.cuda.current_stream(self._dm.device).cuda_stream
                    for _ in range(depth // 2):
                        self._call_f32c(0, src, st)
                        self._call_f32c(1, src, st)
            torch.cuda.current_stream(self._dm.device).wait_stream(s)
            self._graph, self._graph_src = g, _p(src)
        for _ in range(n // depth):
            self._graph.replay()
        if n // depth:
            self._f32_publish(1)
        for _ in range(n % depth):
            self._fused_step_f32c()

    def _depth(self):
        """Steps per graph replay (measured once per mesh size and scheme when 'auto'); with
        ``launch="auto"`` also the launch shapes of the fused phases (once per solver)."""
        from . import autotune
        if self.graph_depth == "auto":
            self.graph_depth = autotune.graph_depth(self)
        if self.launch == "auto":
            self.launch = "tuned"
            self.launch_variant = autotune.launch_variant(self)
        return int(self.graph_depth)

    def _get_graph(self):
        """``graph_depth`` fused steps (A->B, B->A, ...) captured once; the cell buffer ends
        where it began."""
        if self._graph is not None:
            return self._graph
        var = self.var
        a = var.dev("cell")
        b = self._spare
        dm = self._dm
        cs, ns = self._scratch()
        args = (var.device_bc.struct, self._params)
        src = self._source_ptr()
        s = torch.cuda.Stream(device=dm.device)
        s.wait_stream(torch.cuda.current_stream(dm.device))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            # warm-up outside capture is not needed: the library performs no lazy init
            rows = self._use_rows()
            if rows:
                self._rows_of(a), self._rows_of(b)   # allocated before the capture
            with torch.cuda.graph(g, stream=s):
                st = torch.cuda.current_stream(dm.device).cuda_stream
                for x, y in ((a, b), (b, a)) * (int(self.graph_depth) // 2):
                    if rows:
                        _lib.call("mb_advdiff_step_rows", dm.struct, args[0], args[1], _p(x), _p(y),
                                  _p(self._rows_of(x)), _p(self._rows_of(y)), _p(self._sign), src, _p(self._dt_dev),
                                  _p(cs), _p(ns), st)
                    else:
                        _lib.call("mb_advdiff_step", dm.struct, args[0], args[1], _p(x), _p(y), _p(self._sign),
                                  src, _p(self._dt_dev), _p(cs), _p(ns), st)
        torch.cuda.current_stream(dm.device).wait_stream(s)
        self._graph = g
        self._graph_bufs = (a, b)
        return g


class AdvectionSolver(AdvectionDiffusionSolver):
    """manapy/solvers/advec/system.py:20-154: the convective flux only (manapy's options:
    dt, order, cfl).  Same step as ``AdvectionDiffusionSolver`` with no diffusion; manapy's
    advection time step has no zero-speed guard (a cell with zero speed on every face
    divides by zero there), here such a cell does not limit dt."""
    _parameters = [p for p in AdvectionDiffusionSolver._parameters if p[0] not in ("Dxx", "Dyy", "Dzz")]

    def __init__(self, var=None, vel=(None, None, None), conf=None, **kwargs):
        super().__init__(var, vel, conf, **kwargs)
        self.Dxx = self.Dyy = self.Dzz = np.float64(0.)
        self.diffusion = False


class DiffusionSolver(AdvectionDiffusionSolver):
    """manapy/solvers/diffusion/system.py:20-156: the diamond diffusion flux only.  manapy
    takes the velocity variables but uses none of them (its time step is the diffusion
    bound alone, ``manapy/solvers/diffusion/fvm_utils.py:30-47``); here the step runs with
    zero velocity, which adds exact zeros to the same sums."""

    def __init__(self, var=None, vel=(None, None, None), conf=None, **kwargs):
        super().__init__(var, vel, conf, **kwargs)
        self.vel_given = (self.u, self.v, self.w)
        self.u, self.v, self.w = (Variable(domain=self.domain) for _ in range(3))
        self.order = np.int32(1)  # no convective flux, so no reconstruction either


class ShallowWaterSolver:
    _parameters = [("Dxx", float, 0., 0., "Diffusion in x direction"),
                   ("Dyy", float, 0., 0., "Diffusion in y direction"),
                   ("dt", float, 0., 0., "time step"),
                   ("order", int, 1, 1, "order of the convective scheme"),
                   ("cfl", float, .8, 0, "cfl of the explicit scheme"),
                   ("Mann", float, 0., 0., "Manning number for the friction"),
                   ("fc", float, 0., 0., "Coriolis force"),
                   ("grav", float, 9.81, 0., "gravity constant"),
                   ("wind", bool, False, True, "wind"),
                   ("precision", str, "fp64", 0, "fp64 (manapy's arithmetic) or fp32c: FP32 state and fluxes "
                                                 "with compensated per-cell sums, FP64 geometry, source and dt "
                                                 "(first order; no counterpart in manapy)"),
                   ("walls", str, "neumann", 0, "boundary faces of the fused step: neumann (manapy's default "
                                                "ghosts, the interior state) or reflective (mirrored momentum, "
                                                "no mass flux; no counterpart in manapy)")]

    @classmethod
    def process_conf(cls, conf, kwargs):
        return process_conf(cls._parameters, conf, kwargs)

    def __init__(self, h=None, hvel=(None, None), hc=None, Z=None, conf=None, **kwargs):
        if conf is None:
            conf = Struct()
        self.conf = self.process_conf(conf, kwargs)
        get = make_get_conf(self.conf, kwargs)
        if not isinstance(h, Variable):
            raise ValueError("h must be a Variable type")
        if not isinstance(hvel[0], Variable):
            raise ValueError("hu must be a Variable type")
        if not isinstance(hvel[1], Variable):
            raise ValueError("hv must be a Variable type")
        self.h = h
        self.comm = h.comm
        self.domain = h.domain
        self.dim = h.dim
        if self.dim != 2:
            raise ValueError("the shallow-water scheme is two-dimensional")
        self.float_precision = self.domain.float_precision
        self.hu, self.hv = hvel
        if Z is not None and not isinstance(Z, Variable):
            raise ValueError("Z must be a Variable type")
        if hc is not None and not isinstance(hc, Variable):
            raise ValueError("hC must be a Variable type")
        self.Z = Z if Z is not None else Variable(domain=self.domain)
        self.hc = hc if hc is not None else Variable(domain=self.domain)
        self.varbs = {"h": self.h, "hu": self.hu, "hv": self.hv, "hc": self.hc, "Z": self.Z}
        for var in self.varbs.values():
            for term in ("source", "dissipation", "coriolis", "friction", "convective"):
                var.add_term(term)
        self.Dxx = get("Dxx")
        self.Dyy = get("Dyy")
        self.Dzz = 0.
        self.dt = get("dt")
        self.order = get("order")
        self.cfl = get("cfl")
        self.Mann = get("Mann")
        self.fc = get("fc")
        self.grav = get("grav")
        self.wind = get("wind")
        if self.order not in (1, 2):
            raise ValueError("order must be 1 or 2")
        if not (self.Dxx == self.Dyy == 0):
            raise NotImplementedError("shallow-water diffusion: manapy's diffusive branch references "
                                      "attributes it never sets (manapy/solvers/shallowater/system.py:269-271)")
        if self.Mann != 0 or self.fc != 0 or self.wind:
            raise NotImplementedError("friction, Coriolis and wind source terms are not implemented")
        self.precision = str(get("precision"))
        if self.precision not in ("fp64", "fp32c"):
            raise ValueError("precision must be 'fp64' or 'fp32c'")
        if self.precision == "fp32c" and self.order != 1:
            raise NotImplementedError("the fp32c shallow-water step is first order")
        self.walls = str(get("walls"))
        if self.walls not in _lib.WALLS:
            raise ValueError("walls must be 'neumann' or 'reflective'")
        self._q32 = None
        self._q32_key = None
        self._q32_i = 0
        self.diffusion = False
        self.backend = self.domain.backend
        self.signature = self.domain.signature
        self._dm = None
        self._ff = None
        self._spare = None
        self._scratch = None
        self._dt_host = None
        self._fused = False

    def _setup(self):
        if self._dm is None:
            self._dm = self.domain.device_mesh
            dev = self._dm.device
            # dt double buffer: slot _cur holds the dt of the current state when _dt_key matches
            self._dt_buf = torch.zeros(2, dtype=torch.float64, device=dev)
            self._cur = 0
            self._dt_key = None
            self._ff = torch.zeros(5 * self._dm.nbfaces, dtype=torch.float64, device=dev)
            if self.order == 2:
                self._scratch = torch.zeros(5 * self._dm.nbcells, dtype=torch.float64, device=dev)
        return self._dm

    def _stream(self):
        return torch.cuda.current_stream(self._dm.device).cuda_stream

    def _all_neumann(self):
        from . import boundary as B
        for var in self.varbs.values():
            k = var.resolved_bc.kind
            if np.any((k != B.G_NEUMANN) & (k != B.G_NONE)):
                return False
        return True

    def _q(self):
        return [self.varbs[k].dev("cell") for k in ("h", "hu", "hv", "hc", "Z")]

    def _state_key(self):
        return tuple(self.varbs[k].version("cell") for k in ("h", "hu", "hv"))

    def _dt_slot(self):
        """Device slot holding the dt of the current state (computed if stale)."""
        slot = self._dt_buf[self._cur:self._cur + 1]
        if self._dt_key != self._state_key():
            q = self._q()
            if "cell_vtx" in self._dm.t:
                # the fused step's own dt formula (the one it applies to later steps)
                _lib.call("mb_sw_dt", self._dm.struct, _p(q[0]), _p(q[1]), _p(q[2]), float(self.cfl),
                          float(self.grav), _p(slot), self._stream())
            else:
                _lib.call("mb_time_step_sw", self._dm.struct, _p(q[0]), _p(q[1]), _p(q[2]), float(self.cfl),
                          float(self.grav), float(self.Dxx), float(self.Dyy), _p(slot), self._stream())
            self._dt_key = self._state_key()
            self._dt_host = None
        return slot

    def stepper(self):
        """manapy/solvers/shallowater/system.py:186-192 (returns dt; manapy returns None)."""
        self._setup()
        slot = self._dt_slot()
        if self._dt_host is None:
            self._dt_host = float(slot.item())
        self.dt = self._dt_host
        return self.dt

    def update_ghost_values(self):
        for var in self.varbs.values():
            var.update_ghost_value()

    def explicit_convective(self):
        """manapy/solvers/shallowater/system.py:162-178 (unfused)."""
        self._setup()
        if self.order == 2:
            self.h.compute_cell_gradient()
            self.hc.compute_cell_gradient()
        names = ("h", "hu", "hv", "hc", "Z")
        rez = _lib.p5([_p(self.varbs[k].dev_out("convective")) for k in names])
        q = _lib.p5([_p(self.varbs[k].dev("cell")) for k in names])
        g = _lib.p5([_p(self.varbs[k].dev("ghost")) for k in names])
        gr = _lib.p4([_p(self.h.dev("gradcellx")), _p(self.h.dev("gradcelly")), _p(self.hc.dev("gradcellx")),
                      _p(self.hc.dev("gradcelly"))])
        _lib.call("mb_explicitscheme_convective_sw", self._dm.struct, rez, q, g, gr, _p(self.hc.dev("psi")),
                  float(self.grav), int(self.order), _p(self._ff), self._stream())

    def update_term_source(self):
        """manapy/solvers/shallowater/system.py:217-227."""
        self._setup()
        for v in (self.h, self.hc, self.Z):
            v.dev_out("source").zero_()
        _lib.call("mb_term_source_srnh_sw", self._dm.struct, _p(self.h.dev("cell")), _p(self.Z.dev("cell")),
                  _p(self.h.dev("ghost")), _p(self.Z.dev("ghost")), float(self.grav),
                  _p(self.hu.dev_out("source")), _p(self.hv.dev_out("source")), self._stream())

    def compute_fluxes(self):
        """manapy/solvers/shallowater/system.py:248-281; fused into compute_new_val() when
        every variable has manapy's default (Neumann) boundaries."""
        self._setup()
        self._fused = self._all_neumann()
        if not self._fused and self.walls != "neumann":
            raise NotImplementedError("reflective walls run in the fused step, which needs the variables' "
                                      "default (Neumann) boundaries")
        if not self._fused:
            self.stepper()
            self.update_ghost_values()
            self.explicit_convective()
            self.update_term_source()
        else:
            self.stepper()  # manapy evaluates the CFL step inside compute_fluxes

    def _use_dt(self):
        """The dt slot this step uses: the current state's dt, or S.dt if set by hand."""
        slot = self._dt_slot()
        if self._dt_host is not None and float(self.dt) != self._dt_host:
            slot.fill_(float(self.dt))
            self._dt_host = float(self.dt)
        return slot

    def compute_new_val(self):
        """manapy/solvers/shallowater/system.py:237-242."""
        self._setup()
        if getattr(self, "_fused", False):
            self._fused_step()
            self._fused = False
            return
        names = ("h", "hu", "hv", "hc", "Z")
        q = _lib.p5([_p(self.varbs[k].dev("cell")) for k in names])
        rez = _lib.p5([_p(self.varbs[k].dev("convective")) for k in names])
        dt = torch.tensor([float(self.dt)], dtype=torch.float64, device=self._dm.device)
        _lib.call("mb_update_sw", self._dm.struct, q, rez, _p(self.hu.dev("source")),
                  _p(self.hv.dev("source")), _p(dt), self._stream())
        for k in names:
            self.varbs[k]._s.version["cell"] += 1
        self._dt_key = None

    def _fused_step(self):
        if self.precision == "fp32c":
            return self._fused_step_f32c()
        names = ("h", "hu", "hv", "hc")
        qin = [self.varbs[k].dev("cell") for k in names]
        z = self.Z.dev("cell")
        if self._spare is None:
            self._spare = [torch.empty_like(t) for t in qin]
        qout = self._spare
        cur = self._use_dt()
        nxt = self._dt_buf[1 - self._cur:2 - self._cur]
        _lib.call("mb_sw_step_ex", self._dm.struct, _lib.p5([_p(t) for t in qin] + [_p(z)]),
                  _lib.p5([_p(t) for t in qout] + [_p(z)]), float(self.cfl), float(self.grav), int(self.order),
                  _lib.WALLS[self.walls], _p(self._scratch) if self._scratch is not None else None, _p(self._ff),
                  _p(cur), _p(nxt), self._stream())
        self._spare = [self.varbs[k].swap_cell(t) for k, t in zip(names, qout)]
        self._cur = 1 - self._cur
        self._dt_key = self._state_key()
        self._dt_host = None

    # ------------------------------------------------------------ fp32c mode
    _NAMES = ("h", "hu", "hv", "hc", "Z")

    def _keys(self):
        return tuple(self.varbs[k].version("cell") for k in self._NAMES)

    def _f32_state(self):
        """[h, hu, hv, hc] (current buffer) and Z in FP32, reloaded when a cell array changed."""
        dm = self._dm
        if self._q32 is None:
            mk = lambda: torch.empty(dm.nbcells, dtype=torch.float32, device=dm.device)  # noqa: E731
            self._q32 = [[mk() for _ in range(4)], [mk() for _ in range(4)], mk()]
            self._lo32 = [[mk() for _ in range(4)], [mk() for _ in range(4)]]  # rounding errors
            self._ff32 = torch.empty(4 * dm.nbfaces, dtype=torch.float32, device=dm.device)
        if self._keys() != self._q32_key:
            k = self._q32_i
            for c, name in enumerate(self._NAMES):
                w64 = self.varbs[name].dev("cell")
                t = self._q32[k][c] if c < 4 else self._q32[2]
                t.copy_(w64)
                if c < 4:
                    self._lo32[k][c].copy_(w64 - t.double())
            self._q32_key = self._keys()
        return self._q32[self._q32_i], self._q32[2]

    def _fused_step_f32c(self):
        qin, z = self._f32_state()
        qout = self._q32[1 - self._q32_i]
        cur = self._use_dt()
        nxt = self._dt_buf[1 - self._cur:2 - self._cur]
        k0 = self._q32_i
        _lib.call("mb_sw_step_f32c_ex", self._dm.struct, _lib.p5([_p(t) for t in qin] + [_p(z)]),
                  _lib.p5([_p(t) for t in qout] + [_p(z)]), _lib.p4([_p(t) for t in self._lo32[k0]]),
                  _lib.p4([_p(t) for t in self._lo32[1 - k0]]), float(self.cfl), float(self.grav), int(self.order),
                  _lib.WALLS[self.walls], _p(self._ff32), _p(cur), _p(nxt), self._stream())
        self._q32_i = 1 - k0
        for k, buf, lo in zip(self._NAMES[:4], qout, self._lo32[1 - k0]):
            var = self.varbs[k]

            def materialise(var=var, buf=buf, lo=lo):
                var._s.dev["cell"].copy_(buf.double() + lo.double())

            var._s.lazy.pop("cell", None)  # the previous result, superseded
            var._s.version["cell"] += 1
            var.set_lazy("cell", materialise)
        self._q32_key = self._keys()
        self._cur = 1 - self._cur
        self._dt_key = self._state_key()
        self._dt_host = None

    def check(self):
        """Raise if h, hu, hv or hc holds NaN or infinity, or h is negative (a dry-out the
        scheme does not handle; manapy lets both propagate)."""
        self._setup()
        if self.precision == "fp32c" and self._q32 is not None and self._keys() == self._q32_key:
            arrays = self._q32[self._q32_i]
        else:
            arrays = [self.varbs[k].dev("cell") for k in ("h", "hu", "hv", "hc")]
        check_state(arrays, nonneg=(0,), names=["h", "hu", "hv", "hc"])

    def mass(self):
        """FP64 sum of volume x h over the cells (no counterpart in manapy)."""
        dm = self._setup()
        if self.precision == "fp32c" and self._q32 is not None and self._keys() == self._q32_key:
            h = self._q32[self._q32_i][0].double() + self._lo32[self._q32_i][0].double()
        else:
            h = self.h.dev("cell")
        return float(torch.dot(h, dm.t["cell_volume"]).item())

    def boundary_mass_flux(self):
        """FP64 sum over the boundary faces of the h flux (outward, times the face length) of
        the last fused step, as that step applied it: the step changed the FP64 mass
        ``mass()`` by ``-dt * boundary_mass_flux()`` up to rounding, and by nothing up to
        rounding with reflective walls (no counterpart in manapy)."""
        dm = self._setup()
        if getattr(self, "_bfaces", None) is None:
            cid = dm.t["face_cellid"].view(-1, 2)
            self._bfaces = torch.nonzero(cid[:, 1] < 0).flatten()
        if self.precision == "fp32c" and self._q32 is not None:
            ff = self._ff32.view(-1, 4)[:, 0]
        else:
            ff = self._ff.view(-1)[:4 * dm.nbfaces].view(-1, 4)[:, 0]
        return float(ff.index_select(0, self._bfaces).double().sum().item())

    def launches_per_step(self):
        """Kernel launches of one fused step: face fluxes, cells (+ next dt), [gradients]."""
        return 2 + int(self.order == 2)

    def release_graphs(self):
        return None

    def advance(self, nsteps):
        """``nsteps`` fused steps on the device, without host synchronisation (each step's dt
        stays on the device)."""
        self._setup()
        if not self._all_neumann():
            raise NotImplementedError("advance() runs the fused step, which needs Neumann boundaries")
        for _ in range(int(nsteps)):
            self._fused_step()


class EulerSolver:
    """Compressible Euler equations in 2D, first-order Rusanov scheme, on the kernels of
    ``manapy/solvers/euler/fvm_utils2d.py`` (manapy ships them without a driver class).

    One step composes them as: Neumann ghosts (``ghost_value_Neumann``, :592), residuals
    (``explicitscheme_euler_2d_rusanov``, :1490), ``dt`` = the min over cells of
    ``time_step_euler_2d`` (:1083), then ``update_euler_2d_fvc`` (:1687).
    ``compute_new_val()`` / ``advance(n)`` run that step in two launches (every face flux once,
    then update per cell), bit-identical to the sequence; the next step's ``dt`` is reduced on
    the device in the update launch.  Every
    boundary keeps the default Neumann rule.  ``compute_fluxes()`` leaves the residuals in
    ``var.convective`` (rho, rhou, rhov, rhoE) and the ghosts in ``var.ghost``, as the
    unfused kernels produce them.
    """
    _parameters = [("cfl", float, .5, 0, "cfl of the explicit scheme"),
                   ("gamma", float, 1.4, 0, "ratio of specific heats"),
                   ("dt", float, 0., 0., "time step")]
    _NAMES = ("rho", "P", "rhou", "rhov", "rhoE")
    GRAPH_DEPTH = 24        # steps per CUDA-graph replay: a multiple of 6 (buffer pair x dt ring)

    @classmethod
    def process_conf(cls, conf, kwargs):
        return process_conf(cls._parameters, conf, kwargs)

    def __init__(self, rho=None, P=None, rhou=None, rhov=None, rhoE=None, conf=None, **kwargs):
        if conf is None:
            conf = Struct()
        self.conf = self.process_conf(conf, kwargs)
        get = make_get_conf(self.conf, kwargs)
        vs = dict(zip(self._NAMES, (rho, P, rhou, rhov, rhoE)))
        for k, v in vs.items():
            if not isinstance(v, Variable):
                raise ValueError("%s must be a Variable type" % k)
        self.domain = rho.domain
        if any(v.domain is not self.domain for v in vs.values()):
            raise ValueError("the five variables must live on one domain")
        self.dim = rho.dim
        if self.dim != 2:
            raise ValueError("the Euler Rusanov scheme is two-dimensional")
        self.varbs = vs
        for k in ("rho", "rhou", "rhov", "rhoE"):
            vs[k].add_term("convective")
        self.cfl = float(get("cfl"))
        self.gamma = float(get("gamma"))
        self.dt = float(get("dt"))
        self.backend = self.domain.backend
        self._dm = None
        self._graphs = {}

    # ------------------------------------------------------------ state
    def _setup(self):
        if self._dm is None:
            from . import boundary as B
            for k, v in self.varbs.items():
                kind = v.resolved_bc.kind
                if np.any((kind != B.G_NEUMANN) & (kind != B.G_NONE)):
                    raise NotImplementedError("Euler boundaries other than manapy's Neumann rule (%s)" % k)
            if np.any(np.asarray(self.domain.host_arrays["faces_name"]) == 10):
                raise NotImplementedError("halo faces: the Euler step runs on a single-rank mesh")
            dm = self._dm = self.domain.device_mesh
            f64 = torch.float64
            self._bufs = [[torch.empty(dm.nbcells, dtype=f64, device=dm.device) for _ in self._NAMES]
                          for _ in range(2)]
            self._ring = torch.full((3,), 1e300, dtype=f64, device=dm.device)
            self._time = torch.zeros(1, dtype=f64, device=dm.device)
            self._ff = torch.empty(4 * dm.nbfaces, dtype=f64, device=dm.device)   # face fluxes
            # static tables of the fused step: face records and left-cell bits
            self._frec = torch.empty(4 * dm.nbfaces, dtype=f64, device=dm.device)
            self._cleft = torch.empty(dm.nbcells, dtype=torch.uint8, device=dm.device)
            _lib.call("mb_euler_tables_2d", dm.struct, _p(self._frec), _p(self._cleft),
                      torch.cuda.current_stream(dm.device).cuda_stream)
            self._t = 0
            self._key = None
            self._dt_host = None
        return self._dm

    def _stream(self):
        return torch.cuda.current_stream(self._dm.device).cuda_stream

    def _versions(self):
        return tuple(self.varbs[k].version("cell") for k in self._NAMES)

    def _sync(self):
        """Make buffer set t%2 hold (and be) the variables' cell arrays, with the dt of that
        state in ring slot t%3."""
        self._setup()
        if self._key == self._versions():
            return
        cur = self._bufs[self._t % 2]
        for k, b in zip(self._NAMES, cur):
            t = self.varbs[k].dev("cell")
            if t.data_ptr() != b.data_ptr():
                b.copy_(t)
                self.varbs[k].swap_cell(b)
        _lib.call("mb_euler_dt_2d", self._dm.struct, _lib.p5([_p(b) for b in cur]), self.cfl, self.gamma,
                  _p(self._ring), int(self._t), self._stream())
        self._key = self._versions()
        self._dt_host = None

    def _slot(self):
        return self._ring[self._t % 3:self._t % 3 + 1]

    def stepper(self):
        """dt of the current state: the min over cells of time_step_euler_2d."""
        self._sync()
        if self._dt_host is None:
            self._dt_host = float(self._slot().item())
        self.dt = self._dt_host
        return self.dt

    @property
    def time(self):
        """Simulated time: the sum of the dt of every step taken (device accumulator)."""
        self._setup()
        return float(self._time.item())

    # ------------------------------------------------------------ the unfused kernels
    def update_ghost_values(self):
        """ghost_value_Neumann into var.ghost of the five variables."""
        self._sync()
        nf = self._dm.nbfaces
        uv = torch.empty(2 * nf, dtype=torch.float64, device=self._dm.device)
        _lib.call("mb_ghost_euler_neumann_2d", self._dm.struct,
                  _lib.p5([_p(self.varbs[k].dev("cell")) for k in self._NAMES]),
                  _lib.p5([_p(self.varbs[k].dev_out("ghost")) for k in self._NAMES]), _p(uv[:nf]), _p(uv[nf:]),
                  self._stream())

    def compute_fluxes(self):
        """Neumann ghosts, then the Rusanov residuals into var.convective."""
        self.update_ghost_values()
        _lib.call("mb_euler_rusanov_2d", self._dm.struct,
                  _lib.p5([_p(self.varbs[k].dev("cell")) for k in self._NAMES]),
                  _lib.p5([_p(self.varbs[k].dev("ghost")) for k in self._NAMES]),
                  _lib.p4([_p(self.varbs[k].dev_out("convective")) for k in ("rho", "rhou", "rhov", "rhoE")]),
                  self.gamma, self._stream())

    # ------------------------------------------------------------ fused step
    def _launch(self, t):
        a, b = self._bufs[t % 2], self._bufs[(t + 1) % 2]
        _lib.call("mb_euler_step_2d", self._dm.struct, _lib.p5([_p(x) for x in a]), _lib.p5([_p(x) for x in b]),
                  self.cfl, self.gamma, _p(self._frec), _p(self._cleft), _p(self._ff), _p(self._ring), int(t),
                  _p(self._time), self._stream())

    def _publish(self):
        for k, b in zip(self._NAMES, self._bufs[self._t % 2]):
            self.varbs[k].swap_cell(b)
        self._key = self._versions()
        self._dt_host = None

    def compute_new_val(self):
        """One step.  dt is the state's CFL dt, or ``self.dt`` when it was assigned after
        ``stepper()`` returned (manapy's solvers step with ``self.dt``)."""
        self._sync()
        if self._dt_host is not None and float(self.dt) != self._dt_host:
            self._slot().fill_(float(self.dt))
        self._launch(self._t)
        self._t += 1
        self._publish()

    def advance(self, n, graph=False):
        """``n`` fused steps on the device without host synchronisation (CUDA-graph replays of
        GRAPH_DEPTH steps when ``graph``)."""
        self._sync()
        n = int(n)
        D = self.GRAPH_DEPTH
        while n > 0:
            if graph and n >= D and self._t % 6 == 0:
                g = self._graphs.get("main")
                if g is None:
                    s = torch.cuda.Stream(self._dm.device)
                    s.wait_stream(torch.cuda.current_stream(self._dm.device))
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g, stream=s):
                        for k in range(D):
                            self._launch(k)
                    torch.cuda.current_stream(self._dm.device).wait_stream(s)
                    self._graphs["main"] = g
                g.replay()
                self._t += D
                n -= D
            else:
                self._launch(self._t)
                self._t += 1
                n -= 1
        self._publish()

    def release_graphs(self):
        self._graphs.clear()

    def check(self):
        """Raise if a variable holds NaN or infinity, or rho or P is negative."""
        self._sync()
        check_state([self.varbs[k].dev("cell") for k in self._NAMES], nonneg=(0, 1), names=list(self._NAMES))

    def launches_per_step(self):
        return 2
