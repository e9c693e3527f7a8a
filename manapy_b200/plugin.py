"""CUDA implementations behind ``CUDABackend.compile`` with manapy's argument lists.

Each entry binds a manapy kernel name to its C-ABI implementation.  The
callable takes exactly manapy's positional (or keyword) arguments, e.g.
``explicitscheme_convective_2d(rez_w, w_c, w_ghost, ..., shift, order)``
(``manapy/solvers/advecdiff/fvm_utils.py:43-50``):

* field arguments (cell, face or node arrays) are uploaded, permuted into the
  device numbering;
* mesh-table arguments (``centerc``, ``cellidf``, ``normalf`` ...) are not
  transferred: the kernel reads the domain's own device tables.  They are
  checked for the domain's sizes, and must be that domain's arrays;
* output arrays are written back in place, in manapy's numbering;
* scalar results (``time_step``) are returned.

Halo and periodic arguments are accepted and must be empty or unused, as on a
single rank without periodic boundaries.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from . import boundary as B

KERNELS = {}


class _Spec:
    def __init__(self, params, fields, outputs, run, sizes=None):
        self.params = params          # manapy's parameter names, in order
        self.fields = fields          # name -> "cell" | "face" | "node": uploaded inputs
        self.outputs = outputs        # name -> kind: written back in place
        self.run = run                # run(ctx, dev_arrays, scalars) -> optional return value
        self.sizes = sizes or {}      # name -> "cell" | "face" | "node": mesh tables, size-checked


class _Ctx:
    def __init__(self, domain):
        self.domain = domain
        self.dm = domain.device_mesh
        self.stream = torch.cuda.current_stream(self.dm.device).cuda_stream

    def n(self, kind):
        return {"cell": self.dm.nbcells, "face": self.dm.nbfaces, "node": self.dm.nbnodes}[kind]

    def upload(self, kind, a):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
        if len(a) != self.n(kind):
            raise ValueError("%s array of length %d, expected %d" % (kind, len(a), self.n(kind)))
        src = torch.from_numpy(a).to(self.dm.device)
        out = torch.empty_like(src)
        self.dm.to_device_order(kind, src, out)
        return out

    def zeros(self, kind):
        return torch.zeros(self.n(kind), dtype=torch.float64, device=self.dm.device)

    def download(self, kind, t, into):
        h = self.dm.to_host_order(kind, t).cpu().numpy()
        np.copyto(into, h.reshape(np.shape(into)), casting="unsafe")

    def face_mask(self, *lists):
        on = np.zeros(self.dm.nbfaces, dtype=np.uint8)
        for lst in lists:
            lst = np.asarray(lst, dtype=np.int64).reshape(-1)
            if len(lst):
                on[lst] = 1
        return torch.from_numpy(on[self.dm.R.fperm]).to(self.dm.device)


def _p(t):
    return t.data_ptr()


def bind(spec, domain, name):
    params = spec.params

    def call(*args, **kwargs):
        if len(args) > len(params):
            raise TypeError("%s takes %d arguments, got %d" % (name, len(params), len(args)))
        vals = dict(zip(params, args))
        for k, v in kwargs.items():
            if k not in params:
                raise TypeError("%s got an unexpected argument %r" % (name, k))
            vals[k] = v
        missing = [p for p in params if p not in vals]
        if missing:
            raise TypeError("%s missing arguments: %s" % (name, ", ".join(missing)))
        ctx = _Ctx(domain)
        for k, kind in spec.sizes.items():
            if len(np.asarray(vals[k])) != ctx.n(kind):
                raise ValueError("%s: argument %r does not belong to this domain (%d rows, expected %d)"
                                 % (name, k, len(np.asarray(vals[k])), ctx.n(kind)))
        dev = {}
        for k, kind in spec.fields.items():
            dev[k] = ctx.upload(kind, vals[k])
        for k, kind in spec.outputs.items():
            if k not in dev:
                # outputs that manapy only partly overwrites start from the caller's contents
                dev[k] = ctx.upload(kind, vals[k])
        ret = spec.run(ctx, dev, vals)
        for k, kind in spec.outputs.items():
            ctx.download(kind, dev[k], vals[k])
        return ret

    call.__name__ = name
    call.__doc__ = "CUDA implementation of manapy's %s(%s)" % (name, ", ".join(params))
    return call


def _register(names, spec):
    for n in names:
        KERNELS[n] = spec


# ---------------------------------------------------------------- manapy/ast/ast_utils.py:8-18
_register(["facetocell"], _Spec(
    ["u_face", "u_c", "faceidc", "dim"], {"u_face": "face"}, {"u_c": "cell"},
    lambda c, d, v: _lib.call("mb_facetocell", c.dm.struct, _p(d["u_face"]), _p(d["u_c"]), c.stream),
    sizes={"faceidc": "cell"}))

# ---------------------------------------------------------------- manapy/ast/functions2d.py:5, functions3d.py:4
_CG = ["w_c", "w_ghost", "w_halo", "w_haloghost", "centerc", "cellnid", "ghostnid", "haloghostnid", "halonid",
       "nodecid", "periodicn", "periodic", "centergf", "halocenterg", "vertexn", "centerh", "shift",
       "w_x", "w_y", "w_z"]
_register(["cell_gradient_2d", "cell_gradient_3d"], _Spec(
    _CG, {"w_c": "cell", "w_ghost": "face"}, {"w_x": "cell", "w_y": "cell", "w_z": "cell"},
    lambda c, d, v: _lib.call("mb_cell_gradient", c.dm.struct, _p(d["w_c"]), _p(d["w_ghost"]), _p(d["w_x"]),
                              _p(d["w_y"]), _p(d["w_z"]), c.stream),
    sizes={"centerc": "cell", "cellnid": "cell", "vertexn": "node"}))

# ---------------------------------------------------------------- manapy/ast/functions2d.py:280, functions3d.py:364
_BL = ["w_c", "w_ghost", "w_halo", "w_x", "w_y", "w_z", "psi", "cellid", "faceid", "namef", "halofid",
       "centerc", "centerf"]
_register(["barthlimiter_2d", "barthlimiter_3d"], _Spec(
    _BL, {"w_c": "cell", "w_ghost": "face", "w_x": "cell", "w_y": "cell", "w_z": "cell"}, {"psi": "cell"},
    lambda c, d, v: _lib.call("mb_barthlimiter", c.dm.struct, _p(d["w_c"]), _p(d["w_ghost"]), _p(d["w_x"]),
                              _p(d["w_y"]), _p(d["w_z"]), _p(d["psi"]), c.stream),
    sizes={"cellid": "face", "faceid": "cell", "centerc": "cell", "centerf": "face"}))

# ---------------------------------------------------------------- manapy/ast/functions2d.py:199, functions3d.py:251
_CV = ["w_c", "w_ghost", "w_halo", "w_haloghost", "centerc", "centerh", "cellid", "ghostid", "haloghostid",
       "periodicid", "haloid", "vertexn", "centergf", "halocenterg", "R_x", "R_y", "R_z", "lambda_x",
       "lambda_y", "lambda_z", "number", "shift", "w_n"]
_register(["centertovertex_2d", "centertovertex_3d"], _Spec(
    _CV, {"w_c": "cell", "w_ghost": "face"}, {"w_n": "node"},
    lambda c, d, v: _lib.call("mb_centertovertex", c.dm.struct, _p(d["w_c"]), _p(d["w_ghost"]), _p(d["w_n"]),
                              c.stream),
    sizes={"centerc": "cell", "cellid": "node", "vertexn": "node", "R_x": "node"}))


# ---------------------------------------------------------------- manapy/ast/functions2d.py:108, functions3d.py:122
def _face_gradient(c, d, v):
    on = c.face_mask(v["innerfaces"], v["halofaces"], v["dirichletfaces"], v["neumann"], v["periodicfaces"])
    bc = _lib.MbBC()
    bc.face_grad_on = on.data_ptr()
    _lib.call("mb_face_gradient", c.dm.struct, bc, _p(d["w_c"]), _p(d["w_ghost"]), _p(d["w_node"]),
              _p(d["wx_face"]), _p(d["wy_face"]), _p(d["wz_face"]), c.stream)
    torch.cuda.current_stream(c.dm.device).synchronize()  # keep `on` alive until the kernel ran


_FG = ["w_c", "w_ghost", "w_halo", "w_node", "cellidf", "nodeidf", "centergf", "halofid", "centerc", "centerh",
       "vertexn", "airDiamond", "normalf", "f_1", "f_2", "f_3", "f_4", "shift", "wx_face", "wy_face", "wz_face",
       "innerfaces", "halofaces", "dirichletfaces", "neumann", "periodicfaces"]
_register(["face_gradient_2d", "face_gradient_3d"], _Spec(
    _FG, {"w_c": "cell", "w_ghost": "face", "w_node": "node"},
    {"wx_face": "face", "wy_face": "face", "wz_face": "face"}, _face_gradient,
    sizes={"cellidf": "face", "nodeidf": "face", "centerc": "cell", "vertexn": "node"}))

# ---------------------------------------------------------------- manapy/solvers/advecdiff/fvm_utils.py:43, :180
_EC = ["rez_w", "w_c", "w_ghost", "w_halo", "u_face", "v_face", "w_face", "w_x", "w_y", "w_z", "wx_halo",
       "wy_halo", "wz_halo", "psi", "psi_halo", "centerc", "centerf", "centerh", "centerg", "cellidf", "normalf",
       "halofid", "name", "innerfaces", "halofaces", "boundaryfaces", "periodicboundaryfaces", "shift", "order"]
_register(["explicitscheme_convective_2d", "explicitscheme_convective_3d"], _Spec(
    _EC, {"w_c": "cell", "w_ghost": "face", "u_face": "face", "v_face": "face", "w_face": "face",
          "w_x": "cell", "w_y": "cell", "w_z": "cell", "psi": "cell"}, {"rez_w": "cell"},
    lambda c, d, v: _lib.call("mb_explicitscheme_convective", c.dm.struct, _p(d["rez_w"]), _p(d["w_c"]),
                              _p(d["w_ghost"]), _p(d["u_face"]), _p(d["v_face"]), _p(d["w_face"]), _p(d["w_x"]),
                              _p(d["w_y"]), _p(d["w_z"]), _p(d["psi"]), int(v["order"]), c.stream),
    sizes={"centerc": "cell", "centerf": "face", "cellidf": "face", "normalf": "face"}))

# ---------------------------------------------------------------- manapy/solvers/advecdiff/fvm_utils.py:5
_register(["explicitscheme_dissipative"], _Spec(
    ["wx_face", "wy_face", "wz_face", "cellidf", "normalf", "namef", "dissip_w", "Dxx", "Dyy", "Dzz"],
    {"wx_face": "face", "wy_face": "face", "wz_face": "face"}, {"dissip_w": "cell"},
    lambda c, d, v: _lib.call("mb_explicitscheme_dissipative", c.dm.struct, _p(d["wx_face"]), _p(d["wy_face"]),
                              _p(d["wz_face"]), _p(d["dissip_w"]), float(v["Dxx"]), float(v["Dyy"]),
                              float(v["Dzz"]), c.stream),
    sizes={"cellidf": "face", "normalf": "face"}))


# ---------------------------------------------------------------- manapy/solvers/advecdiff/fvm_utils.py:317
def _time_step(c, d, v):
    dt = torch.zeros(1, dtype=torch.float64, device=c.dm.device)
    _lib.call("mb_time_step", c.dm.struct, _p(d["u"]), _p(d["v"]), _p(d["w"]), float(v["cfl"]), float(v["Dxx"]),
              float(v["Dyy"]), float(v["Dzz"]), _p(dt), c.stream)
    return float(dt.item())


_register(["time_step"], _Spec(
    ["u", "v", "w", "cfl", "normal", "mesure", "volume", "faceid", "dim", "Dxx", "Dyy", "Dzz"],
    {"u": "cell", "v": "cell", "w": "cell"}, {}, _time_step,
    sizes={"normal": "face", "volume": "cell", "faceid": "cell"}))


# ---------------------------------------------------------------- manapy/solvers/advecdiff/fvm_utils.py:342
def _update(c, d, v):
    dt = torch.tensor([float(v["dtime"])], dtype=torch.float64, device=c.dm.device)
    _lib.call("mb_update_new_value", c.dm.struct, _p(d["ne_c"]), _p(d["rez_ne"]), _p(d["dissip_ne"]),
              _p(d["src_ne"]), _p(dt), c.stream)
    torch.cuda.current_stream(c.dm.device).synchronize()


_register(["update_new_value"], _Spec(
    ["ne_c", "rez_ne", "dissip_ne", "src_ne", "dtime", "vol"],
    {"ne_c": "cell", "rez_ne": "cell", "dissip_ne": "cell", "src_ne": "cell"}, {"ne_c": "cell"}, _update,
    sizes={"vol": "cell"}))


# ---------------------------------------------------------------- manapy/boundary/bc_utils.py:45-68
def _ghost(kind):
    def run(c, d, v):
        faces = np.asarray(v["faces"], dtype=np.int64).reshape(-1)
        nf = c.dm.nbfaces
        k = np.zeros(nf, dtype=np.int8)
        val = np.zeros(nf)
        k[faces] = kind
        if kind == B.G_DIRICHLET:
            val[faces] = np.asarray(v["value"], dtype=np.float64).reshape(-1)[faces]
        elif kind == B.G_NEUMANN_NH:
            val[faces] = np.asarray(v["cst"], dtype=np.float64).reshape(-1)[faces]
        fp = c.dm.R.fperm
        kt = torch.from_numpy(k[fp]).to(c.dm.device)
        vt = torch.from_numpy(val[fp]).to(c.dm.device)
        bc = _lib.MbBC()
        bc.kind, bc.value = kt.data_ptr(), vt.data_ptr()
        w_c = d["w_c"]
        _lib.call("mb_ghost_value", c.dm.struct, bc, _p(w_c), _p(d["w_ghost"]), c.stream)
        torch.cuda.current_stream(c.dm.device).synchronize()
    return run


for _name, _kind, _first in (("ghost_value_dirichlet", B.G_DIRICHLET, "value"),
                             ("ghost_value_neumann", B.G_NEUMANN, "w_c"),
                             ("ghost_value_nonslip", B.G_NONSLIP, "w_c"),
                             ("ghost_value_neumannNH", B.G_NEUMANN_NH, "w_c")):
    _fields = {"w_c": "cell"} if _first == "w_c" else {}
    _spec = _Spec([_first, "w_ghost", "cellid", "faces", "cst", "dist"], _fields, {"w_ghost": "face"},
                  _ghost(_kind), sizes={"cellid": "face"})
    if _first == "value":
        # a dirichlet rule reads no cell values; give the kernel a valid (unused) cell array
        _orig = _spec.run

        def _run(c, d, v, _orig=_orig):
            d["w_c"] = c.zeros("cell")
            return _orig(c, d, v)
        _spec.run = _run
    _register([_name], _spec)


# ---------------------------------------------------------------- manapy/solvers/shallowater/fvm_utils.py:16
def _time_step_sw(c, d, v):
    dt = torch.zeros(1, dtype=torch.float64, device=c.dm.device)
    _lib.call("mb_time_step_sw", c.dm.struct, _p(d["h_c"]), _p(d["hu_c"]), _p(d["hv_c"]), float(v["cfl"]),
              float(v["grav"]), float(v["Dxx"]), float(v["Dyy"]), _p(dt), c.stream)
    return float(dt.item())


_register(["time_step_SW"], _Spec(
    ["h_c", "hu_c", "hv_c", "cfl", "normal", "mesure", "volume", "faceid", "grav", "Dxx", "Dyy"],
    {"h_c": "cell", "hu_c": "cell", "hv_c": "cell"}, {}, _time_step_sw,
    sizes={"normal": "face", "volume": "cell", "faceid": "cell"}))

# ---------------------------------------------------------------- manapy/solvers/shallowater/fvm_utils.py:344
_SWQ = ["h", "hu", "hv", "hc", "Z"]
_ESW = (["rez_h", "rez_hu", "rez_hv", "rez_hc", "rez_Z"] + [q + "_c" for q in _SWQ] + [q + "_ghost" for q in _SWQ]
        + [q + "_halo" for q in _SWQ] + ["h_x", "h_y", "hx_halo", "hy_halo", "hc_x", "hc_y", "hcx_halo",
                                         "hcy_halo", "psi", "psi_halo", "centerc", "centerf", "centerh", "centerg",
                                         "cellidf", "mesuref", "normalf", "halofid", "innerfaces", "halofaces",
                                         "boundaryfaces", "grav", "order"])


def _conv_sw(c, d, v):
    ff = torch.zeros(5 * c.dm.nbfaces, dtype=torch.float64, device=c.dm.device)
    _lib.call("mb_explicitscheme_convective_sw", c.dm.struct,
              _lib.p5([_p(d["rez_" + q]) for q in _SWQ]), _lib.p5([_p(d[q + "_c"]) for q in _SWQ]),
              _lib.p5([_p(d[q + "_ghost"]) for q in _SWQ]),
              _lib.p4([_p(d[k]) for k in ("h_x", "h_y", "hc_x", "hc_y")]), _p(d["psi"]), float(v["grav"]),
              int(v["order"]), _p(ff), c.stream)
    torch.cuda.current_stream(c.dm.device).synchronize()


_register(["explicitscheme_convective_SW"], _Spec(
    _ESW, dict([(q + "_c", "cell") for q in _SWQ] + [(q + "_ghost", "face") for q in _SWQ]
               + [(k, "cell") for k in ("h_x", "h_y", "hc_x", "hc_y", "psi")]),
    {"rez_" + q: "cell" for q in _SWQ}, _conv_sw,
    sizes={"centerc": "cell", "centerf": "face", "cellidf": "face", "normalf": "face"}))

# ---------------------------------------------------------------- manapy/solvers/shallowater/fvm_utils.py:44
_TS = (["src_" + q for q in _SWQ] + [q + "_c" for q in _SWQ] + [q + "_ghost" for q in _SWQ]
       + [q + "_halo" for q in _SWQ] + ["h_x", "h_y", "psi", "hx_halo", "hy_halo", "psi_halo", "nodeidc",
                                        "faceidc", "cellidc", "cellidf", "centerc", "normalc", "namef",
                                        "centerf", "centerh", "vertexn", "halofid", "grav", "order"])


def _source_sw(c, d, v):
    for q in ("h", "hc", "Z"):
        d["src_" + q].zero_()
    _lib.call("mb_term_source_srnh_sw", c.dm.struct, _p(d["h_c"]), _p(d["Z_c"]), _p(d["h_ghost"]),
              _p(d["Z_ghost"]), float(v["grav"]), _p(d["src_hu"]), _p(d["src_hv"]), c.stream)


_register(["term_source_srnh_SW"], _Spec(
    _TS, {"h_c": "cell", "Z_c": "cell", "h_ghost": "face", "Z_ghost": "face"},
    {"src_" + q: "cell" for q in _SWQ}, _source_sw,
    sizes={"nodeidc": "cell", "faceidc": "cell", "centerc": "cell", "vertexn": "node"}))


# ---------------------------------------------------------------- manapy/solvers/shallowater/fvm_utils.py:3
def _update_sw(c, d, v):
    for k in ("corio_hu", "corio_hv", "dissip_hc", "src_h", "src_hc", "src_Z"):
        if np.any(np.asarray(v[k])):
            raise NotImplementedError("update_SW with non-zero %s is not implemented" % k)
    if float(v["wind_hu"]) != 0 or float(v["wind_hv"]) != 0:
        raise NotImplementedError("update_SW with wind is not implemented")
    dt = torch.tensor([float(v["dtime"])], dtype=torch.float64, device=c.dm.device)
    _lib.call("mb_update_sw", c.dm.struct, _lib.p5([_p(d[q + "_c"]) for q in _SWQ]),
              _lib.p5([_p(d["rez_" + q]) for q in _SWQ]), _p(d["src_hu"]), _p(d["src_hv"]), _p(dt), c.stream)
    torch.cuda.current_stream(c.dm.device).synchronize()


_register(["update_SW"], _Spec(
    [q + "_c" for q in _SWQ] + ["rez_" + q for q in _SWQ] + ["src_" + q for q in _SWQ]
    + ["dissip_hc", "corio_hu", "corio_hv", "wind_hu", "wind_hv", "dtime", "vol"],
    dict([(q + "_c", "cell") for q in _SWQ] + [("rez_" + q, "cell") for q in _SWQ]
         + [("src_hu", "cell"), ("src_hv", "cell")]),
    {q + "_c": "cell" for q in _SWQ}, _update_sw, sizes={"vol": "cell"}))


# ---------------------------------------------------------------- manapy/solvers/euler/fvm_utils2d.py (2D Euler)
_EQ = ["rho", "P", "rhou", "rhov", "rhoE"]
_EC = [q for q in _EQ if q != "P"]          # conserved: the residual components


def _euler_rusanov(c, d, v):
    _lib.call("mb_euler_rusanov_2d", c.dm.struct, _lib.p5([_p(d[q + "_c"]) for q in _EQ]),
              _lib.p5([_p(d[q + "_g"]) for q in _EQ]), _lib.p4([_p(d["rez_" + q]) for q in _EC]),
              float(v["gamma"]), c.stream)
    torch.cuda.current_stream(c.dm.device).synchronize()


# fvm_utils2d.py:1490 (halo arrays accepted, unused on a single rank)
_register(["explicitscheme_euler_2d_rusanov"], _Spec(
    ["rez_" + q for q in _EC] + [q + "_c" for q in _EQ] + [q + "_g" for q in _EQ] + [q + "_h" for q in _EQ]
    + ["cellidf", "halofid", "normal", "mesurf", "name", "gamma"],
    dict([(q + "_c", "cell") for q in _EQ] + [(q + "_g", "face") for q in _EQ]),
    {"rez_" + q: "cell" for q in _EC}, _euler_rusanov,
    sizes={"cellidf": "face", "normal": "face", "mesurf": "face", "name": "face"}))


def _time_step_euler(c, d, v):
    # reads rho, P, rhou, rhov; the fifth pointer is unused
    _lib.call("mb_time_step_euler_2d", c.dm.struct, _lib.p5([_p(d[q]) for q in _EQ[:4]] + [_p(d["rho"])]),
              float(v["cfl"]), float(v["gamma"]), _p(d["dt_c"]), c.stream)
    torch.cuda.current_stream(c.dm.device).synchronize()


# fvm_utils2d.py:1083
_register(["time_step_euler_2d"], _Spec(
    ["rho", "P", "rhou", "rhov", "cfl", "normal", "mesure", "volume", "faceid", "gamma", "dt_c"],
    {q: "cell" for q in _EQ[:4]}, {"dt_c": "cell"}, _time_step_euler,
    sizes={"normal": "face", "mesure": "face", "volume": "cell", "faceid": "cell"}))


def _update_euler(c, d, v):
    _lib.call("mb_update_euler_2d", c.dm.struct, _lib.p5([_p(d[q + "_c"]) for q in _EQ]),
              _lib.p4([_p(d["rez_" + q]) for q in _EC]), float(v["gamma"]), float(v["dtime"]), c.stream)
    torch.cuda.current_stream(c.dm.device).synchronize()


# fvm_utils2d.py:1687
_register(["update_euler_2d_fvc"], _Spec(
    [q + "_c" for q in _EQ] + ["rez_" + q for q in _EC] + ["gamma", "dtime", "vol"],
    dict([(q + "_c", "cell") for q in _EQ] + [("rez_" + q, "cell") for q in _EC]),
    {q + "_c": "cell" for q in _EQ}, _update_euler, sizes={"vol": "cell"}))


def _ghost_euler(c, d, v):
    _lib.call("mb_ghost_euler_neumann_2d", c.dm.struct, _lib.p5([_p(d[q + "c"]) for q in _EQ]),
              _lib.p5([_p(d[q + "g"]) for q in _EQ]), _p(d["ug"]), _p(d["vg"]), c.stream)
    torch.cuda.current_stream(c.dm.device).synchronize()


# fvm_utils2d.py:592 (faces named 1-4 are written; the others keep the caller's values)
_register(["ghost_value_Neumann"], _Spec(
    ["rhog", "Pg", "rhoug", "rhovg", "ug", "vg", "rhoEg", "rhoc", "Pc", "rhouc", "rhovc", "rhoEc", "cellid", "name",
     "normal", "mesure", "center", "t"],
    {q + "c": "cell" for q in _EQ}, dict([(q + "g", "face") for q in _EQ] + [("ug", "face"), ("vg", "face")]),
    _ghost_euler, sizes={"cellid": "face", "name": "face", "normal": "face", "mesure": "face", "center": "face"}))
