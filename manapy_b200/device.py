"""Device-resident mesh tables and ghost rules (the ``mb_mesh`` / ``mb_bc`` of the C ABI).

``DeviceMesh`` turns the host arrays of ``geometry.build`` into the tables the
kernels read: SoA geometry, CSR neighbour lists, per-cell face slots with the
order manapy accumulates them in, and precomputed centre->vertex weights.
Device memory comes from torch tensors (the allocator is plumbing only); the
kernels are called through the C ABI with their raw pointers.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .geometry import padded_from_csr  # noqa: F401  (re-export for callers)


def _t(a, dtype, dev):
    """A table as a contiguous array of ``dtype``: numpy when ``dev`` is None (built on the
    host for a later upload), else a tensor on ``dev``."""
    a = np.ascontiguousarray(a, dtype=dtype)
    return a if dev is None else torch.from_numpy(a).to(dev)


def _upload(a, dev, stream):
    t = torch.from_numpy(a)
    if stream is None:
        return t.to(dev)
    with torch.cuda.stream(stream):
        return t.pin_memory().to(dev, non_blocking=True)


_TORCH_DT = {np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64, np.dtype(np.float64): torch.float64,
             np.dtype(np.float32): torch.float32, np.dtype(np.uint8): torch.uint8, np.dtype(np.int8): torch.int8}


def staged_nbytes(arrays):
    return sum((int(a.nbytes) + 255) // 256 * 256 for a in arrays.values())


def stage_upload(arrays, device, stream, staging):
    """Host arrays to ``device`` with one copy: packed at 256-byte aligned offsets into the
    pinned byte tensor ``staging`` (the caller keeps it unused until the copy on ``stream``
    has run), copied into one device buffer on ``stream``; returns (views by name, buffer)."""
    layout, off = [], 0
    for k, a in arrays.items():
        a = np.ascontiguousarray(a)
        layout.append((k, a, off))
        off += (a.nbytes + 255) // 256 * 256
    if staging.numel() < off:
        raise ValueError("staging buffer too small: %d < %d bytes" % (staging.numel(), off))
    host = staging.numpy()
    for k, a, o in layout:
        host[o:o + a.nbytes] = a.reshape(-1).view(np.uint8)
    with torch.cuda.stream(stream):
        buf = torch.empty(max(off, 1), dtype=torch.uint8, device=device)
        buf.copy_(staging[:max(off, 1)], non_blocking=True)
    views = {k: buf[o:o + a.nbytes].view(_TORCH_DT[a.dtype]).view(a.shape) for k, a, o in layout}
    return views, buf


def cell_order_codes(faceid_local):
    """uint8 per cell: slot visited k-th in ascending face id, 2 bits per k."""
    order = np.argsort(faceid_local, axis=1, kind="stable").astype(np.uint32)
    code = np.zeros(len(order), dtype=np.uint32)
    for k in range(order.shape[1]):
        code |= order[:, k] << (2 * k)
    return code.astype(np.uint8)


def sell32(ptr, idx, vals=None, fill=-1):
    """SELL-32 layout of a CSR table: rows in groups of 32, each group stored
    [longest row][32] so entry k of the 32 rows is contiguous.  Padding is -1,
    or each row's first entry with ``fill="first"`` (padding values are 0).
    Returns (group_ptr, idx_sell, vals_sell)."""
    ptr = np.asarray(ptr, dtype=np.int64)
    n = len(ptr) - 1
    ng = (n + 31) // 32
    cnt = np.zeros(ng * 32, dtype=np.int64)
    cnt[:n] = np.diff(ptr)
    glen = cnt.reshape(ng, 32).max(axis=1)
    gptr = np.zeros(ng + 1, dtype=np.int64)
    np.cumsum(glen * 32, out=gptr[1:])
    row = np.repeat(np.arange(n), np.diff(ptr))
    k = np.arange(len(idx)) - np.repeat(ptr[:-1], np.diff(ptr))
    dest = gptr[row // 32] + k * 32 + (row % 32)
    if fill != "first":
        out = np.full(int(gptr[-1]), fill, dtype=np.int32)
    else:
        # pad each row with its own first entry (callers give such entries a zero weight)
        first = np.zeros(ng * 32, dtype=np.int64)
        nz = np.diff(ptr) > 0
        first[:n][nz] = np.asarray(idx)[ptr[:-1][nz]]
        slot = np.arange(int(gptr[-1]))
        g = np.searchsorted(gptr, slot, side="right") - 1
        out = first[g * 32 + (slot - gptr[g]) % 32].astype(np.int32)
    out[dest] = idx
    outv = None
    if vals is not None:
        outv = np.zeros(int(gptr[-1]), dtype=np.float64)
        outv[dest] = vals
    if gptr[-1] >= 2 ** 31:
        raise ValueError("neighbour table too large for 32-bit offsets")
    return gptr.astype(np.int32), out, outv


STENCILS = ("shared", "manapy")


def lsq_sell(ptr, idx, stencil):
    """(group_ptr, idx) of the least-squares stencil (vertex neighbours of every cell) in
    SELL-32.  ``"manapy"``: each row keeps manapy's neighbour order, padded with -1 at its
    end, so a cell's sums are formed in the same order whatever the numbering of the other
    cells.  ``"shared"``: a neighbour held by several cells of one warp is placed in the
    same slot for all of them where their free slots allow (``native.sell_aligned``), so a
    warp-wide gather touches fewer distinct rows; each cell's sums are then formed in slot
    order, which depends on the cells it shares a warp with (results differ from the
    ``"manapy"`` layout by rounding)."""
    if stencil == "manapy":
        gp, gi, _ = sell32(ptr, idx)
        return gp, gi
    if stencil == "shared":
        from . import native
        return native.sell_aligned(ptr, idx)
    raise ValueError("stencil must be one of %s" % (STENCILS,))


def vertex_weights(A):
    """Centre->vertex weight of every node->cell and node->ghost incidence, in
    manapy's expression order (manapy/ast/functions2d.py:219, functions3d.py:272-274)."""
    dim = A["dim"]
    vx = A["nodes_vertex"]
    lx, ly, lz = A["nodes_lambda_x"], A["nodes_lambda_y"], A["nodes_lambda_z"]
    Rx, Ry, Rz = A["nodes_R_x"], A["nodes_R_y"], A["nodes_R_z"]
    num = A["nodes_number"].astype(np.float64)
    if dim == 2:
        den = num + lx * Rx + ly * Ry
    else:
        den = num + lx * Rx + ly * Ry + lz * Rz

    def alpha(ptr, pts):
        node = np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))
        xd = pts[:, 0] - vx[node, 0]
        yd = pts[:, 1] - vx[node, 1]
        if dim == 2:
            num_ = 1. + lx[node] * xd + ly[node] * yd
        else:
            zd = pts[:, 2] - vx[node, 2]
            num_ = 1. + lx[node] * xd + ly[node] * yd + lz[node] * zd
        return num_ / den[node]

    a_c = alpha(A["n2c_ptr"], A["cells_center"][A["n2c_idx"]])
    a_g = alpha(A["n2g_ptr"], A["faces_ghostcenter"][A["n2g_idx"], :3])
    return a_c, a_g


class DeviceMesh:
    """All mesh tables on one CUDA device plus the ``mb_mesh`` struct pointing at them.

    With ``reorder=True`` (the default) the tables use the locality numbering of
    ``reorder.Renumbering``; ``to_device_order`` / ``to_host_order`` move field
    arrays between that numbering and manapy's.
    """

    def __init__(self, A, device="cuda", reorder=True, stencil="shared", first_cells=None):
        """``device=None`` builds the tables as numpy arrays on the host (``upload`` moves
        them to a device later, e.g. after building in a worker process); ``stencil``: the
        layout of the least-squares stencil (``lsq_sell``); ``first_cells``: boolean mask of
        cells numbered first (``nfirst`` of them; ``mb_advdiff_step_split``)."""
        if stencil not in STENCILS:
            raise ValueError("stencil must be one of %s" % (STENCILS,))
        self.stencil = stencil
        from .reorder import Renumbering
        dev = torch.device(device) if device is not None else None
        self.device = dev
        self.A = A
        dim = int(A["dim"])
        nc, nf, nn = int(A["nbcells"]), int(A["nbfaces"]), int(A["nbnodes"])
        nlf = 3 if dim == 2 else 4
        if len(A.get("unmatched_boundary_faces", ())):
            raise ValueError("mesh has boundary faces that match no boundary side (manapy names them "
                             "100/200 and leaves them out of every face list)")
        self.dim, self.nbcells, self.nbfaces, self.nbnodes, self.nlf = dim, nc, nf, nn, nlf
        R = Renumbering(A, enabled=reorder, first=first_cells)
        self.R = R
        self.nfirst = int(np.count_nonzero(first_cells)) if first_cells is not None else 0
        cp, fp, np_ = R.cperm, R.fperm, R.nperm
        ci, fi, ni = R.cinv, R.finv, R.ninv
        f64, i32 = np.float64, np.int32
        T = {}
        T["cell_center"] = _t(A["cells_center"][cp], f64, dev)
        T["cell_volume"] = _t(A["cells_volume"][cp], f64, dev)
        faces_old = A["cells_faceid"][cp, :nlf]
        faces = np.full((nc, 4), -1, dtype=i32)
        faces[:, :nlf] = fi[faces_old]
        T["cell_faces"] = _t(faces, i32, dev)
        # accumulation order: ascending manapy face id
        T["cell_order"] = _t(cell_order_codes(faces_old), np.uint8, dev)
        if "cellnid_ptr" in A:
            ptr, idx, _ = R.relabel_csr(A["cellnid_ptr"], A["cellnid_idx"], cp, ci)
            T["cellnid_ptr"] = _t(ptr, i32, dev)
            T["cellnid_idx"] = _t(idx, i32, dev)
            gp, gi = lsq_sell(ptr, idx, stencil)
            T["lsq_sell_ptr"], T["lsq_sell_idx"] = _t(gp, i32, dev), _t(gi, i32, dev)
        ptr, idx, _ = R.relabel_csr(A["ghostnid_ptr"], A["ghostnid_idx"], cp, fi)
        T["ghostnid_ptr"] = _t(ptr, i32, dev)
        T["ghostnid_idx"] = _t(idx, i32, dev)
        cid = A["faces_cellid"][fp]
        cid_new = np.where(cid >= 0, ci[np.maximum(cid, 0)], -1)
        T["face_cellid"] = _t(cid_new, i32, dev)
        fn = np.full((nf, 4), -1, dtype=i32)
        k = A["faces_nodeid"].shape[1] - 1
        fn[:, :k] = ni[A["faces_nodeid"][fp, :k]]
        T["face_nodeid"] = _t(fn, i32, dev)
        T["face_name"] = _t(A["faces_name"][fp], i32, dev)
        T["face_normal"] = _t(A["faces_normal"][fp], f64, dev)
        T["face_center"] = _t(A["faces_center"][fp], f64, dev)
        T["face_mesure"] = _t(A["faces_mesure"][fp], f64, dev)
        if dim == 2:
            nm = np.zeros((nf, 4))
            nm[:, :2] = A["faces_normal"][fp, :2]
            nm[:, 2] = 1.0 / A["faces_mesure"][fp]
            T["face_nm_f32"] = _t(nm, np.float32, dev)
        T["face_ghostcenter"] = _t(A["faces_ghostcenter"][fp, :3], f64, dev)
        T["face_air"] = _t(A["faces_airDiamond"][fp], f64, dev)
        if dim == 2:
            ff = np.concatenate([A["faces_f_1"], A["faces_f_2"], A["faces_f_3"], A["faces_f_4"]], axis=1)
        else:
            ff = np.concatenate([A["faces_f_1"], A["faces_f_2"]], axis=1)
        T["face_f"] = _t(ff[fp], f64, dev)
        T["face_dist"] = _t(A["faces_dist_ortho"][fp], f64, dev)
        a_c, a_g = vertex_weights(A)
        ptr, idx, src = R.relabel_csr(A["n2c_ptr"], A["n2c_idx"], np_, ci)
        T["n2c_ptr"], T["n2c_idx"], T["n2c_alpha"] = _t(ptr, i32, dev), _t(idx, i32, dev), _t(a_c[src], f64, dev)
        if dim == 3:
            self._node_sum_tables(ptr, idx, a_c[src], T, dev)
        gp, gi, gv = sell32(ptr, idx, a_c[src], fill="first")
        T["n2c_sell_ptr"], T["n2c_sell_idx"], T["n2c_sell_alpha"] = _t(gp, i32, dev), _t(gi, i32, dev), _t(gv, f64, dev)
        T["n2c_sell_alpha_f32"] = _t(gv, np.float32, dev)
        ptr, idx, src = R.relabel_csr(A["n2g_ptr"], A["n2g_idx"], np_, fi)
        T["n2g_ptr"], T["n2g_idx"], T["n2g_alpha"] = _t(ptr, i32, dev), _t(idx, i32, dev), _t(a_g[src], f64, dev)
        if dim == 2:
            # compacted face-neighbour table; its -1 padding is read by manapy as the
            # last cell (negative-index wrap), which is cell ci[nc-1] in this numbering
            cf_old = A["cells_cellfid"][cp, :3]
            cf = np.full((nc, 4), -1, dtype=i32)
            cf[:, :3] = np.where(cf_old >= 0, ci[np.maximum(cf_old, 0)], ci[nc - 1])
            T["cell_cellfid"] = _t(cf, i32, dev)
            T["cell_nf"] = _t(A["cells_nf"][cp], f64, dev)
            T["cell_vertex1"] = _t(A["nodes_vertex"][A["cells_nodeid"][cp, 1], :2], f64, dev)
        if dim == 2:
            self._compact_2d(A, T, dev)
        else:
            self._compact_3d(A, T, dev)
        self.t = T
        # field permutations: device[k] = host[perm[k]], host[j] = device[inv[j]]
        i64 = np.int64
        self.perm = {"cell": _t(cp, i64, dev), "face": _t(fp, i64, dev), "node": _t(np_, i64, dev)}
        self.inv = {"cell": _t(ci, i64, dev), "face": _t(fi, i64, dev), "node": _t(ni, i64, dev)}
        self.reordered = bool(reorder)
        self.struct = self._make_struct() if dev is not None else None

    @classmethod
    def from_host_tables(cls, A, T, R, device=None):
        """A mesh from tables built earlier on the host (``meshcache``): ``A`` the host
        geometry, ``T`` the table dict of ``DeviceMesh(A, device=None)``, ``R`` its
        renumbering (``cperm``, ``cinv``, ``fperm``, ``finv``, ``nperm``, ``ninv``, ``enabled``)."""
        self = cls.__new__(cls)
        dim = int(A["dim"])
        self.dim, self.nbcells, self.nbfaces, self.nbnodes = dim, int(A["nbcells"]), int(A["nbfaces"]), int(A["nbnodes"])
        self.nlf = 3 if dim == 2 else 4
        self.A = A
        self.R = R
        self.reordered = bool(R.enabled)
        self.stencil = str(T.pop("stencil", np.array("manapy")))
        self.nbedges = len(T["edge_origin"]) if "edge_origin" in T else 0
        dev = torch.device(device) if device is not None else None
        self.device = dev
        self.t = {k: _t(v, v.dtype, dev) for k, v in T.items()}
        i64 = np.int64
        self.perm = {"cell": _t(R.cperm, i64, dev), "face": _t(R.fperm, i64, dev), "node": _t(R.nperm, i64, dev)}
        self.inv = {"cell": _t(R.cinv, i64, dev), "face": _t(R.finv, i64, dev), "node": _t(R.ninv, i64, dev)}
        self.struct = self._make_struct() if dev is not None else None
        return self

    @classmethod
    def from_native(cls, elements, vertex, device=None, reorder=True, full=False, stencil="shared"):
        """The tables of a 2D triangle mesh from the native host builder (``native.tables2d``),
        bit-identical to ``DeviceMesh(geometry.build(...))``; ``A`` then holds only the
        manapy-numbered arrays the boundary set-up reads, or with ``full`` every array of
        ``geometry.build`` (bit-identical too)."""
        from types import SimpleNamespace
        from . import native
        if stencil not in STENCILS:
            raise ValueError("stencil must be one of %s" % (STENCILS,))
        T = native.tables2d(elements, vertex, reorder=reorder, full=full, stencil=stencil)
        self = cls.__new__(cls)
        self.stencil = stencil
        nc, nf, nn = len(T["cell_volume"]), len(T["face_name"]), len(T["node_coord"])
        self.dim, self.nbcells, self.nbfaces, self.nbnodes, self.nlf = 2, nc, nf, nn, 3
        self.A = {"dim": 2, "nbcells": nc, "nbfaces": nf, "nbnodes": nn}
        for k in [k for k in T if k.startswith("A.")]:
            self.A[k[2:]] = T.pop(k)
        perm = {kind: T.pop("perm_" + kind) for kind in ("cell", "face", "node")}
        inv = {kind: T.pop("inv_" + kind) for kind in ("cell", "face", "node")}
        self.R = SimpleNamespace(cperm=perm["cell"], fperm=perm["face"], nperm=perm["node"], cinv=inv["cell"],
                                 finv=inv["face"], ninv=inv["node"], enabled=bool(reorder))
        self.reordered = bool(reorder)
        dev = torch.device(device) if device is not None else None
        self.device = dev
        self.t = {k: _t(v, v.dtype, dev) for k, v in T.items()}
        self.perm = {k: _t(v, np.int64, dev) for k, v in perm.items()}
        self.inv = {k: _t(v, np.int64, dev) for k, v in inv.items()}
        self.struct = self._make_struct() if dev is not None else None
        return self

    def _make_struct(self):
        s = _lib.MbMesh()
        s.dim, s.nbcells, s.nbfaces, s.nbnodes, s.nlf = (self.dim, self.nbcells, self.nbfaces, self.nbnodes,
                                                         self.nlf)
        s.variant = int(getattr(self, "variant", 0))
        for name, _ in _lib.MbMesh._fields_:
            if name in self.t and name not in self.EDGE_TABLES:
                setattr(s, name, self.t[name].data_ptr())
        return s

    # the edge tables change the scratch a second-order 3D step needs, so a struct carries
    # them only once its user asks (use_edge_sums)
    EDGE_TABLES = ("cell_edges", "edge_origin", "edge_sell_ptr", "edge_sell_idx", "n2c_sum_ptr", "n2c_sum_idx",
                   "n2c_sum_alpha")

    def use_edge_sums(self):
        """Tetrahedra: point the struct at the edge tables, so that the second-order step
        forms the least-squares sums by inclusion-exclusion (it then needs ``cell_lsq`` and
        ``cell_scratch_size()`` doubles of cell scratch).  Returns False where the tables are
        absent."""
        if self.dim != 3 or "cell_edges" not in self.t or self.device is None:
            return False
        for name in self.EDGE_TABLES:
            setattr(self.struct, name, self.t[name].data_ptr())
        self.struct.nbedges = int(self.nbedges)
        return True

    def cell_scratch_size(self):
        """Doubles of cell scratch a fused step needs with this struct: 4 nbcells (2D), 8 nbcells
        (3D), plus 4 (nbnodes + nbedges) when the edge sums are in use."""
        if self.dim == 2:
            return 4 * self.nbcells
        extra = 4 * (self.nbnodes + int(self.nbedges)) if self.struct is not None and self.struct.cell_edges else 0
        return 8 * self.nbcells + extra

    def cell_scratch_size_f32c(self):
        """Floats of cell scratch an FP32-compensated second-order step needs with this struct:
        4 nbcells (2D), 5 nbcells (3D); with the edge sums in use, 5 nbcells rounded up to 8,
        plus the FP64 vertex and edge sums, 8 (nbnodes + nbedges) floats."""
        if self.dim == 2:
            return 4 * self.nbcells
        if self.struct is not None and self.struct.cell_edges:
            return ((5 * self.nbcells + 7) // 8) * 8 + 8 * (self.nbnodes + int(self.nbedges))
        return 5 * self.nbcells

    def check_tables(self, stream=None):
        """Debug check of every index table on the device (``mb_check_tables``): raises
        ValueError naming the first entry outside the range the kernels gather with."""
        first = torch.empty(1, dtype=torch.int64, device=self.device)
        st = stream if stream is not None else torch.cuda.current_stream(self.device).cuda_stream
        _lib.call("mb_check_tables", self.struct, first.data_ptr(), st)
        torch.cuda.synchronize(self.device)
        bad = _lib.decode_table_check(int(first.item()) & (2 ** 64 - 1))
        if bad is None:
            return
        name, offs, pos = bad
        value = int(self.t[name].reshape(-1)[pos].item())
        tid = [t[1] if offs else t[0] for t in _lib.CHECK_TABLES].index(name)
        lo, hi = _lib.CHECK_TABLES[tid][3](self.nbcells, self.nbfaces, self.nbnodes)
        if hi is None:                       # cell_edges: the edge count
            hi = int(getattr(self, "nbedges", 0))
        what = "is out of order" if offs else "is outside [%d, %d)" % (lo, hi)
        raise ValueError("mesh table %s: entry %d = %d %s" % (name, pos, value, what))

    def ensure_lsq_matrix(self, stream=None):
        """Tetrahedra with compact tables: the ``cell_lsq`` table (the least-squares moment
        matrix of every cell, ``mb_lsq_matrix``), formed once on the device and pointed at by
        the struct, so that the second-order fused step reads it instead of forming it every
        step.  No-op for triangles, host-built tables, or when it is there already."""
        if self.dim != 3 or self.device is None or "cell_lsq" in self.t or "lsq_sell_idx" not in self.t:
            return
        out = torch.empty(12 * self.nbcells, dtype=torch.float64, device=self.device)
        st = stream if stream is not None else torch.cuda.current_stream(self.device).cuda_stream
        _lib.call("mb_lsq_matrix", self.struct, out.data_ptr(), st)
        self.t["cell_lsq"] = out
        self.struct.cell_lsq = out.data_ptr()

    def upload(self, device, stream=None):
        """Move host-built tables (``device=None`` at construction) to ``device``; with a
        CUDA ``stream`` the copies are asynchronous on it.  Drops the host arrays ``A``."""
        dev = torch.device(device)
        self.t = {k: _upload(a, dev, stream) for k, a in self.t.items()}
        self.perm = {k: _upload(a, dev, stream) for k, a in self.perm.items()}
        self.inv = {k: _upload(a, dev, stream) for k, a in self.inv.items()}
        self.device = dev
        self.A = None
        self.struct = self._make_struct()
        return self

    # tables the FP32-compensated steps and their set-up kernels read (batched serving)
    SERVE_TABLES = ("cell_volume", "cell_order", "cell_faces", "cell_vtx", "cell_nbr", "cell_flags", "node_coord",
                    "cell_xy", "lsq_sell_ptr", "lsq_sell_idx", "n2c_sell_ptr", "n2c_sell_idx", "n2c_sell_alpha_f32",
                    "ghostnid_ptr", "ghostnid_idx", "face_ghostcenter", "n2g_ptr", "n2g_idx", "n2g_alpha",
                    "face_cellid", "face_dist", "face_normal", "face_mesure", "face_nm_f32", "cell_cellfid")

    def keep_only(self, names):
        """Drop every table not in ``names`` (host-built tables, before an upload)."""
        self.t = {k: v for k, v in self.t.items() if k in names}
        return self

    def upload_staged(self, device, stream, staging, extra=None):
        """Upload host-built tables with one copy (``stage_upload``); the permutations stay on
        the host.  ``extra``: more host arrays to send in the same copy; returns their device
        views."""
        arrays = dict(self.t)
        for k, a in (extra or {}).items():
            arrays["extra." + k] = a
        views, buf = stage_upload(arrays, device, stream, staging)
        self.t = {k: v for k, v in views.items() if not k.startswith("extra.")}
        self._buf = buf
        self.device = torch.device(device)
        self.A = None
        self.struct = self._make_struct()
        return {k[6:]: v for k, v in views.items() if k.startswith("extra.")}

    def strip(self):
        """Drop the host arrays ``A`` (before sending host-built tables to another process)."""
        self.A = None
        return self

    def _compact_2d(self, A, T, dev):
        """Cell-centred tables of the fused 2D step (see ``mb_mesh`` in the C header)."""
        R = self.R
        cp, ci, fi, ni, np_ = R.cperm, R.cinv, R.finv, R.ninv, R.nperm
        nc = self.nbcells
        nodes = A["cells_nodeid"][cp, :3].astype(np.int64)          # manapy's local vertex order
        faces = A["cells_faceid"][cp, :3].astype(np.int64)          # local face j = (v_j, v_j+1)
        fcid = A["faces_cellid"]
        c0 = fcid[faces, 0]
        c1 = fcid[faces, 1]
        own = c0 == cp[:, None]
        other = np.where(own, c1, c0)
        bnd = c1 < 0
        nbr = np.where(bnd, -1 - fi[faces], ci[np.maximum(other, 0)])
        fa = A["faces_nodeid"][faces, 0]                            # faces.nodeid[f][0]
        v_next = np.roll(nodes, -1, axis=1)
        rev = fa == v_next
        assert np.all(rev | (fa == nodes)), "face nodes do not match the cell's local faces"
        X = A["nodes_vertex"]
        a = np.where(rev, v_next, nodes)
        b = np.where(rev, nodes, v_next)
        n0 = X[a, 1] - X[b, 1]
        n1 = X[b, 0] - X[a, 0]
        stored = A["faces_normal"][faces]
        flip = (stored[..., 0] != n0) | (stored[..., 1] != n1)
        assert np.array_equal(np.where(flip, -1 * n0, n0), stored[..., 0]) and \
            np.array_equal(np.where(flip, -1 * n1, n1), stored[..., 1]), "normals are not vertex differences"
        # cells.nf: the outward normal table of the bathymetry source (+- the face normal)
        nf_tab = A["cells_nf"][cp]
        nfneg = (nf_tab[..., 0] != stored[..., 0]) | (nf_tab[..., 1] != stored[..., 1])
        assert np.array_equal(np.where(nfneg, -1 * stored[..., 0], stored[..., 0]), nf_tab[..., 0]), \
            "cells.nf is not +- the face normal"
        flags = np.zeros(nc, dtype=np.uint32)
        for j in range(3):
            flags |= (own[:, j].astype(np.uint32) << j) | (rev[:, j].astype(np.uint32) << (3 + j)) \
                | (flip[:, j].astype(np.uint32) << (6 + j)) | (nfneg[:, j].astype(np.uint32) << (9 + j))
        vtx = np.zeros((nc, 4), dtype=np.int32)
        vtx[:, :3] = ni[nodes]
        nb4 = np.full((nc, 4), -1, dtype=np.int32)
        nb4[:, :3] = nbr
        T["cell_vtx"] = _t(vtx, np.int32, dev)
        T["cell_nbr"] = _t(nb4, np.int32, dev)
        T["cell_flags"] = _t(flags.view(np.int32), np.int32, dev)
        T["node_coord"] = _t(X[np_, :2], np.float64, dev)
        T["cell_xy"] = _t(A["cells_center"][cp, :2], np.float64, dev)

    # local faces of a tetrahedron (manapy/ddm/ddm_utils3d.py:785-791) and the six
    # permutations of three items, in the order the kernels decode them
    TET_FACES = np.array([[0, 1, 2], [2, 3, 0], [0, 1, 3], [3, 1, 2]])
    PERM3 = np.array([[0, 1, 2], [0, 2, 1], [1, 0, 2], [1, 2, 0], [2, 0, 1], [2, 1, 0]])

    def _compact_3d(self, A, T, dev):
        """Cell-centred tables of the fused 3D step (see ``mb_mesh`` in the C header)."""
        R = self.R
        cp, ci, fi, ni, np_ = R.cperm, R.cinv, R.finv, R.ninv, R.nperm
        nc = self.nbcells
        nodes = A["cells_nodeid"][cp, :4].astype(np.int64)
        faces = A["cells_faceid"][cp, :4].astype(np.int64)
        fcid = A["faces_cellid"]
        c0 = fcid[faces, 0]
        c1 = fcid[faces, 1]
        own = c0 == cp[:, None]
        other = np.where(own, c1, c0)
        bnd = c1 < 0
        nbr = np.where(bnd, -1 - fi[faces], ci[np.maximum(other, 0)])
        X = A["nodes_vertex"][:, :3]
        stored = A["faces_normal"][faces]                          # [nc, 4, 3]
        fnodes = A["faces_nodeid"][faces][..., :3]                 # oriented order
        flags = np.zeros(nc, dtype=np.uint32)
        for j in range(4):
            loc = nodes[:, self.TET_FACES[j]]                       # [nc, 3] original node ids
            order = np.argsort(-loc, axis=1, kind="stable")         # descending original id
            code = self._perm_codes(order)
            desc = np.take_along_axis(loc, order, axis=1)
            ori = fnodes[:, j]
            swap = (ori[:, 1] == desc[:, 2]) & (ori[:, 2] == desc[:, 1])
            assert np.all(ori[:, 0] == desc[:, 0]) and np.all(swap | ((ori[:, 1] == desc[:, 1]) & (ori[:, 2] == desc[:, 2]))), \
                "face nodes are not the descending order of the cell's local face"
            V0, V1, V2 = X[desc[:, 0]], X[desc[:, 1]], X[desc[:, 2]]
            u = V1 - V0
            v = V2 - V0
            Nd = 0.5 * np.stack([u[:, 1] * v[:, 2] - u[:, 2] * v[:, 1], u[:, 2] * v[:, 0] - u[:, 0] * v[:, 2],
                                 u[:, 0] * v[:, 1] - u[:, 1] * v[:, 0]], axis=1)
            st = stored[:, j]
            flip = np.any(st != Nd, axis=1)
            assert np.array_equal(np.where(flip[:, None], -1 * Nd, Nd), st), "normals are not vertex cross products"
            flags |= (own[:, j].astype(np.uint32) << (6 * j)) | (code << (6 * j + 1)) \
                | (swap.astype(np.uint32) << (6 * j + 4)) | (flip.astype(np.uint32) << (6 * j + 5))
        T["cell_vtx"] = _t(ni[nodes], np.int32, dev)
        T["cell_nbr"] = _t(nbr, np.int32, dev)
        T["cell_flags"] = _t(flags.view(np.int32), np.int32, dev)
        nc4 = np.zeros((len(np_), 4))
        nc4[:, :3] = X[np_]
        T["node_coord"] = _t(nc4, np.float64, dev)
        cc4 = np.zeros((nc, 4))
        cc4[:, :3] = A["cells_center"][cp]
        T["cell_xy"] = _t(cc4, np.float64, dev)
        self._edge_tables(ni[nodes], T, dev)

    def _node_sum_tables(self, ptr, idx, alpha, T, dev):
        """Tetrahedra: the vertex -> cells lists in the slot-shared SELL-32 layout with their
        centre->vertex weights (``n2c_sum_ptr`` / ``n2c_sum_idx`` / ``n2c_sum_alpha``; -1 and
        weight 0 in empty slots), read by the vertex sums of the edge-sum step."""
        from . import native
        ptr = np.asarray(ptr, dtype=np.int64)
        idx = np.asarray(idx, dtype=np.int64)
        nrow, ncell = len(ptr) - 1, int(self.nbcells)
        gp, gi = native.sell_aligned(ptr, idx.astype(np.int32))
        gp64 = np.asarray(gp, dtype=np.int64)
        # the CSR position of every (row, cell) slot
        slot = np.arange(int(gp64[-1]), dtype=np.int64)
        grp = np.searchsorted(gp64, slot, side="right") - 1
        row = 32 * grp + (slot - gp64[grp]) % 32
        key_csr = np.repeat(np.arange(nrow, dtype=np.int64), np.diff(ptr)) * ncell + idx
        order = np.argsort(key_csr, kind="stable")
        gi64 = np.asarray(gi, dtype=np.int64)
        used = gi64 >= 0
        pos = order[np.searchsorted(key_csr[order], row[used] * ncell + gi64[used])]
        al = np.zeros(len(gi64))
        al[used] = np.asarray(alpha)[pos]
        T["n2c_sum_ptr"] = _t(gp, np.int32, dev)
        T["n2c_sum_idx"] = _t(gi, np.int32, dev)
        T["n2c_sum_alpha"] = _t(al, np.float64, dev)

    # the six edges of a tetrahedron as pairs of local vertices
    TET_EDGES = np.array([[0, 1], [0, 2], [0, 3], [1, 2], [1, 3], [2, 3]])

    def _edge_tables(self, vt, T, dev):
        """Edges of a tetrahedral mesh for the least-squares sums by inclusion-exclusion:
        ``cell_edges`` [nc][8] (the edge of each local vertex pair in TET_EDGES order, then
        -1, -1), ``edge_origin`` [ne] (the edge's vertex of smaller device number, the origin
        of its sums), ``edge_sell_ptr`` / ``edge_sell_idx`` (edge -> cells, SELL-32,
        slot-shared, -1 in empty slots).  Edges are numbered by their first cell."""
        nc, nn = len(vt), self.nbnodes
        ends = np.sort(vt[:, self.TET_EDGES], axis=2).reshape(-1, 2).astype(np.int64)   # [nc*6, 2]
        key = ends[:, 0] * nn + ends[:, 1]
        uk, first, inv = np.unique(key, return_index=True, return_inverse=True)
        # number edges by their first cell (the device cell numbering keeps locality)
        order = np.argsort(first // 6, kind="stable")
        rank = np.empty(len(uk), dtype=np.int64)
        rank[order] = np.arange(len(uk))
        eid = rank[inv].reshape(nc, 6)
        ce = np.full((nc, 8), -1, dtype=np.int32)
        ce[:, :6] = eid
        T["cell_edges"] = _t(ce, np.int32, dev)
        T["edge_origin"] = _t((uk[order] // nn).astype(np.int32), np.int32, dev)
        cells = np.repeat(np.arange(nc, dtype=np.int64), 6)
        flat = eid.reshape(-1)
        srt = np.argsort(flat, kind="stable")
        ptr = np.zeros(len(uk) + 1, dtype=np.int64)
        np.cumsum(np.bincount(flat, minlength=len(uk)), out=ptr[1:])
        gp, gi = lsq_sell(ptr, cells[srt].astype(np.int32), "shared")
        T["edge_sell_ptr"] = _t(gp, np.int32, dev)
        T["edge_sell_idx"] = _t(gi, np.int32, dev)
        self.nbedges = len(uk)

    @classmethod
    def _perm_codes(cls, order):
        """Index in PERM3 of each row of ``order`` (a permutation of 0, 1, 2)."""
        key = order[:, 0] * 9 + order[:, 1] * 3 + order[:, 2]
        table = np.zeros(27, dtype=np.uint32)
        for k, p in enumerate(cls.PERM3):
            table[p[0] * 9 + p[1] * 3 + p[2]] = k
        return table[key]

    def to_device_order(self, kind, host_t, out):
        """out[k] = host_t[perm[k]] (``host_t`` already on the device, manapy order)."""
        if not self.reordered or kind is None:
            out.copy_(host_t)
        else:
            torch.index_select(host_t, 0, self.perm[kind], out=out)

    def to_host_order(self, kind, dev_t):
        if not self.reordered or kind is None:
            return dev_t
        return torch.index_select(dev_t, 0, self.inv[kind])

    def has_lsq(self):
        return "cellnid_ptr" in self.t

    def nbytes(self):
        return sum(int(t.nbytes) if isinstance(t, np.ndarray) else t.numel() * t.element_size()
                   for t in self.t.values())


class DeviceBC:
    """One variable's ghost rules on the device (``mb_bc``)."""

    def __init__(self, A, resolved, device="cuda", mesh=None):
        from .boundary import G_CELL_AT_FACE
        dev = torch.device(device) if device is not None else None
        nf = int(A["nbfaces"])
        self.resolved = resolved
        fp = mesh.R.fperm if mesh is not None else np.arange(nf)
        ci = mesh.R.cinv if mesh is not None else np.arange(int(A["nbcells"]))
        kind = resolved.kind
        value = resolved.value.copy()
        # MB_G_CELL_AT_FACE reads the cell array at the face's manapy index; the cell
        # to read (in the device numbering) travels in value[f]
        caf = np.nonzero(kind == G_CELL_AT_FACE)[0]
        value[caf] = ci[caf]
        self.kind = _t(kind[fp], np.int8, dev)
        self.value = _t(value[fp], np.float64, dev)
        on = np.zeros(nf, dtype=np.uint8)
        on[A["innerfaces"]] = 1
        on[resolved.dirichletfaces] = 1
        on[resolved.neumannfaces] = 1
        self.face_grad_on = _t(on[fp], np.uint8, dev)
        self.struct = self._make_struct() if dev is not None else None

    def _make_struct(self):
        s = _lib.MbBC()
        s.kind = self.kind.data_ptr()
        s.value = self.value.data_ptr()
        s.face_grad_on = self.face_grad_on.data_ptr()
        return s

    def upload(self, device, stream=None):
        dev = torch.device(device)
        self.kind, self.value, self.face_grad_on = (_upload(a, dev, stream)
                                                    for a in (self.kind, self.value, self.face_grad_on))
        self.struct = self._make_struct()
        return self
