"""Host-side mesh connectivity and FP64 geometry, array-for-array as manapy builds it.

``build(elements, vertex, dim)`` returns every ``Domain`` array the explicit
finite-volume step reads, with manapy's numbering, orientation and padding
conventions, computed with vectorised numpy instead of manapy's per-cell loops
(``manapy/ddm/domain.py:130-160``).  Ragged integer tables use manapy's padded
layout: ``[n, width+1]`` with ``-1`` padding and the row count in the last
column.  Single-rank meshes only: halo, halo-ghost and periodic tables are the
empty placeholders manapy creates when ``size == 1``.

What each step reproduces (reference file:line):

* cell centre / volume: ``manapy/ddm/ddm_utils2d.py:433-452``,
  ``manapy/ddm/ddm_utils3d.py:686-725``
* node->cell and cell->vertex-neighbour tables: ``ddm_utils2d.py:55-97``
* faces: local faces per cell (``ddm_utils2d.py:482-497``,
  ``ddm_utils3d.py:766-791``), node tuples sorted descending, numbered by
  ``np.unique(axis=0)`` (``domain.py:313-315``)
* cell->face, face->cell, face-neighbour tables: ``ddm_utils2d.py:12-53``
* face names / normals / areas / centres: ``ddm_utils2d.py:507-551``,
  ``ddm_utils3d.py:530-684``; 3D node order of faces re-oriented with the
  normal: ``ddm_utils3d.py:362-377``
* outward normals per cell (2D): ``ddm_utils2d.py:99-120``
* boundary face lists: ``domain.py:395-460``
* ghost centres and node->ghost tables: ``ddm_utils2d.py:163-197``,
  ``ddm_utils3d.py:87-130``, ``ddm_utils2d.py:122-161``
* centre->vertex weights (R, lambda, number): ``ddm_utils2d.py:608-705``,
  ``ddm_utils3d.py:813-981``
* diamond-cell geometry: ``ddm_utils2d.py:553-605``, ``ddm_utils3d.py:459-527``
* orthogonal distances (2D): ``ddm_utils2d.py:716-744``
"""
from __future__ import annotations

import numpy as np

__all__ = ["build", "csr_from_padded", "padded_from_csr", "ragged_union"]

I32 = np.int32


def padded_from_csr(ptr, idx, min_width=1, fill=-1):
    """manapy padded table ``[n, w+1]`` (count in the last column) from CSR."""
    n = len(ptr) - 1
    cnt = np.diff(ptr)
    w = max(int(cnt.max()) if n else 0, min_width)
    out = np.full((n, w + 1), fill, dtype=I32)
    rows = np.repeat(np.arange(n), cnt)
    cols = np.arange(len(idx)) - np.repeat(ptr[:-1], cnt)
    out[rows, cols] = idx
    out[:, -1] = cnt
    return out


def csr_from_padded(tab):
    """CSR ``(ptr, idx)`` from a manapy padded table."""
    tab = np.asarray(tab)
    cnt = tab[:, -1].astype(np.int64)
    ptr = np.zeros(len(tab) + 1, dtype=np.int64)
    np.cumsum(cnt, out=ptr[1:])
    mask = np.arange(tab.shape[1] - 1)[None, :] < cnt[:, None]
    return ptr, tab[:, :-1][mask].astype(I32)


def _group_ptr(keys_sorted, n):
    """CSR row pointer for a key array already sorted ascending in [0, n)."""
    cnt = np.bincount(keys_sorted, minlength=n)
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(cnt, out=ptr[1:])
    return ptr


def ragged_union(row_items_ptr, row_items, item_ptr, item_vals, exclude_self=False):
    """For each row r: sorted unique union of ``item_vals[item_ptr[i]:item_ptr[i+1]]``
    over items ``i`` listed for ``r`` in ``row_items[row_items_ptr[r]:...]``.

    Returns CSR ``(ptr, idx)``.  ``exclude_self`` drops value ``r`` from row ``r``.
    """
    nrows = len(row_items_ptr) - 1
    rcnt = np.diff(row_items_ptr)
    row_of_item = np.repeat(np.arange(nrows, dtype=np.int64), rcnt)
    icnt = np.diff(item_ptr)[row_items]
    total = int(icnt.sum())
    # candidates of each row in a padded [nrows, width] matrix, sorted per row
    per_row = np.bincount(row_of_item, weights=icnt, minlength=nrows).astype(np.int64)
    width = max(int(per_row.max()) if nrows else 0, 1)
    row_of_val = np.repeat(row_of_item, icnt)
    starts = np.repeat(item_ptr[row_items], icnt)
    offs = np.arange(total, dtype=np.int64) - np.repeat(np.cumsum(icnt) - icnt, icnt)
    vals = item_vals[starts + offs]
    rstart = np.zeros(nrows + 1, dtype=np.int64)
    np.cumsum(per_row, out=rstart[1:])
    col = np.arange(total, dtype=np.int64) - rstart[row_of_val]
    big = np.iinfo(np.int32).max
    mat = np.full((nrows, width), big, dtype=np.int32)
    mat[row_of_val, col] = vals
    mat.sort(axis=1)
    keep = mat != big
    keep[:, 1:] &= mat[:, 1:] != mat[:, :-1]
    if exclude_self:
        keep &= mat != np.arange(nrows, dtype=np.int32)[:, None]
    cnt = keep.sum(axis=1)
    ptr = np.zeros(nrows + 1, dtype=np.int64)
    np.cumsum(cnt, out=ptr[1:])
    return ptr, mat[keep].astype(I32)


class Arrays(dict):
    """``dict`` with attribute access."""

    __getattr__ = dict.__getitem__


def _face_names_2d(namen, nodeid, boundary):
    a = namen[nodeid[:, 0]]
    b = namen[nodeid[:, 1]]
    name = np.zeros(len(nodeid), dtype=I32)
    res = np.full(len(nodeid), 100, dtype=I32)
    # precedence of the elif chain at ddm_utils2d.py:519-537, applied in reverse
    for tag in (44, 33, 4, 3):
        m = ((a == tag) & (b != 0)) | ((a != 0) & (b == tag))
        res = np.where(m, tag, res)
    res = np.where(a == b, a, res)
    name[boundary] = res[boundary]
    return name


def _face_names_3d(namen, nodeid, boundary):
    k = 3
    nn = namen[nodeid[:, :k]]
    res = np.full(len(nodeid), 100, dtype=I32)
    nz = nn != 0
    for tag in (44, 33, 66, 55, 4, 3, 6, 5):
        m = np.zeros(len(nodeid), dtype=bool)
        for j in range(k):
            mj = nn[:, j] == tag
            for jj in range(k):
                if jj != j:
                    mj &= nz[:, jj]
            m |= mj
        res = np.where(m, tag, res)
    same = (nn[:, 0] == nn[:, 1]) & (nn[:, 0] == nn[:, 2])
    res = np.where(same, nn[:, 0], res)
    name = np.zeros(len(nodeid), dtype=I32)
    name[boundary] = res[boundary]
    return name


def _cross(a, b):
    return np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1],
                     a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                     a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], axis=1)


def _dot3(a, b):
    return a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1] + a[:, 2] * b[:, 2]


def build(elements, vertex, dim, need_cellnid=True, halo_rim=False):
    """All ``Domain`` arrays of the explicit step for a single-rank mesh.

    ``halo_rim=True`` (the submesh of one shard, ``partition.py``): boundary faces that
    belong to no side are the cut between the shard's halo and the rest of the mesh; they
    are named 10, manapy's halo-face name, and listed in ``halofaces`` instead of being
    rejected."""
    elements = np.ascontiguousarray(elements, dtype=I32)
    vertex = np.ascontiguousarray(vertex, dtype=np.float64)
    dim = int(dim)
    nc = len(elements)
    nn = len(vertex)
    k = int(elements[0, -1])
    if dim == 2 and not np.all(elements[:, -1] == 3):
        raise ValueError("2D meshes must be all triangles")
    if dim == 3 and not np.all(elements[:, -1] == 4):
        raise ValueError("3D meshes must be all tetrahedra")
    cn = elements[:, :k].astype(np.int64)
    A = Arrays(dim=dim, nbcells=nc, nbnodes=nn)
    A["cells_nodeid"] = elements
    A["nodes_vertex"] = vertex
    X = vertex[:, 0]
    Y = vertex[:, 1]
    Zc = vertex[:, 2]

    # ---- cell centre and volume
    center = np.zeros((nc, 3))
    if dim == 2:
        x1, x2, x3 = X[cn[:, 0]], X[cn[:, 1]], X[cn[:, 2]]
        y1, y2, y3 = Y[cn[:, 0]], Y[cn[:, 1]], Y[cn[:, 2]]
        center[:, 0] = 1.0 / 3 * (x1 + x2 + x3)
        center[:, 1] = 1.0 / 3 * (y1 + y2 + y3)
        volume = 0.5 * np.abs((x1 - x2) * (y1 - y3) - (x1 - x3) * (y1 - y2))
    else:
        P = [vertex[cn[:, j], :3] for j in range(4)]
        c = np.zeros((nc, 3))
        for j in range(4):
            c = c + P[j]
        center = c / 4
        u = P[1] - P[0]
        v = P[2] - P[0]
        w = P[3] - P[0]
        volume = np.abs(_dot3(u, _cross(v, w))) / 6.0
    A["cells_center"] = center
    A["cells_volume"] = volume

    # ---- node -> cell (ascending cell order), cell -> vertex neighbours
    flat_nodes = cn.ravel()
    flat_cells = np.repeat(np.arange(nc, dtype=np.int64), k)
    order = np.argsort(flat_nodes, kind="stable")
    n2c_ptr = _group_ptr(flat_nodes[order], nn)
    n2c_idx = flat_cells[order].astype(I32)
    A["n2c_ptr"], A["n2c_idx"] = n2c_ptr, n2c_idx
    c2n_ptr = np.arange(0, nc * k + 1, k, dtype=np.int64)
    if need_cellnid:
        A["cellnid_ptr"], A["cellnid_idx"] = ragged_union(c2n_ptr, flat_nodes, n2c_ptr, n2c_idx,
                                                          exclude_self=True)

    # ---- faces
    if dim == 2:
        loc = np.array([[0, 1], [1, 2], [2, 0]])
    else:
        loc = np.array([[0, 1, 2], [2, 3, 0], [0, 1, 3], [3, 1, 2]])
    nlf = len(loc)
    pf = cn[:, loc].reshape(-1, loc.shape[1])
    pf = -np.sort(-pf, axis=1)  # descending
    if dim == 2:
        key = pf[:, 0] * nn + pf[:, 1]
    else:
        key = (pf[:, 0] * nn + pf[:, 1]) * nn + pf[:, 2]
    ukey, first, inv = np.unique(key, return_index=True, return_inverse=True)
    nf = len(ukey)
    fnodes = pf[first].astype(I32)
    cell_faceid = inv.reshape(nc, nlf).astype(I32)
    # face -> cells: first (smaller) and second cell, ddm_utils2d.py:12-20
    order = np.argsort(inv, kind="stable")
    fptr = _group_ptr(inv[order], nf)
    fcnt = np.diff(fptr)
    owner = (order // nlf).astype(I32)
    cellid = np.full((nf, 2), -1, dtype=I32)
    cellid[:, 0] = owner[fptr[:-1]]
    two = fcnt == 2
    cellid[two, 1] = owner[fptr[:-1][two] + 1]
    if np.any(fcnt > 2):
        raise ValueError("non-manifold mesh: a face is shared by more than two cells")
    A["nbfaces"] = nf
    A["faces_cellid"] = cellid
    faceid = np.full((nc, nlf + 1), -1, dtype=I32)
    faceid[:, :nlf] = cell_faceid
    faceid[:, -1] = nlf
    A["cells_faceid"] = faceid
    # face neighbours, compacted (boundary faces skipped), ddm_utils2d.py:32-53
    other = np.where(cellid[cell_faceid, 0] == np.arange(nc)[:, None],
                     cellid[cell_faceid, 1], cellid[cell_faceid, 0])
    valid = cellid[cell_faceid, 1] != -1
    cnt = valid.sum(axis=1)
    cellfid = np.full((nc, nlf + 1), -1, dtype=I32)
    srt = np.argsort(~valid, axis=1, kind="stable")
    comp = np.take_along_axis(other, srt, axis=1)
    comp = np.where(np.arange(nlf)[None, :] < cnt[:, None], comp, -1)
    cellfid[:, :nlf] = comp
    cellfid[:, -1] = cnt
    A["cells_cellfid"] = cellfid

    # ---- face names, normals, areas, centres
    namen = vertex[:, 3].astype(I32)
    boundary_mask = cellid[:, 1] == -1
    fn = fnodes.astype(np.int64)
    if dim == 2:
        name = _face_names_2d(namen, fn, boundary_mask)
        norm = np.zeros((nf, 3))
        norm[:, 0] = Y[fn[:, 0]] - Y[fn[:, 1]]
        norm[:, 1] = X[fn[:, 1]] - X[fn[:, 0]]
        fcenter = 0.5 * (vertex[fn[:, 0], :3] + vertex[fn[:, 1], :3])
        snorm = center[cellid[:, 0]] - fcenter
        flip = (snorm[:, 0] * norm[:, 0] + snorm[:, 1] * norm[:, 1]) > 0
        normal = np.where(flip[:, None], -1 * norm, norm)
        mesure = np.sqrt(normal[:, 0] ** 2 + normal[:, 1] ** 2)
    else:
        name = _face_names_3d(namen, fn, boundary_mask)
        V0, V1, V2 = (vertex[fn[:, j], :3] for j in range(3))
        fcenter = 1.0 / 3 * (V0 + V1 + V2)
        norm = 0.5 * _cross(V1 - V0, V2 - V0)
        mesure = np.sqrt(norm[:, 0] ** 2 + norm[:, 1] ** 2 + norm[:, 2] ** 2)
        snorm = center[cellid[:, 0]] - fcenter
        flip = _dot3(snorm, norm) > 0
        normal = np.where(flip[:, None], -1 * norm, norm)
        # node order re-oriented with the normal, ddm_utils3d.py:362-377
        swap = _dot3(_cross(V1 - V0, V2 - V0), normal) < 0
        fnodes = fnodes.copy()
        fnodes[swap, 1], fnodes[swap, 2] = fnodes[swap, 2].copy(), fnodes[swap, 1].copy()
        fn = fnodes.astype(np.int64)
    fnodeid = np.empty((nf, fnodes.shape[1] + 1), dtype=I32)
    fnodeid[:, :-1] = fnodes
    fnodeid[:, -1] = fnodes.shape[1]
    A["faces_nodeid"] = fnodeid
    A["faces_name"] = name
    A["faces_normal"] = normal
    A["faces_mesure"] = mesure
    A["faces_center"] = fcenter
    A["nodes_name"] = namen

    if dim == 2:
        # outward normal of each local face, ddm_utils2d.py:99-120
        G = center[:, None, :]
        cfc = fcenter[cell_faceid]
        nrm = normal[cell_faceid]
        s = ((G[..., 0] - cfc[..., 0]) * nrm[..., 0] + (G[..., 1] - cfc[..., 1]) * nrm[..., 1]
             + (G[..., 2] - cfc[..., 2]) * nrm[..., 2])
        A["cells_nf"] = np.where((s < 0)[..., None], nrm, -1.0 * nrm)

    # ---- boundary face lists, domain.py:401-457
    where = lambda t: np.nonzero(name == t)[0].astype(I32)  # noqa: E731
    A["innerfaces"] = where(0)
    for nm, t in (("infaces", 1), ("outfaces", 2), ("upperfaces", 3), ("bottomfaces", 4)):
        A[nm] = where(t)
    lists = [A["infaces"], A["outfaces"], A["bottomfaces"], A["upperfaces"]]
    if dim == 3:
        A["frontfaces"] = where(5)
        A["backfaces"] = where(6)
        lists += [A["backfaces"], A["frontfaces"]]
    A["boundaryfaces"] = np.sort(np.concatenate(lists)).astype(I32)
    A["halofaces"] = np.zeros(0, dtype=I32)
    A["periodicboundaryfaces"] = np.zeros(0, dtype=I32)
    # boundary faces that belong to no side: names 100/200 (manapy leaves them out of every
    # list), and name 0 (all vertices untagged: manapy would treat them as inner faces
    # reading cell -1)
    unmatched = boundary_mask & ((name >= 100) | (name == 0))
    if halo_rim:
        name[unmatched] = 10
        A["faces_name"] = name
        A["innerfaces"] = where(0)
        A["halofaces"] = np.nonzero(unmatched)[0].astype(I32)
        unmatched = np.zeros_like(unmatched)
    A["unmatched_boundary_faces"] = np.nonzero(unmatched)[0].astype(I32)

    # ---- ghost centres, ddm_utils2d.py:172-187 / ddm_utils3d.py:96-118
    bf = A["boundaryfaces"].astype(np.int64)
    if dim == 2:
        gc = -1 * np.ones((nf, 3))
        x_1 = vertex[fn[bf, 1]]
        x_2 = vertex[fn[bf, 0]]
        v_1 = center[cellid[bf, 0]]
        gamma = (((v_1[:, 0] - x_2[:, 0]) * (x_1[:, 0] - x_2[:, 0])
                  + (v_1[:, 1] - x_2[:, 1]) * (x_1[:, 1] - x_2[:, 1]))
                 / ((x_1[:, 0] - x_2[:, 0]) ** 2 + (x_1[:, 1] - x_2[:, 1]) ** 2))
        kk0 = gamma * x_1[:, 0] + (1 - gamma) * x_2[:, 0]
        kk1 = gamma * x_1[:, 1] + (1 - gamma) * x_2[:, 1]
        gc[bf, 0] = 2 * kk0 + (-1 * v_1[:, 0])
        gc[bf, 1] = 2 * kk1 + (-1 * v_1[:, 1])
        gc[bf, 2] = gamma
    else:
        gc = -1 * np.ones((nf, 4))
        n = normal[bf] / mesure[bf][:, None]
        v_1 = center[cellid[bf, 0]]
        u = fcenter[bf] - v_1
        gamma = _dot3(u, n)
        kk = v_1 + gamma[:, None] * n
        gc[bf, :3] = 2 * kk + (-1 * v_1)
        gc[bf, 3] = gamma
    A["faces_ghostcenter"] = gc

    # node -> boundary faces (ascending face order), cell -> ghost neighbours
    kf = fn.shape[1]
    gnodes = fn[bf].ravel()
    gfaces = np.repeat(bf, kf)
    order = np.argsort(gnodes, kind="stable")
    n2g_ptr = _group_ptr(gnodes[order], nn)
    n2g_idx = gfaces[order].astype(I32)
    A["n2g_ptr"], A["n2g_idx"] = n2g_ptr, n2g_idx
    A["ghostnid_ptr"], A["ghostnid_idx"] = ragged_union(c2n_ptr, flat_nodes, n2g_ptr, n2g_idx)

    # ---- centre->vertex weights, ddm_utils2d.py:608-705 / ddm_utils3d.py:813-981
    _vertex_weights(A, center, gc, vertex, dim)

    # ---- diamond cells, ddm_utils2d.py:553-605 / ddm_utils3d.py:459-527
    inner = name == 0
    v_1 = center[cellid[:, 0], :dim]
    v_2 = np.where(inner[:, None], center[np.where(inner, cellid[:, 1], 0), :dim], gc[:, :dim])
    if dim == 2:
        xy_1 = vertex[fn[:, 0], :2]
        xy_2 = vertex[fn[:, 1], :2]
        f1 = v_1 - xy_1
        f2 = xy_2 - v_1
        f3 = v_2 - xy_2
        f4 = xy_1 - v_2
        air = 0.5 * ((xy_2[:, 0] - xy_1[:, 0]) * (v_2[:, 1] - v_1[:, 1])
                     + (v_1[:, 0] - v_2[:, 0]) * (xy_2[:, 1] - xy_1[:, 1]))
        n1 = normal[:, 0]
        n2 = normal[:, 1]
        inv2a = 1.0 / (2.0 * air)
        A["faces_param1"] = inv2a * ((f1[:, 1] + f2[:, 1]) * n1 - (f1[:, 0] + f2[:, 0]) * n2)
        A["faces_param2"] = inv2a * ((f2[:, 1] + f3[:, 1]) * n1 - (f2[:, 0] + f3[:, 0]) * n2)
        A["faces_param3"] = inv2a * ((f3[:, 1] + f4[:, 1]) * n1 - (f3[:, 0] + f4[:, 0]) * n2)
        A["faces_param4"] = inv2a * ((f4[:, 1] + f1[:, 1]) * n1 - (f4[:, 0] + f1[:, 0]) * n2)
        A["faces_f_1"], A["faces_f_2"], A["faces_f_3"], A["faces_f_4"] = f1, f2, f3, f4
    else:
        i_1, i_2, i_3 = fn[:, 0], fn[:, 1], fn[:, 2]
        i_4 = i_3
        P1, P2, P3, P4 = (vertex[i, :3] for i in (i_1, i_2, i_3, i_4))
        s1 = v_2 - P2
        s2 = P4 - P2
        s3 = v_1 - P2
        f1 = (0.5 * _cross(s1, s2)) + (0.5 * _cross(s2, s3))
        s4 = v_2 - P3
        s5 = P1 - P3
        s6 = v_1 - P3
        f2 = (0.5 * _cross(s4, s5)) + (0.5 * _cross(s5, s6))
        air = _dot3(normal, v_2 - v_1)
        A["faces_param1"] = _dot3(f1, normal) / air
        A["faces_param2"] = _dot3(f2, normal) / air
        A["faces_param3"] = _dot3(normal, normal) / air
        A["faces_f_1"], A["faces_f_2"] = f1, f2
        A["faces_f_3"] = np.zeros((nf, 3))
        A["faces_f_4"] = np.zeros((nf, 3))
    A["faces_airDiamond"] = air

    if dim == 2:
        A["faces_dist_ortho"] = _dist_ortho_2d(A, center, fcenter, normal, cellid)
    else:
        A["faces_dist_ortho"] = np.zeros(nf)
    return A


def _vertex_weights(A, center, gc, vertex, dim):
    nn = A["nbnodes"]
    n2c_ptr, n2c_idx = A["n2c_ptr"], A["n2c_idx"]
    n2g_ptr, n2g_idx = A["n2g_ptr"], A["n2g_idx"]
    # per node, cells first then ghosts, each in ascending order; summed in
    # that order with an explicit sequential loop over the (short) rows.
    ptr = np.zeros(nn + 1, dtype=np.int64)
    cnt = np.diff(n2c_ptr) + np.diff(n2g_ptr)
    np.cumsum(cnt, out=ptr[1:])
    pts = np.zeros((int(ptr[-1]), 3))
    node_of = np.repeat(np.arange(nn), cnt)
    pos = np.arange(len(pts)) - np.repeat(ptr[:-1], cnt)
    ccnt = np.diff(n2c_ptr)
    is_cell = pos < np.repeat(ccnt, cnt)
    pts[is_cell] = center[n2c_idx]
    pts[~is_cell, :dim] = gc[n2g_idx, :dim]
    R = pts - vertex[node_of, :3]
    if dim == 2:
        R[:, 2] = 0.0
    width = int(cnt.max())
    acc = {k: np.zeros(nn) for k in ("xx", "yy", "zz", "xy", "xz", "yz", "x", "y", "z")}
    for j in range(width):
        m = cnt > j
        r = R[ptr[:-1][m] + j]
        acc["xx"][m] += r[:, 0] * r[:, 0]
        acc["yy"][m] += r[:, 1] * r[:, 1]
        acc["zz"][m] += r[:, 2] * r[:, 2]
        acc["xy"][m] += r[:, 0] * r[:, 1]
        acc["xz"][m] += r[:, 0] * r[:, 2]
        acc["yz"][m] += r[:, 1] * r[:, 2]
        acc["x"][m] += r[:, 0]
        acc["y"][m] += r[:, 1]
        acc["z"][m] += r[:, 2]
    Ixx, Iyy, Izz = acc["xx"], acc["yy"], acc["zz"]
    Ixy, Ixz, Iyz = acc["xy"], acc["xz"], acc["yz"]
    Rx, Ry, Rz = acc["x"], acc["y"], acc["z"]
    with np.errstate(divide="ignore", invalid="ignore"):
        if dim == 2:
            D = Ixx * Iyy - Ixy * Ixy
            lx = (Ixy * Ry - Iyy * Rx) / D
            ly = (Ixy * Rx - Ixx * Ry) / D
            lz = np.zeros(nn)
            Rz = np.zeros(nn)
        else:
            D = Ixx * Iyy * Izz + 2 * Ixy * Ixz * Iyz - Ixx * Iyz * Iyz - Iyy * Ixz * Ixz - Izz * Ixy * Ixy
            lx = ((Iyz * Iyz - Iyy * Izz) * Rx + (Ixy * Izz - Ixz * Iyz) * Ry + (Ixz * Iyy - Ixy * Iyz) * Rz) / D
            ly = ((Ixy * Izz - Ixz * Iyz) * Rx + (Ixz * Ixz - Ixx * Izz) * Ry + (Iyz * Ixx - Ixz * Ixy) * Rz) / D
            lz = ((Ixz * Iyy - Ixy * Iyz) * Rx + (Iyz * Ixx - Ixz * Ixy) * Ry + (Ixy * Ixy - Ixx * Iyy) * Rz) / D
    A["nodes_R_x"], A["nodes_R_y"], A["nodes_R_z"] = Rx, Ry, Rz
    A["nodes_lambda_x"], A["nodes_lambda_y"], A["nodes_lambda_z"] = lx, ly, lz
    A["nodes_number"] = cnt.astype(I32)


def _dist_ortho_2d(A, center, fcenter, normal, cellid):
    nf = len(cellid)
    d = np.zeros(nf)
    bf = A["boundaryfaces"].astype(np.int64)
    inner = A["innerfaces"].astype(np.int64)

    def proj_dist(K, f):
        v = center[K] - fcenter[f]
        u = normal[f]
        s = (v[:, 0] * u[:, 0] + v[:, 1] * u[:, 1])
        p = center[K] - s[:, None] * u
        z0 = center[K][:, 0] - p[:, 0]
        z1 = center[K][:, 1] - p[:, 1]
        return np.sqrt(z0 ** 2 + z1 ** 2)

    d[bf] = 2 * proj_dist(cellid[bf, 0], bf)
    d[inner] = proj_dist(cellid[inner, 0], inner) + proj_dist(cellid[inner, 1], inner)
    return d
