"""gmsh ``.msh`` reader (ASCII formats 4.1 and 2.2) producing manapy's mesh layout.

manapy reads a gmsh file through meshio and derives, per vertex, a boundary tag
from the physical groups of the boundary elements
(``manapy/partitions/meshpartitioning.py:160-194``,
``manapy/partitions/partitions_utils.py:16-111``); the cells keep gmsh's node
order and gain a count column (``convert_2d_cons_to_array``).  This module does
the same without meshio:

* points in the order of the ``$Nodes`` section (meshio's order), node tags
  mapped to 0-based indices;
* cells of the domain's dimension: triangles (2D) or tetrahedra (3D); other
  cell types (quadrangles, pyramids, hexahedra) are rejected;
* vertex tags from the boundary elements (lines in 2D, triangles and
  quadrangles in 3D), in manapy's three passes: physical tags 1 and 2 first
  (a later element overwrites an earlier one), then 3 and 4 on vertices not
  already tagged 1 or 2, then any tag on vertices still untagged;
* the physical tag of an element is the first physical tag of its entity
  (format 4.1) or its first tag (format 2.2), 0 when there is none.

Returns ``(elements, vertex)``: ``elements`` int32 [nc, k+1] (nodes then k),
``vertex`` float64 [nn, 4] (x, y, z, tag), the layout of manapy's per-rank HDF5
mesh files (``manapy/ddm/pure_ddm.py:21-33``).
"""
from __future__ import annotations

import numpy as np

__all__ = ["read_msh", "vertex_tags", "write_msh"]

# gmsh element type -> (name, number of nodes)
_TYPES = {1: ("line", 2), 2: ("triangle", 3), 3: ("quad", 4), 4: ("tetra", 4), 5: ("hexahedron", 8),
          6: ("wedge", 6), 7: ("pyramid", 5), 15: ("vertex", 1)}


def _sections(text):
    out = {}
    lines = text.splitlines()
    i = 0
    while i < len(lines):
        ln = lines[i].strip()
        if ln.startswith("$") and not ln.startswith("$End"):
            name = ln[1:]
            j = i + 1
            while j < len(lines) and lines[j].strip() != "$End" + name:
                j += 1
            if j == len(lines):
                raise ValueError("gmsh file: section $%s is not closed" % name)
            out[name] = lines[i + 1:j]
            i = j + 1
        else:
            i += 1
    return out


def _tokens(lines):
    return iter(" ".join(lines).split())


def _read_41(sec):
    # entities: physical tags per (dim, tag)
    phys = {}
    if "Entities" in sec:
        it = _tokens(sec["Entities"])
        counts = [int(next(it)) for _ in range(4)]
        for dim, cnt in enumerate(counts):
            for _ in range(cnt):
                tag = int(next(it))
                for _ in range(3 if dim == 0 else 6):
                    next(it)
                nphys = int(next(it))
                tags = [int(next(it)) for _ in range(nphys)]
                phys[(dim, tag)] = tags[0] if tags else 0
                if dim > 0:
                    nb = int(next(it))
                    for _ in range(nb):
                        next(it)
    it = _tokens(sec["Nodes"])
    nblocks, nnodes = int(next(it)), int(next(it))
    next(it), next(it)
    tags = np.empty(nnodes, dtype=np.int64)
    pts = np.empty((nnodes, 3), dtype=np.float64)
    k = 0
    for _ in range(nblocks):
        next(it), next(it)
        param = int(next(it))
        n = int(next(it))
        tags[k:k + n] = [int(next(it)) for _ in range(n)]
        for j in range(n):
            pts[k + j] = [float(next(it)) for _ in range(3)]
            if param:
                raise ValueError("gmsh file: parametric node coordinates are not supported")
        k += n
    it = _tokens(sec["Elements"])
    nblocks = int(next(it))
    next(it), next(it), next(it)
    blocks = []
    for _ in range(nblocks):
        edim, etag, etype, n = int(next(it)), int(next(it)), int(next(it)), int(next(it))
        if etype not in _TYPES:
            raise ValueError("gmsh file: element type %d is not supported" % etype)
        name, nn = _TYPES[etype]
        conn = np.empty((n, nn), dtype=np.int64)
        for j in range(n):
            next(it)
            conn[j] = [int(next(it)) for _ in range(nn)]
        blocks.append((name, conn, np.full(n, phys.get((edim, etag), 0), dtype=np.int64)))
    return tags, pts, blocks


def _read_22(sec):
    it = _tokens(sec["Nodes"])
    nnodes = int(next(it))
    tags = np.empty(nnodes, dtype=np.int64)
    pts = np.empty((nnodes, 3), dtype=np.float64)
    for j in range(nnodes):
        tags[j] = int(next(it))
        pts[j] = [float(next(it)) for _ in range(3)]
    it = _tokens(sec["Elements"])
    nel = int(next(it))
    per = {}
    for _ in range(nel):
        next(it)
        etype, ntags = int(next(it)), int(next(it))
        etags = [int(next(it)) for _ in range(ntags)]
        if etype not in _TYPES:
            raise ValueError("gmsh file: element type %d is not supported" % etype)
        name, nn = _TYPES[etype]
        conn = [int(next(it)) for _ in range(nn)]
        per.setdefault(name, ([], []))
        per[name][0].append(conn)
        per[name][1].append(etags[0] if etags else 0)
    blocks = [(name, np.array(c, dtype=np.int64).reshape(-1, _TYPES_BY_NAME[name]), np.array(p, dtype=np.int64))
              for name, (c, p) in per.items()]
    return tags, pts, blocks


_TYPES_BY_NAME = {name: nn for name, nn in _TYPES.values()}


def vertex_tags(nnodes, boundary):
    """manapy's vertex tags from boundary elements ``[(connectivity, physical tags)]``
    (``manapy/partitions/partitions_utils.py:16-111``, without periodic relabelling)."""
    g = np.zeros(nnodes, dtype=np.int32)
    for conn, ph in boundary:           # pass 1: tags 1 and 2, last write wins
        for row, t in zip(conn, ph):
            if t in (1, 2):
                g[row] = t
    for conn, ph in boundary:           # pass 2: tags 3 and 4 where not 1 or 2
        for row, t in zip(conn, ph):
            if t in (3, 4):
                for v in row:
                    if g[v] not in (1, 2):
                        g[v] = t
    for conn, ph in boundary:           # pass 3: any tag where still untagged
        for row, t in zip(conn, ph):
            for v in row:
                if g[v] == 0:
                    g[v] = t
    return g


def read_msh(path, dim):
    """``(elements, vertex)`` of a gmsh ASCII file for a ``dim``-dimensional domain."""
    with open(path) as f:
        text = f.read()
    sec = _sections(text)
    if "MeshFormat" not in sec:
        raise ValueError("%s: not a gmsh file" % path)
    version, ftype = sec["MeshFormat"][0].split()[:2]
    if ftype != "0":
        raise ValueError("%s: binary gmsh files are not supported" % path)
    if version.startswith("4"):
        tags, pts, blocks = _read_41(sec)
    elif version.startswith("2"):
        tags, pts, blocks = _read_22(sec)
    else:
        raise ValueError("%s: gmsh format %s is not supported" % (path, version))
    index = {int(t): k for k, t in enumerate(tags)}
    remap = np.vectorize(index.__getitem__, otypes=[np.int64])
    cell_name = {2: "triangle", 3: "tetra"}[dim]
    other = {2: ("quad",), 3: ("pyramid", "hexahedron", "wedge")}[dim]
    face_names = {2: ("line",), 3: ("triangle", "quad")}[dim]
    cells, boundary = [], []
    for name, conn, ph in blocks:
        if name in other:
            raise ValueError("%s: %s cells are not supported (triangles / tetrahedra only)" % (path, name))
        if name == cell_name:
            cells.append(remap(conn))
        elif name in face_names:
            boundary.append((remap(conn), ph))
    if not cells:
        raise ValueError("%s: no %s cells" % (path, cell_name))
    conn = np.concatenate(cells)
    k = conn.shape[1]
    elements = np.empty((len(conn), k + 1), dtype=np.int32)
    elements[:, :k] = conn
    elements[:, k] = k
    vertex = np.zeros((len(pts), 4), dtype=np.float64)
    vertex[:, :3] = pts
    vertex[:, 3] = vertex_tags(len(pts), boundary)
    return elements, vertex


def write_msh(path, elements, vertex, boundary):
    """Write a gmsh 4.1 ASCII file: cells ``elements`` (count column ignored), points
    ``vertex[:, :3]``, and ``boundary`` = [(physical tag, connectivity)] of boundary
    elements (lines in 2D, triangles in 3D), one entity per physical tag."""
    k = int(elements[0, -1])
    dim = 2 if k == 3 else 3
    nn = len(vertex)
    ctype = 2 if dim == 2 else 4
    btype = 1 if dim == 2 else 2
    L = ["$MeshFormat", "4.1 0 8", "$EndMeshFormat", "$Entities"]
    nb = len(boundary)
    counts = [0, nb, 1, 0] if dim == 2 else [0, 0, nb, 1]
    L.append(" ".join(map(str, counts)))
    bdim = dim - 1
    for t, _ in boundary:
        L.append("%d 0 0 0 1 1 1 1 %d 0" % (t, t))
    L.append("%d 0 0 0 1 1 1 0 0" % (nb + 1))
    L.append("$EndEntities")
    L += ["$Nodes", "1 %d 1 %d" % (nn, nn), "%d 1 0 %d" % (dim, nn)]
    L += [str(j + 1) for j in range(nn)]
    L += ["%.17g %.17g %.17g" % tuple(p) for p in vertex[:, :3]]
    L.append("$EndNodes")
    nel = len(elements) + sum(len(c) for _, c in boundary)
    L += ["$Elements", "%d %d 1 %d" % (nb + 1, nel, nel)]
    e = 1
    for t, conn in boundary:
        L.append("%d %d %d %d" % (bdim, t, btype, len(conn)))
        for row in conn:
            L.append(" ".join([str(e)] + [str(int(v) + 1) for v in row]))
            e += 1
    L.append("%d %d %d %d" % (dim, nb + 1, ctype, len(elements)))
    for row in elements[:, :k]:
        L.append(" ".join([str(e)] + [str(int(v) + 1) for v in row]))
        e += 1
    L.append("$EndElements")
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")
