"""VTK XML unstructured-grid output (``.vtu`` pieces and the ``.pvtu`` index).

manapy writes its results with meshio (``manapy/ddm/domain.py:735-849``:
``save_on_cell_multi`` / ``save_on_node_multi`` write ``results/visu<rank>-<miter>.vtu``
and a ``visu<miter>.pvtu`` that lists the rank pieces).  This module writes the same
files without meshio: points as Float64 triples, triangle (VTK type 5) or
tetrahedron (type 10) cells, cell or point data arrays, base64 "binary" encoding
(a little-endian uint32 byte count followed by the data).
"""
from __future__ import annotations

import base64
import os

import numpy as np

__all__ = ["write_vtu", "write_pvtu", "read_vtu_arrays"]

_VTK_TYPE = {3: 5, 4: 10}          # nodes per cell -> VTK cell type
_NP_TO_VTK = {np.dtype(np.float64): "Float64", np.dtype(np.float32): "Float32",
              np.dtype(np.int32): "Int32", np.dtype(np.int64): "Int64", np.dtype(np.uint8): "UInt8"}


def _host(a):
    if hasattr(a, "detach"):  # a torch tensor, possibly on the GPU
        a = a.detach().cpu().numpy()
    return np.ascontiguousarray(a)


def _b64(a):
    raw = np.ascontiguousarray(a).astype(a.dtype.newbyteorder("<"), copy=False).tobytes()
    return base64.b64encode(np.uint32(len(raw)).tobytes() + raw).decode("ascii")


def _array(name, a, ncomp=1):
    return ('<DataArray type="%s" Name="%s" NumberOfComponents="%d" format="binary">\n%s\n</DataArray>\n'
            % (_NP_TO_VTK[a.dtype], name, ncomp, _b64(a)))


def write_vtu(path, points, cells, cell_data=None, point_data=None):
    """One unstructured-grid piece: ``points`` [nn, 3], ``cells`` [nc, 3 or 4] node ids."""
    pts = _host(points).astype(np.float64)[:, :3]
    conn = _host(cells).astype(np.int32)
    nc, k = conn.shape
    if k not in _VTK_TYPE:
        raise ValueError("cells must be triangles or tetrahedra")
    out = ['<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian" '
           'header_type="UInt32">\n<UnstructuredGrid>\n<Piece NumberOfPoints="%d" NumberOfCells="%d">\n'
           % (len(pts), nc)]
    out.append("<Points>\n" + _array("Points", pts.reshape(-1), 3) + "</Points>\n")
    out.append("<Cells>\n" + _array("connectivity", conn.reshape(-1))
               + _array("offsets", (k * np.arange(1, nc + 1)).astype(np.int32))
               + _array("types", np.full(nc, _VTK_TYPE[k], dtype=np.uint8)) + "</Cells>\n")
    for tag, data, n in (("CellData", cell_data, nc), ("PointData", point_data, len(pts))):
        if data:
            out.append("<%s>\n" % tag)
            for name, v in data.items():
                v = _host(v).astype(np.float64).reshape(-1)
                if len(v) != n:
                    raise ValueError("%s: %d values for %d %s" % (name, len(v), n, tag))
                out.append(_array(name, v))
            out.append("</%s>\n" % tag)
    out.append("</Piece>\n</UnstructuredGrid>\n</VTKFile>\n")
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "w") as f:
        f.write("".join(out))


def write_pvtu(path, pieces, names, on="cell"):
    """The parallel index listing ``pieces`` (file names) with arrays ``names``."""
    tag = "PCellData" if on == "cell" else "PPointData"
    lines = ['<?xml version="1.0"?>', '<VTKFile type="PUnstructuredGrid" version="0.1" byte_order="LittleEndian">',
             '<PUnstructuredGrid GhostLevel="0">', "<PPoints>",
             '<PDataArray type="Float64" Name="Points" NumberOfComponents="3" format="binary"/>', "</PPoints>",
             "<PCells>", '<PDataArray type="Int32" Name="connectivity" format="binary"/>',
             '<PDataArray type="Int32" Name="offsets" format="binary"/>',
             '<PDataArray type="UInt8" Name="types" format="binary"/>', "</PCells>",
             '<%s Scalars="%s">' % (tag, names[0] if names else "")]
    lines += ['<PDataArray type="Float64" Name="%s" format="binary"/>' % n for n in names]
    lines.append("</%s>" % tag)
    lines += ['<Piece Source="%s"/>' % p for p in pieces]
    lines += ["</PUnstructuredGrid>", "</VTKFile>"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def read_vtu_arrays(path):
    """Decode every DataArray of a file written by ``write_vtu`` (name -> numpy array)."""
    import re
    txt = open(path).read()
    rev = {v: k for k, v in _NP_TO_VTK.items()}
    out = {}
    for m in re.finditer(r'<DataArray type="(\w+)" Name="([^"]+)" NumberOfComponents="(\d+)" format="binary">\n'
                         r'([^<]*)\n</DataArray>', txt):
        raw = base64.b64decode(m.group(4))
        n = int(np.frombuffer(raw[:4], dtype="<u4")[0])
        a = np.frombuffer(raw[4:4 + n], dtype=rev[m.group(1)].newbyteorder("<"))
        k = int(m.group(3))
        out[m.group(2)] = a.reshape(-1, k) if k > 1 else a
    return out
