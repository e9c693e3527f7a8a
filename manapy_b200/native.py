"""ctypes binding of the native host mesh builder (``lib/libmanapy_b200_host.so``).

``tables2d(elements, vertex)`` returns every device table of a 2D triangle mesh
(the ``DeviceMesh`` tables, in the locality numbering), the permutations, and
the few manapy-numbered arrays the boundary set-up reads, computed in C++
(``host/mesh2d.cpp``) with the same operations as ``geometry.build`` +
``DeviceMesh``: the results are bit-identical, 20-50 times faster.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .build import HOST_OUT

_DT = {b"i": np.int32, b"l": np.int64, b"d": np.float64, b"f": np.float32, b"b": np.uint8}
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(HOST_OUT):
            from .build import build_host
            build_host()
        L = ctypes.CDLL(HOST_OUT)
        L.mbh_build2d.restype = ctypes.c_void_p
        L.mbh_build2d.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                                  ctypes.c_int32, ctypes.c_int32]
        L.mbh_error.restype = ctypes.c_char_p
        L.mbh_error.argtypes = [ctypes.c_void_p]
        L.mbh_count.restype = ctypes.c_int32
        L.mbh_count.argtypes = [ctypes.c_void_p]
        L.mbh_info.restype = ctypes.c_int32
        L.mbh_info.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_char_p),
                               ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]
        L.mbh_data.restype = ctypes.c_void_p
        L.mbh_data.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        L.mbh_free.argtypes = [ctypes.c_void_p]
        L.mbh_sell_aligned.restype = ctypes.c_void_p
        L.mbh_sell_aligned.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int32]
        L.mbh_geometry3d.restype = ctypes.c_void_p
        L.mbh_geometry3d.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64]
        _lib = L
    return _lib


def available():
    """True when the native host library loads (it is built with the CUDA library)."""
    try:
        lib()
        return True
    except OSError:
        return False


def tables2d(elements, vertex, reorder=True, full=False, stencil="manapy"):
    """dict name -> numpy array (see ``host/mesh2d.cpp``); raises ValueError on a bad mesh.
    ``full``: also every array of ``geometry.build`` as ``"A.<name>"``; ``stencil``: the
    layout of ``lsq_sell_*``, ``"manapy"`` (manapy's neighbour order) or ``"shared"`` (the
    slot-shared layout of ``sell_aligned``)."""
    if stencil not in ("manapy", "shared"):
        raise ValueError("stencil must be 'manapy' or 'shared'")
    el = np.ascontiguousarray(elements, dtype=np.int32)
    vx = np.ascontiguousarray(vertex, dtype=np.float64)
    if el.ndim != 2 or el.shape[1] != 4 or vx.ndim != 2 or vx.shape[1] != 4:
        raise ValueError("expected elements [nc, 4] and vertex [nn, 4]")
    L = lib()
    h = L.mbh_build2d(el.ctypes.data, len(el), vx.ctypes.data, len(vx), int(bool(reorder)), int(bool(full)),
                      int(stencil == "shared"))
    if not h:
        raise ValueError("empty mesh")
    return _read(L, h)


def sell_aligned(ptr, idx, slack=0):
    """(group_ptr, idx) of the slot-shared SELL-32 layout of a CSR table (``host/common.hpp``
    ``sell32_aligned``): rows in warps of 32, values that several rows of a warp hold placed
    in one slot for all of them where their free slots allow; ``slack`` extra slots per warp;
    empty slots -1."""
    p = np.ascontiguousarray(ptr, dtype=np.int64)
    ix = np.ascontiguousarray(idx, dtype=np.int32)
    if p.ndim != 1 or len(p) < 1 or p[0] != 0 or len(ix) != p[-1] or np.any(np.diff(p) < 0):
        raise ValueError("expected a CSR table (ptr from 0, ascending, idx of length ptr[-1])")
    L = lib()
    h = L.mbh_sell_aligned(p.ctypes.data, len(p) - 1, ix.ctypes.data, int(slack))
    if not h:
        raise ValueError("bad arguments")
    T = _read(L, h)
    return T["gptr"], T["idx"]


def geometry3d(elements, vertex):
    """Every array of ``geometry.build(elements, vertex, 3)`` from the native host builder
    (``host/geom3d.cpp``), bit-identical; raises ValueError on a bad mesh."""
    el = np.ascontiguousarray(elements, dtype=np.int32)
    vx = np.ascontiguousarray(vertex, dtype=np.float64)
    if el.ndim != 2 or el.shape[1] != 5 or vx.ndim != 2 or vx.shape[1] != 4:
        raise ValueError("expected elements [nc, 5] and vertex [nn, 4]")
    L = lib()
    h = L.mbh_geometry3d(el.ctypes.data, len(el), vx.ctypes.data, len(vx))
    if not h:
        raise ValueError("empty mesh")
    T = _read(L, h)
    A = {k[2:]: v for k, v in T.items()}
    A.update(dim=3, nbcells=len(el), nbnodes=len(vx), nbfaces=len(A["faces_name"]))
    return A


def _read(L, h):
    """The named tables of a builder result as numpy arrays viewing its buffers."""
    owner = _Handle(L, h)
    err = L.mbh_error(h)
    if err:
        raise ValueError(err.decode())
    # the arrays view the builder's own buffers (no copy); the handle is released when the
    # last of them is gone
    out = {}
    name = ctypes.c_char_p()
    dt = ctypes.create_string_buffer(1)
    shape = (ctypes.c_int64 * 3)()
    for k in range(L.mbh_count(h)):
        nd = L.mbh_info(h, k, ctypes.byref(name), dt, shape)
        shp = tuple(shape[d] for d in range(nd))
        dtype = np.dtype(_DT[dt.raw])
        n = int(np.prod(shp)) if shp else 0
        if n:
            buf = (ctypes.c_char * (n * dtype.itemsize)).from_address(L.mbh_data(h, k))
            buf.owner = owner
            out[name.value.decode()] = np.frombuffer(buf, dtype=dtype).reshape(shp)
        else:
            out[name.value.decode()] = np.zeros(shp, dtype=dtype)
    return out


class _Handle:
    """Owns one builder result; frees it when the last array viewing it is collected."""

    def __init__(self, L, h):
        self.L, self.h = L, h

    def __del__(self):
        if self.h:
            try:
                self.L.mbh_free(self.h)
            except Exception:          # interpreter shutdown: the library may be gone already
                pass
            self.h = None
