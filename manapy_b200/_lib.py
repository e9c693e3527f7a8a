"""ctypes binding of ``lib/libmanapy_b200.so`` (the C ABI in ``include/manapy_b200.h``).

The library is built in-tree by ``manapy_b200.build.build()``.  Importing
this module does not load it; ``lib()`` does, and raises ``RuntimeError`` when
the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# MANAPY_B200_LIB selects another build of the same library (A/B comparisons of build options)
LIB_PATH = os.environ.get("MANAPY_B200_LIB") or os.path.join(HERE, "lib", "libmanapy_b200.so")

MB_OK, MB_EINVAL, MB_ECUDA, MB_ETOOBIG, MB_ENONFINITE, MB_ENEGATIVE = 0, -1, -2, -3, -4, -5
NOALLOC_SCRATCH_DOUBLES = 2 * 1024 * 1024
G_NONE, G_DIRICHLET, G_NEUMANN, G_NONSLIP, G_NEUMANN_NH, G_CELL_AT_FACE = 0, 1, 2, 3, 4, 5

_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_d = ctypes.c_double


class MbMesh(ctypes.Structure):
    _fields_ = [("dim", _i32), ("nbcells", _i32), ("nbfaces", _i32), ("nbnodes", _i32),
                ("nlf", _i32), ("variant", _i32),
                ("cell_center", _vp), ("cell_volume", _vp), ("cell_faces", _vp),
                ("cell_order", _vp), ("cellnid_ptr", _vp), ("cellnid_idx", _vp),
                ("ghostnid_ptr", _vp), ("ghostnid_idx", _vp),
                ("face_cellid", _vp), ("face_nodeid", _vp), ("face_name", _vp),
                ("face_normal", _vp), ("face_center", _vp), ("face_mesure", _vp),
                ("face_ghostcenter", _vp), ("face_air", _vp), ("face_f", _vp), ("face_dist", _vp),
                ("n2c_ptr", _vp), ("n2c_idx", _vp), ("n2c_alpha", _vp),
                ("n2g_ptr", _vp), ("n2g_idx", _vp), ("n2g_alpha", _vp),
                ("cell_cellfid", _vp), ("cell_nf", _vp), ("cell_vertex1", _vp),
                ("cell_vtx", _vp), ("cell_nbr", _vp), ("cell_flags", _vp), ("node_coord", _vp), ("cell_xy", _vp),
                ("lsq_sell_ptr", _vp), ("lsq_sell_idx", _vp), ("n2c_sell_ptr", _vp), ("n2c_sell_idx", _vp),
                ("n2c_sell_alpha", _vp), ("n2c_sell_alpha_f32", _vp), ("face_nm_f32", _vp), ("cell_lsq", _vp),
                ("cell_edges", _vp), ("edge_origin", _vp), ("edge_sell_ptr", _vp), ("edge_sell_idx", _vp),
                ("nbedges", _i32), ("pad_", _i32), ("n2c_sum_ptr", _vp), ("n2c_sum_idx", _vp),
                ("n2c_sum_alpha", _vp)]


class MbBC(ctypes.Structure):
    _fields_ = [("kind", _vp), ("value", _vp), ("face_grad_on", _vp)]


class MbAdvDiffParams(ctypes.Structure):
    _fields_ = [("order", _i32), ("diffusion", _i32), ("Dxx", _d), ("Dyy", _d), ("Dzz", _d)]


class MbAdvDiffItem(ctypes.Structure):
    _fields_ = [("m", MbMesh), ("bc", MbBC), ("p", MbAdvDiffParams), ("w", _vp * 2), ("lo", _vp * 2), ("sign_cf", _vp),
                ("src", _vp), ("dt_dev", _vp), ("cell_scratch", _vp), ("node_scratch", _vp),
                ("start_step", _i32), ("end_step", _i32), ("p1_begin", _i32), ("p1_cell_blocks", _i32),
                ("p2_begin", _i32), ("pad_", _i32)]


class MbSwItem(ctypes.Structure):
    _fields_ = [("m", MbMesh), ("q", (_vp * 4) * 2), ("lo", (_vp * 4) * 2), ("Z", _vp), ("face_flux", _vp), ("dt", _vp),
                ("cfl", _d), ("grav", _d), ("start_step", _i32), ("end_step", _i32), ("f_begin", _i32),
                ("c_begin", _i32)]


class MbAdvDiffItemF64(ctypes.Structure):
    _fields_ = [("m", MbMesh), ("bc", MbBC), ("p", MbAdvDiffParams), ("w", _vp * 2), ("sign_cf", _vp),
                ("src", _vp), ("dt_dev", _vp), ("cell_scratch", _vp), ("node_scratch", _vp),
                ("start_step", _i32), ("end_step", _i32), ("p1_begin", _i32), ("p1_cell_blocks", _i32),
                ("p2_begin", _i32), ("pad_", _i32)]


class MbSwItemF64(ctypes.Structure):
    _fields_ = [("m", MbMesh), ("q", (_vp * 5) * 2), ("face_flux", _vp), ("dt", _vp), ("cfl", _d), ("grav", _d),
                ("start_step", _i32), ("end_step", _i32), ("f_begin", _i32), ("c_begin", _i32)]


WALLS = {"neumann": 0, "reflective": 1}

# mb_check_tables: table ids -> (device table holding the checked values, offsets table or
# None, first checked column offset, accepted range as a function of (nbcells, nbfaces,
# nbnodes))
CHECK_TABLES = (
    ("cell_faces", None, 0, lambda c, f, n: (0, f)),
    ("cellnid_idx", "cellnid_ptr", 0, lambda c, f, n: (0, c)),
    ("ghostnid_idx", "ghostnid_ptr", 0, lambda c, f, n: (0, f)),
    ("face_cellid", None, 0, lambda c, f, n: (0, c)),
    ("face_cellid", None, 1, lambda c, f, n: (-1, c)),
    ("face_nodeid", None, 0, lambda c, f, n: (0, n)),
    ("n2c_idx", "n2c_ptr", 0, lambda c, f, n: (0, c)),
    ("n2g_idx", "n2g_ptr", 0, lambda c, f, n: (0, f)),
    ("cell_cellfid", None, 0, lambda c, f, n: (0, c)),
    ("cell_vtx", None, 0, lambda c, f, n: (0, n)),
    ("cell_nbr", None, 0, lambda c, f, n: (-f, c)),
    ("lsq_sell_idx", "lsq_sell_ptr", 0, lambda c, f, n: (-1, c)),
    ("n2c_sell_idx", "n2c_sell_ptr", 0, lambda c, f, n: (0, c)),
    ("cell_edges", None, 0, lambda c, f, n: (0, None)),
    ("edge_origin", None, 0, lambda c, f, n: (0, n)),
    ("edge_sell_idx", "edge_sell_ptr", 0, lambda c, f, n: (-1, c)),
    ("n2c_sum_idx", "n2c_sum_ptr", 0, lambda c, f, n: (-1, c)),
)


def decode_table_check(key):
    """mb_check_tables' result -> None (all tables valid) or (table, offsets?, position):
    the device table name (the offsets table's name when offsets? is true) and the flat
    position of the first bad entry in it."""
    key = int(key)
    if key == 2 ** 64 - 1:
        return None
    tid, offs, pos = key >> 40, bool((key >> 39) & 1), key & ((1 << 39) - 1)
    name, ptr, col, _ = CHECK_TABLES[tid]
    if offs:
        return ptr, True, pos
    return name, False, pos + col

_M = ctypes.POINTER(MbMesh)
_B = ctypes.POINTER(MbBC)
_P5 = _vp * 5
_P4 = _vp * 4

# name -> argtypes (restype is int unless listed in _RESTYPES)
_SIGS = {
    "mb_facetocell": [_M, _vp, _vp, _vp],
    "mb_ghost_value": [_M, _B, _vp, _vp, _vp],
    "mb_cell_gradient": [_M, _vp, _vp, _vp, _vp, _vp, _vp],
    "mb_barthlimiter": [_M, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "mb_centertovertex": [_M, _vp, _vp, _vp, _vp],
    "mb_face_gradient": [_M, _B, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "mb_explicitscheme_convective": [_M, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _vp],
    "mb_explicitscheme_dissipative": [_M, _vp, _vp, _vp, _vp, _d, _d, _d, _vp],
    "mb_time_step": [_M, _vp, _vp, _vp, _d, _d, _d, _d, _vp, _vp],
    "mb_update_new_value": [_M, _vp, _vp, _vp, _vp, _vp, _vp],
    "mb_srnh_flux": [_i32, _vp, _vp, _vp, _d, _vp, _vp],
    "mb_time_step_sw": [_M, _vp, _vp, _vp, _d, _d, _d, _d, _vp, _vp],
    "mb_explicitscheme_convective_sw": [_M, _P5, _P5, _P5, _P4, _vp, _d, _i32, _vp, _vp],
    "mb_term_source_srnh_sw": [_M, _vp, _vp, _vp, _vp, _d, _vp, _vp, _vp],
    "mb_update_sw": [_M, _P5, _P5, _vp, _vp, _vp, _vp],
    "mb_euler_rusanov_2d": [_M, _P5, _P5, _P4, _d, _vp],
    "mb_time_step_euler_2d": [_M, _P5, _d, _d, _vp, _vp],
    "mb_update_euler_2d": [_M, _P5, _P4, _d, _d, _vp],
    "mb_ghost_euler_neumann_2d": [_M, _P5, _P5, _vp, _vp, _vp],
    "mb_euler_dt_2d": [_M, _P5, _d, _d, _vp, _i32, _vp],
    "mb_euler_tables_2d": [_M, _vp, _vp, _vp],
    "mb_euler_step_2d": [_M, _P5, _P5, _d, _d, _vp, _vp, _vp, _vp, _i32, _vp, _vp],
    "mb_advdiff_step": [_M, _B, ctypes.POINTER(MbAdvDiffParams), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "mb_face_sign": [_M, _vp, _vp, _vp, _vp, _vp],
    "mb_pack_rows": [_M, _vp, _vp, _vp],
    "mb_lsq_matrix": [_M, _vp, _vp],
    "mb_check_tables": [_M, _vp, _vp],
    "mb_advdiff_step_split": [_M, _B, ctypes.POINTER(MbAdvDiffParams), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32,
                              _i32, _vp],
    "mb_advdiff_step_rows": [_M, _B, ctypes.POINTER(MbAdvDiffParams), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                             _vp],
    "mb_cell_face_sign": [_M, _vp, _vp, _vp, _vp, _vp],
    "mb_advdiff_step_noalloc": [_M, _B, ctypes.POINTER(MbAdvDiffParams), _vp, _vp, _vp, _vp, _vp, _vp],
    "mb_cell_face_sign_f32c": [_M, _vp, _vp, _vp],
    "mb_advdiff_step_f32c": [_M, _B, ctypes.POINTER(MbAdvDiffParams), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                             _vp, _vp],
    "mb_sw_step_f32c": [_M, _P5, _P5, _P4, _P4, _d, _d, _i32, _vp, _vp, _vp, _vp],
    "mb_advdiff_batch_step_f32c": [_vp, _vp, _i32, _vp, _i32, _i32, _i32, _vp, _vp],
    "mb_sw_batch_step_f32c": [_vp, _vp, _i32, _vp, _i32, _vp, _vp],
    "mb_sw_step": [_M, _P5, _P5, _d, _d, _i32, _vp, _vp, _vp, _vp, _vp],
    "mb_sw_dt": [_M, _vp, _vp, _vp, _d, _d, _vp, _vp],
    "mb_sw_step_ex": [_M, _P5, _P5, _d, _d, _i32, _i32, _vp, _vp, _vp, _vp, _vp],
    "mb_sw_step_split": [_M, _P5, _P5, _d, _d, _i32, _i32, _vp, _vp, _vp, _vp, _i32, _i32, _vp],
    "mb_sw_step_f32c_ex": [_M, _P5, _P5, _P4, _P4, _d, _d, _i32, _i32, _vp, _vp, _vp, _vp],
    "mb_advdiff_batch_step": [_vp, _vp, _i32, _vp, _i32, _i32, _i32, _vp, _vp],
    "mb_sw_batch_step": [_vp, _vp, _i32, _vp, _i32, _vp, _vp],
    "mb_check_state": [_vp, _vp, ctypes.c_int64, _i32, _vp, _vp],
    "mb_halo_pack": [_vp, _i32, _vp, ctypes.c_int64, _vp, _vp],
    "mb_halo_unpack": [_vp, _i32, _vp, ctypes.c_int64, _vp, _vp],
    "mb_build_info": [],
}
_RESTYPES = {"mb_build_info": ctypes.c_char_p}

EXPORTED = tuple(_SIGS)

_lib = None


def lib(path: str = LIB_PATH):
    """Load the CUDA library (once); raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            "manapy_b200 CUDA library not found at %s; build it with "
            "`python -c 'import manapy_b200.build as b; b.build()'`" % path)
    L = ctypes.CDLL(path)
    for name, args in _SIGS.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    _lib = L
    return L


class MbError(RuntimeError):
    pass


def check(rc: int, name: str = "call"):
    if rc != MB_OK:
        what = {MB_EINVAL: "invalid argument", MB_ECUDA: "CUDA error",
                MB_ETOOBIG: "mesh too large for the built-in scratch", MB_ENONFINITE: "non-finite value",
                MB_ENEGATIVE: "negative value"}.get(rc, "error %d" % rc)
        raise MbError("%s failed: %s" % (name, what))


def call(name, *args):
    check(getattr(lib(), name)(*args), name)


def ptrs(addresses):
    """A host array of device pointers (for the multi-field entry points)."""
    return (_vp * len(addresses))(*addresses)


def p5(ptrs):
    return _P5(*ptrs)


def p4(ptrs):
    return _P4(*ptrs)
