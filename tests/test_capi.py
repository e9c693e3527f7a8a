"""The C-ABI library loads and exports every function the public header declares."""
import ctypes
import os
import re

from conftest import ROOT
import manapy_b200.build as build
from manapy_b200 import _lib


def header_functions():
    txt = open(os.path.join(ROOT, "include", "manapy_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(mb_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_header_symbols():
    path = build.build()
    lib = ctypes.CDLL(path)
    names = header_functions()
    assert len(names) >= 19
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers exactly the header
    assert sorted(_lib.EXPORTED) == names


def test_build_info():
    build.build()
    assert b"sm_100a" in _lib.lib().mb_build_info()


def test_struct_layouts_match_the_header(tmp_path):
    """ctypes mirrors of mb_mesh, mb_bc, mb_advdiff_params and the batch items have the
    C compiler's size and field offsets."""
    import subprocess
    structs = {"mb_mesh": _lib.MbMesh, "mb_bc": _lib.MbBC, "mb_advdiff_params": _lib.MbAdvDiffParams,
               "mb_advdiff_item": _lib.MbAdvDiffItem, "mb_sw_item": _lib.MbSwItem}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "manapy_b200.h"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (name, name))
        for field, _ in cls._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (name, field, name, field))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                 check=True).stdout.splitlines())
    for name, cls in structs.items():
        assert int(got[name]) == ctypes.sizeof(cls), name
        for field, _ in cls._fields_:
            assert int(got[name + "." + field]) == getattr(cls, field).offset, (name, field)


def test_entry_points_reject_null_arguments():
    """Every entry point validates its arguments on the host: null meshes, states and
    scratch give MB_EINVAL before any CUDA call (runs without a GPU).  mb_srnh_flux with
    zero states has nothing to do and succeeds."""
    import ctypes
    from manapy_b200 import _lib
    L = _lib.lib()
    for name, argt in _lib._SIGS.items():
        if name == "mb_build_info":
            continue
        args = []
        for t in argt:
            if isinstance(t, type) and issubclass(t, ctypes.Array):
                args.append(t())
            elif t in (ctypes.c_double, ctypes.c_float):
                args.append(0.0)
            elif t in (ctypes.c_int32, ctypes.c_int64, ctypes.c_int):
                args.append(0)
            else:
                args.append(None)
        rc = getattr(L, name)(*args)
        assert rc == (_lib.MB_OK if name == "mb_srnh_flux" else _lib.MB_EINVAL), (name, rc)


def test_table_check_keys_decode():
    from manapy_b200 import _lib
    assert _lib.decode_table_check(2 ** 64 - 1) is None
    assert _lib.decode_table_check((11 << 40) | 5) == ("lsq_sell_idx", False, 5)
    assert _lib.decode_table_check((1 << 40) | (1 << 39) | 9) == ("cellnid_ptr", True, 9)
    # face_cellid's second column is checked from face_cellid + 1
    assert _lib.decode_table_check((4 << 40) | 22) == ("face_cellid", False, 23)
    assert len(_lib.CHECK_TABLES) == 17
