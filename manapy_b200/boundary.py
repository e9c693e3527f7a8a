"""Boundary-condition resolution, as manapy's ``Variable`` wires it.

``resolve(mesh, BC, values)`` turns the user's ``{side: type}`` and
``{side: value}`` dicts into per-face ghost rules, following
``Variable._update_boundaries`` (``manapy/ast/core.py:105-335``) and the ghost
kernels of ``manapy/boundary/bc_utils.py:45-68``:

* ``dirichlet``: ghost = the face's prescribed value (a constant, or a callable
  ``f(x, y, z)`` evaluated at the face centre);
* ``neumann`` (and ``BC=None``): ghost = the interior cell value;
* ``nonslip``: ghost = minus the interior cell value;
* ``neumannNH``: ghost = cell value + prescribed gradient x orthogonal distance;
* ``slip``: manapy defines no ghost rule of its own for it
  (``manapy/boundary/bc.py:59-76``) and falls back to the class-level rule of the
  first boundary type the process created, which is ``neumann`` whenever a
  variable without explicit BCs exists (the common case).  It is resolved as
  ``neumann`` here.

Two reference behaviours are reproduced on purpose:

* all ``dirichlet`` sides share one face-value array, and a ``dirichlet`` side
  listed *after* a ``neumann``/``slip``/``nonslip`` side writes its values into
  the variable's cell array at the face indices and reads its ghost values back
  from the cell array at the face indices (``core.py:125-207``, the rebinding
  ``valueface = self.cell`` at ``:146,266,290,306``).  Where a face index is
  beyond the cell array this is undefined in the reference and raises
  ``ValueError`` here;
* face gradients are computed for inner, ``dirichlet`` and ``neumann``-list faces
  only; ``neumannNH`` faces keep their previous face gradient
  (``core.py:480-490``).
"""
from __future__ import annotations

from types import LambdaType

import numpy as np

# ghost rule per face
G_NONE, G_DIRICHLET, G_NEUMANN, G_NONSLIP, G_NEUMANN_NH, G_CELL_AT_FACE = 0, 1, 2, 3, 4, 5

SIDES_2D = ("in", "out", "bottom", "upper")
SIDES_3D = ("in", "out", "bottom", "upper", "front", "back")
SIDE_LIST = {"in": "infaces", "out": "outfaces", "upper": "upperfaces", "bottom": "bottomfaces",
             "front": "frontfaces", "back": "backfaces"}
SIDE_TAG = {"in": 1, "out": 2, "upper": 3, "bottom": 4, "front": 5, "back": 6}


class ResolvedBC:
    """Per-face ghost rules of one variable."""

    def __init__(self, nbfaces):
        self.kind = np.zeros(nbfaces, dtype=np.int8)
        self.value = np.zeros(nbfaces, dtype=np.float64)   # dirichlet value / NH gradient
        self.dirichletfaces = np.zeros(0, dtype=np.int32)
        self.neumannfaces = np.zeros(0, dtype=np.int32)
        self.sides = {}          # side -> (type, faces)
        self.cell_writes = None  # (face ids, values) written into the cell array at set-up

    @property
    def has_cell_at_face(self):
        return bool(np.any(self.kind == G_CELL_AT_FACE))


def _eval(val, centers):
    if isinstance(val, LambdaType):
        return np.array([val(c[0], c[1], c[2]) for c in centers], dtype=np.float64)
    if isinstance(val, (int, float, np.integer, np.floating)):
        return np.full(len(centers), float(val))
    raise ValueError("boundary value must be a number or a function f(x, y, z)")


def resolve(mesh, BC=None, values=None):
    """Resolve ``BC``/``values`` for a mesh exposing manapy's face lists."""
    A = mesh
    dim = A["dim"]
    sides = SIDES_2D if dim == 2 else SIDES_3D
    R = ResolvedBC(A["nbfaces"])
    fc = A["faces_center"]
    if BC is None:
        neu = []
        for s in sides:
            f = A[SIDE_LIST[s]]
            R.kind[f] = G_NEUMANN
            R.sides[s] = ("neumann", f)
            neu.append(f)
        R.neumannfaces = np.sort(np.concatenate(neu)).astype(np.int32)
        return R

    missing = [s for s in sides if s not in BC]
    if missing:
        raise ValueError("boundary condition missing for side(s) %s" % ", ".join(missing))
    values = values or {}
    valueface_is_cell = False
    dir_faces, neu_faces = [], []
    cell_writes_f, cell_writes_v = [], []
    for loc, bct in BC.items():
        if loc not in sides:
            raise ValueError("unknown boundary side %r" % loc)
        f = A[SIDE_LIST[loc]]
        if bct == "periodic":
            raise ValueError("BC must be not periodic for " + str(loc))
        if bct in ("dirichlet", "neumannNH"):
            if loc not in values:
                raise ValueError("Value of dirichlet BC for " + str(loc) + " faces must be given")
            v = _eval(values[loc], fc[f])
            if bct == "dirichlet":
                dir_faces.append(f)
                if valueface_is_cell:
                    if len(f) and int(f.max()) >= A["nbcells"]:
                        raise ValueError(
                            "dirichlet side %r follows a neumann-type side: manapy then reads the "
                            "boundary value from the cell array at face indices beyond its "
                            "length (undefined); list dirichlet sides first" % loc)
                    R.kind[f] = G_CELL_AT_FACE
                    cell_writes_f.append(f)
                    cell_writes_v.append(v)
                else:
                    R.kind[f] = G_DIRICHLET
                    R.value[f] = v
            else:
                if valueface_is_cell:
                    raise ValueError(
                        "neumannNH side %r follows a neumann-type side: manapy then takes the "
                        "prescribed gradient from the cell array at face indices; list it first"
                        % loc)
                R.kind[f] = G_NEUMANN_NH
                R.value[f] = v
        elif bct in ("neumann", "slip", "nonslip"):
            neu_faces.append(f)
            R.kind[f] = G_NONSLIP if bct == "nonslip" else G_NEUMANN
            valueface_is_cell = True
        else:
            raise ValueError("unknown boundary type %r for %s" % (bct, loc))
        R.sides[loc] = (bct, f)
    if dir_faces:
        R.dirichletfaces = np.sort(np.concatenate(dir_faces)).astype(np.int32)
    if neu_faces:
        R.neumannfaces = np.sort(np.concatenate(neu_faces)).astype(np.int32)
    if cell_writes_f:
        R.cell_writes = (np.concatenate(cell_writes_f).astype(np.int64), np.concatenate(cell_writes_v))
    return R
