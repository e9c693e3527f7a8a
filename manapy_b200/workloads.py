"""The benchmark workloads: seeded meshes plus the physics set-up of each run.

Each workload names a mesh (``meshgen``), the initial state, the boundary
conditions and the solver options in the same terms a manapy driver script
uses (``manapy/examples/2D/advecdiff2d.py:104-147``,
``manapy/examples/2D/shallowwater2d.py:80-107``).

* ``C1``: 2D first-order upwind + diamond diffusion, 100x100 squares
  (20,000 triangles), 200 steps.
* ``C2``: 2D second-order (LSQ gradient + Barth limiter) advection-diffusion in
  a rotating velocity field, 1000x1000 squares (2,000,000 triangles), 1000 steps.
* ``C3``: 2D shallow-water dam break over a Gaussian bump, 2000x2000 squares
  (8,000,000 triangles), SRNH flux, 500 steps.
* ``C4``: 3D second-order advection-diffusion, 64^3 hexes x 6 tetrahedra
  (1,572,864 cells), 300 steps.
* ``E1``: 2D compressible Euler, first-order Rusanov (manapy's euler kernels), a
  pressure pulse in a sheared flow, 1000x1000 squares (2,000,000 triangles), 1000 steps.
"""
from __future__ import annotations

import dataclasses
from typing import Callable, Optional

import numpy as np

__all__ = ["Workload", "C1", "C2", "C3", "C4", "E1", "ALL", "pressure_pulse"]


def _gauss2d(cc):
    return np.exp(-((cc[:, 0] - 0.5) ** 2 + (cc[:, 1] - 0.5) ** 2) / 0.01)


def _gauss3d(cc):
    return np.exp(-((cc[:, 0] - 0.5) ** 2 + (cc[:, 1] - 0.5) ** 2 + (cc[:, 2] - 0.5) ** 2) / 0.01)


def _const_vel(u, v, w):
    def f(fc):
        n = len(fc)
        return np.full(n, u), np.full(n, v), np.full(n, w)
    return f


def _rotating(fc):
    x = fc[:, 0]
    y = fc[:, 1]
    return (np.sin(np.pi * x) * np.cos(np.pi * y), -np.cos(np.pi * x) * np.sin(np.pi * y),
            np.zeros(len(fc)))


def _dam_break(cc, left=2.0, right=1.0):
    x = cc[:, 0]
    y = cc[:, 1]
    h = np.where(x < 0.5, left, right).astype(np.float64)
    z = 0.1 * np.exp(-((x - 0.7) ** 2 + (y - 0.5) ** 2) / 0.02)
    zero = np.zeros(len(cc))
    return h, zero.copy(), zero.copy(), zero.copy(), z


def pressure_pulse(cc, gamma=1.4, seed=5):
    """Euler state (rho, P, rhou, rhov, rhoE): a Gaussian pressure pulse in a smooth density
    field with a shear flow; rho and P stay positive."""
    rng = np.random.default_rng(seed)
    x, y = cc[:, 0], cc[:, 1]
    rho = 1.0 + 0.2 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) + 0.01 * rng.standard_normal(len(x))
    P = 1.0 + 0.3 * np.exp(-40 * ((x - 0.5) ** 2 + (y - 0.5) ** 2))
    u = 0.3 * np.cos(np.pi * y)
    v = 0.2 * np.sin(np.pi * x)
    return [rho, P, rho * u, rho * v, P / (gamma - 1) + 0.5 * rho * (u * u + v * v)]


_DIRICHLET0_2D = ({"in": "dirichlet", "out": "dirichlet", "upper": "dirichlet", "bottom": "dirichlet"},
                  {"in": 0.0, "out": 0.0, "upper": 0.0, "bottom": 0.0})
_DIRICHLET0_3D = ({"in": "dirichlet", "out": "dirichlet", "upper": "dirichlet", "bottom": "dirichlet",
                   "front": "dirichlet", "back": "dirichlet"},
                  {"in": 0.0, "out": 0.0, "upper": 0.0, "bottom": 0.0, "front": 0.0, "back": 0.0})


@dataclasses.dataclass(frozen=True)
class Workload:
    name: str
    kind: str  # "advdiff", "sw" or "euler"
    dim: int
    n: int
    steps: int
    order: int
    cfl: float
    seed: int = 0
    diffusion: tuple = (0.0, 0.0, 0.0)
    velocity: Optional[Callable] = None
    init: Optional[Callable] = None
    init_sw: Optional[Callable] = None
    grav: float = 9.81
    init_euler: Optional[Callable] = None
    gamma: float = 1.4
    bc: Optional[dict] = None
    bc_values: Optional[dict] = None

    @property
    def cells(self) -> int:
        return 2 * self.n * self.n if self.dim == 2 else 6 * self.n ** 3

    def scaled(self, **kw) -> "Workload":
        return dataclasses.replace(self, **kw)

    def mesh(self):
        from . import meshgen
        if self.dim == 2:
            return meshgen.square_triangles(self.n, seed=self.seed)
        return meshgen.cube_tetrahedra(self.n, seed=self.seed)


C1 = Workload("C1-adv-diff-2d-o1-20k", "advdiff", 2, n=100, steps=200, order=1, cfl=0.8,
              diffusion=(1e-3, 1e-3, 0.0), velocity=_const_vel(1.0, 0.5, 0.0), init=_gauss2d,
              bc=_DIRICHLET0_2D[0], bc_values=_DIRICHLET0_2D[1])
C2 = Workload("C2-adv-diff-2d-o2-2M", "advdiff", 2, n=1000, steps=1000, order=2, cfl=0.8,
              diffusion=(5e-4, 5e-4, 0.0), velocity=_rotating, init=_gauss2d,
              bc=_DIRICHLET0_2D[0], bc_values=_DIRICHLET0_2D[1])
C3 = Workload("C3-shallow-water-2d-8M", "sw", 2, n=2000, steps=500, order=1, cfl=0.5,
              init_sw=_dam_break, grav=9.81)
C4 = Workload("C4-adv-diff-3d-o2-1.57M", "advdiff", 3, n=64, steps=300, order=2, cfl=0.8,
              diffusion=(1e-3, 1e-3, 1e-3), velocity=_const_vel(1.0, 0.5, 0.25), init=_gauss3d,
              bc=_DIRICHLET0_3D[0], bc_values=_DIRICHLET0_3D[1])

E1 = Workload("E1-euler-rusanov-2d-2M", "euler", 2, n=1000, steps=1000, order=1, cfl=0.5,
              init_euler=pressure_pulse, gamma=1.4)

ALL = {"C1": C1, "C2": C2, "C3": C3, "C4": C4, "E1": E1}
