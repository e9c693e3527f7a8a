"""manapy_b200: manapy's explicit finite-volume step on NVIDIA B200 (sm_100a).

Public surface mirrors manapy's: ``Domain``, ``Variable``, ``Struct`` and the
explicit solvers ``AdvectionDiffusionSolver``, ``AdvectionSolver``, ``DiffusionSolver`` and
``ShallowWaterSolver``.  The
arithmetic runs in hand-written CUDA kernels behind the C ABI of
``include/manapy_b200.h`` (``lib/libmanapy_b200.so``).
"""
from .base import Struct, make_get_conf  # noqa: F401
from .domain import Domain  # noqa: F401
from .variable import Variable  # noqa: F401
from .solvers import (AdvectionDiffusionSolver, AdvectionSolver, DiffusionSolver, EulerSolver,  # noqa: F401
                      ShallowWaterSolver)

__version__ = "0.1.0"
