"""2D Euler (``manapy/solvers/euler/fvm_utils2d.py``): the oracle against golden
vectors of the reference kernels (CPU), and the CUDA kernels against the oracle (GPU)."""
import os

import numpy as np
import pytest

from manapy_b200 import geometry as G

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ("rho", "P", "rhou", "rhov", "rhoE")


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(HERE, "golden", "k_euler.npz"))


@pytest.fixture(scope="module")
def mesh(gold):
    import oracle as O
    return O.Mesh(G.build(gold["in_elements"], gold["in_vertex"], 2))


def _q0(gold):
    return [gold[k + "0"].copy() for k in NAMES]


def _close(a, b, rtol):
    scale = max(1.0, float(np.max(np.abs(b))))
    return float(np.max(np.abs(np.asarray(a) - b))) <= rtol * scale


def test_oracle_matches_reference_kernels(gold, mesh):
    import oracle as O
    q = _q0(gold)
    g, ug, vg = O.ghost_neumann_euler_2d(mesh, q)
    for k, a in zip(NAMES, g):
        assert np.array_equal(a, gold["g_" + k]), k
    assert _close(ug, gold["g_u"], 1e-15) and _close(vg, gold["g_v"], 1e-15)
    rez = O.euler_rusanov_2d(mesh, q, g, float(gold["gamma"]))
    for k, a in zip(("rho", "rhou", "rhov", "rhoE"), rez):
        assert np.array_equal(a, gold["rez_" + k]), k          # same operations, same order: bit for bit
    # manapy compiles time_step_euler_2d with fastmath: agreement to rounding
    dt_c = O.time_step_euler_2d(mesh, q, float(gold["cfl"]), float(gold["gamma"]))
    assert _close(dt_c, gold["dt_c"], 1e-14)
    O.update_euler_2d(mesh, q, [gold["rez_" + k] for k in ("rho", "rhou", "rhov", "rhoE")], float(gold["gamma"]),
                      float(gold["dts"][0]))
    for k, a in zip(NAMES, q):
        assert _close(a, gold["new_" + k], 1e-14), k


def test_oracle_run_matches_reference_run(gold, mesh):
    import oracle as O
    q = _q0(gold)
    dts = [O.euler_step_2d(mesh, q, float(gold["cfl"]), float(gold["gamma"])) for _ in range(len(gold["dts"]))]
    assert np.allclose(dts, gold["dts"], rtol=1e-13, atol=0)
    for k, a in zip(NAMES, q):
        assert _close(a, gold["final_" + k], 1e-12), k
