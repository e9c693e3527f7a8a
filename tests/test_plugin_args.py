"""CUDABackend.compile on the CPU: every registered kernel takes exactly manapy's argument
list, and calls with a wrong one fail before any device work, as Python calls of manapy's
own kernels do."""
import inspect

import pytest

import manapy_b200 as M
from manapy_b200 import meshgen, plugin


def _fn(name):
    def f():
        pass
    f.__name__ = name
    return f


@pytest.fixture(scope="module")
def dom():
    el, vx = meshgen.square_triangles(4, seed=1)
    return M.Domain(dim=2, mesh=(el, vx))


@pytest.mark.parametrize("name", sorted(plugin.KERNELS))
def test_wrong_argument_lists_raise_type_error(dom, name):
    k = dom.backend.compile(_fn(name))
    n = len(plugin.KERNELS[name].params)
    assert k.__name__ == name and all(p in k.__doc__ for p in plugin.KERNELS[name].params)
    with pytest.raises(TypeError, match="takes %d arguments" % n):
        k(*([0] * (n + 1)))
    with pytest.raises(TypeError, match="missing arguments"):
        k(*([0] * (n - 1)))
    with pytest.raises(TypeError, match="unexpected argument"):
        k(*([0] * n), no_such_argument=1)


def test_unknown_kernel_is_not_implemented(dom):
    with pytest.raises(NotImplementedError):
        dom.backend.compile(_fn("no_such_kernel"))


def test_parameter_names_of_the_euler_kernels_follow_manapy():
    # manapy/solvers/euler/fvm_utils2d.py argument lists
    assert plugin.KERNELS["explicitscheme_euler_2d_rusanov"].params[:5] == ["rez_rho", "rez_rhou", "rez_rhov",
                                                                            "rez_rhoE", "rho_c"]
    assert plugin.KERNELS["time_step_euler_2d"].params == ["rho", "P", "rhou", "rhov", "cfl", "normal", "mesure",
                                                           "volume", "faceid", "gamma", "dt_c"]
    assert plugin.KERNELS["update_euler_2d_fvc"].params[-3:] == ["gamma", "dtime", "vol"]
    assert plugin.KERNELS["ghost_value_Neumann"].params[-1] == "t"
    assert inspect.isfunction(plugin.bind)
