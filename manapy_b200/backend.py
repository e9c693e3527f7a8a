"""The kernel plugin point: ``CUDABackend.compile(func, signature)``.

manapy compiles each kernel with ``CPUBackend.compile`` (Numba,
``manapy/backends/cpu/backend.py:69-93``) and calls the result positionally
with numpy arrays.  ``CUDABackend.compile`` instead returns a callable bound to
the sm_100a implementation of the kernel with the same name and argument list:
field arguments are uploaded, the kernel runs on the domain's device tables,
and output arrays are written back in place.  Mesh-table arguments are taken
from the domain the backend belongs to (they must be that domain's arrays).
"""
from __future__ import annotations

from . import plugin

__all__ = ["CUDABackend"]


class CUDABackend:
    name = "cuda"

    def __init__(self, domain, float_precision="double", int_precision="signed"):
        self.domain = domain
        self.backend = "cuda"
        self.device = "cuda"
        self.float_precision = "float64"
        self.int_precision = "int32" if int_precision == "signed" else "uint32"

    @classmethod
    def for_manapy_domain(cls, manapy_domain, device="cuda"):
        """Backend for a domain built by manapy itself: the device tables are rebuilt
        from its element and vertex arrays (the same arrays manapy derives its
        geometry from), so kernel arguments taken from that domain line up."""
        from .domain import Domain
        nodeid = manapy_domain.cells.nodeid
        vertex = manapy_domain.nodes.vertex
        dom = Domain(dim=int(manapy_domain.dim), mesh=(nodeid, vertex), device=device)
        return cls(dom)

    def compile(self, func, signature=False, forcedbackend=None, outer=False):
        name = getattr(func, "__name__", None)
        impl = plugin.KERNELS.get(name)
        if impl is None:
            raise NotImplementedError("no CUDA implementation of manapy kernel %r" % name)
        return plugin.bind(impl, self.domain, name)
