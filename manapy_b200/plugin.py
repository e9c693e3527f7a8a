"""CUDA implementations behind ``CUDABackend.compile`` (filled in below)."""
from __future__ import annotations

KERNELS = {}


def bind(impl, domain, name):
    def call(*args, **kwargs):
        return impl(domain, *args, **kwargs)
    call.__name__ = name
    return call
