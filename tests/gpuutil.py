"""Helpers of the GPU parity tests: device tensors and C-ABI calls."""
import numpy as np
import torch

from manapy_b200 import _lib
from manapy_b200.device import DeviceBC, DeviceMesh


_KEEP = []  # tensors whose raw pointers were handed to asynchronous kernels


def T(a, dev="cuda"):
    t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    _KEEP.append(t)
    return t


def Z(n, dev="cuda"):
    return torch.zeros(int(n), dtype=torch.float64, device=dev)


def P(t):
    return t.data_ptr()


def H(t):
    torch.cuda.synchronize()
    out = t.cpu().numpy()
    _KEEP.clear()
    return out


def stream():
    return torch.cuda.current_stream().cuda_stream


def call(name, *args):
    _lib.call(name, *args)


def mesh(A, reorder=False):
    return DeviceMesh(A, "cuda", reorder=reorder)


def bc(A, resolved, mesh=None):
    return DeviceBC(A, resolved, "cuda", mesh=mesh)
