"""Helpers for the GPU tests: numpy <-> device tensors and raw-pointer calls."""
import ctypes as C

import numpy as np
import torch

from diploma_thesis_b200 import _lib
from diploma_thesis_b200.api import ptr, stream_handle


def dev(a: np.ndarray) -> torch.Tensor:
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    elif a.dtype == np.uint64:
        a = a.view(np.int64)
    return torch.from_numpy(a.copy()).cuda()


def host(t: torch.Tensor, dtype=None) -> np.ndarray:
    torch.cuda.synchronize()
    a = t.detach().cpu().numpy()
    if dtype is not None:
        a = a.view(dtype)
    return a


def empty(shape, dtype=torch.float32) -> torch.Tensor:
    return torch.zeros(shape, dtype=dtype, device="cuda")


def call(name, *args):
    _lib.call(name, *args)


S = stream_handle
P = ptr
F3 = C.c_float * 3
F4 = C.c_float * 4
