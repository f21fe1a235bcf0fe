"""Helpers shared by the gpu tests (device arrays through torch)."""
import numpy as np
import torch


def dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def empty(n, dtype):
    return torch.empty(max(int(n), 1), dtype=dtype, device="cuda")
