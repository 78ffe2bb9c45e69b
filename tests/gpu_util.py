"""Helpers for the GPU tests: host <-> device copies and the reference kernels' checker library."""
import ctypes

import numpy as np


def dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def bits(x):
    return np.ascontiguousarray(x).view(np.uint64)


def ref_kernels(oracle):
    """MGXBench's own kernels compiled from its sources (oracle/_ref), or None."""
    return oracle.ref_lib()


def vp(t):
    return ctypes.c_void_p(t.data_ptr())
