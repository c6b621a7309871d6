"""Device-buffer helpers for calling the C ABI from tests (torch as plumbing)."""
import ctypes as C

import numpy as np


def to_dev(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return t


def dptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def empty(shape, dtype):
    import torch
    return torch.empty(shape, dtype=dtype, device="cuda")


def to_host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()
