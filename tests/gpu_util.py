"""Device-memory helpers for the GPU tests (torch is only the allocator)."""
import ctypes as C

import numpy as np


def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("no CUDA device")
    return torch


def dev(a):
    torch = torch_cuda()
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def ptr(t):
    return C.c_void_p(t.data_ptr())


class DevCSR:
    def __init__(self, ia, ja, val):
        self.n = len(ia) - 1
        self.nnz = int(ia[-1])
        self.ia, self.ja, self.val = dev(np.int32(ia)), dev(np.int32(ja)), dev(np.float64(val))

    def args(self):
        return (self.n, self.nnz, ptr(self.ia), ptr(self.ja), ptr(self.val))
