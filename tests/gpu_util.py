"""Device-buffer helpers for the gpu tests (torch is used only for memory and sync)."""
import ctypes

import numpy as np


def dev(torch, a, dtype=None):
    a = np.ascontiguousarray(a)
    t = torch.from_numpy(a.astype(dtype) if dtype is not None else a).cuda()
    return t


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def host(torch, t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def rel_err(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))
