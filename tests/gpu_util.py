"""Helpers of the GPU tests: numpy <-> CUDA tensors (torch is only the
device-memory plumbing; every kernel call goes through libcudapic's C ABI)."""
import numpy as np


def dev(a):
    import torch
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32).copy()).cuda()
    return torch.from_numpy(a.copy()).cuda()


def host(t):
    import torch
    torch.cuda.synchronize()
    a = t.detach().cpu().numpy()
    return a.view(np.uint32) if a.dtype == np.int32 else a


def counter(v):
    return dev(np.array([v], np.uint32))


def zeros(n, dtype=np.float32):
    return dev(np.zeros(n, dtype))


def rows(*cols):
    """Rows of float32/uint32 columns as one uint32 matrix (bit patterns)."""
    return np.stack([np.ascontiguousarray(c).view(np.uint32) for c in cols], axis=1)


def sorted_rows(*cols):
    r = rows(*cols)
    if r.shape[0] == 0:
        return r
    order = np.lexsort(r.T[::-1])
    return r[order]
