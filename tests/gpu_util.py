"""Helpers of the GPU tests: move reference-layout numpy arrays to and from the
device.  A Fortran-ordered numpy array [x, z, y] has the memory of a
C-contiguous tensor [y, z, x]."""
import numpy as np


def to_dev(a, device="cuda:0"):
    import torch
    a = np.asfortranarray(a, dtype=np.float64)
    return torch.from_numpy(np.ascontiguousarray(a.T)).to(device)


def from_dev(t):
    return np.asfortranarray(t.detach().cpu().numpy().T)


def empty_like_dev(shape_xzy, device="cuda:0", fill=np.nan):
    import torch
    return torch.full(tuple(reversed(shape_xzy)), fill, dtype=torch.float64, device=device)
