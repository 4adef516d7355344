"""Helpers shared by the GPU parity tests."""
import numpy as np


def col_relerr(got: np.ndarray, ref: np.ndarray) -> np.ndarray:
    """Per column: max |got - ref| / max |ref| (max-norm relative error)."""
    got = np.asarray(got)
    ref = np.asarray(ref)
    den = np.abs(ref).max(axis=0)
    den = np.where(den == 0, 1.0, den)
    return np.abs(got - ref).max(axis=0) / den


def to_dev_fortran(a):
    """numpy (n, c) F-order -> torch CUDA tensor (c, n) whose memory is the same column-major layout."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda()


def from_dev_fortran(t):
    return t.cpu().numpy().T
