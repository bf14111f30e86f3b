"""Comparison helpers for parity tests."""
import numpy as np


def rel_err(a, b, axis_last=True):
    """Max abs difference per variable divided by the variable's max magnitude."""
    a = np.asarray(a)
    b = np.asarray(b)
    if axis_last and a.ndim >= 1 and a.shape[-1] == 5:
        d = np.abs(a - b).reshape(-1, 5).max(axis=0)
        s = np.maximum(np.abs(b).reshape(-1, 5).max(axis=0), 1e-300)
        return (d / s).max()
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def l1_rel(a, b):
    a = np.asarray(a).reshape(-1, 5)
    b = np.asarray(b).reshape(-1, 5)
    return (np.abs(a - b).sum(axis=0) / np.maximum(np.abs(b).sum(axis=0), 1e-300)).max()


def inner(A):
    return A[1:-1, 1:-1, 1:-1]


def face_ghosts_mask(shape):
    """Boolean mask of interior + face-ghost nodes of a ghosted box."""
    nz, ny, nx = shape[:3]
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    out = ((k == 0) | (k == nz - 1)).astype(int) + ((j == 0) | (j == ny - 1)).astype(int) + \
          ((i == 0) | (i == nx - 1)).astype(int)
    return out <= 1
