"""Comparison helpers for parity tests."""
import ctypes as C

import numpy as np

from m2c_b200 import abi


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


def host_riemann(lib, s, mats, VL, idl, VR, idr, dirs, libm=True):
    """Solve with the host build of the library's exact Riemann solver
    (tests/host/riemann_host.cpp): libm=True takes pow from the C library as
    the reference does, libm=False the correctly rounded roots the GPU uses.
    Returns (Vs, id, Vsm, Vsp, err, retried, misrounded): misrounded[q]
    counts problem q's step-control pow calls where the C library's result is
    not the correctly rounded one."""
    n = len(VL)
    table = (abi.Material * len(mats))(*mats)
    Vs, Vsm, Vsp = np.zeros((n, 5)), np.zeros((n, 5)), np.zeros((n, 5))
    mid, err, retried = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, np.int32)
    mis = np.zeros(n, np.int32)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    args = [np.ascontiguousarray(a) for a in (dirs, VL, np.asarray(idl, np.int32), VR, np.asarray(idr, np.int32))]
    lib.host_riemann(C.byref(s), table, len(mats), n, *[p(a) for a in args], p(Vs), p(mid), p(Vsm), p(Vsp),
                     p(err), p(retried), int(bool(libm)), p(mis))
    return Vs, mid, Vsm, Vsp, err, retried, mis


def host_riemann_wall(lib, s, mats, Vm, idm, uwall, dirs, libm=True):
    """One-sided (wall) problems with the host build of the library's solver
    (RiemannSolver::solve_wall); pow chosen as in host_riemann. Returns (Vs,
    id, Vsm, err, misrounded)."""
    n = len(Vm)
    table = (abi.Material * len(mats))(*mats)
    Vs, Vsm = np.zeros((n, 5)), np.zeros((n, 5))
    mid, err, mis = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, np.int32)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    args = [np.ascontiguousarray(a) for a in (dirs, np.asarray(Vm, np.float64), np.asarray(idm, np.int32),
                                              np.asarray(uwall, np.float64))]
    lib.host_riemann_wall(C.byref(s), table, len(mats), n, *[p(a) for a in args], p(Vs), p(mid), p(Vsm), p(err),
                          int(bool(libm)), p(mis))
    return Vs, mid, Vsm, err, mis
