"""m2cg_riemann_batch_noalloc, the Riemann batch entry point for callers that
cannot allocate device memory (an application whose memory pool owns the
whole GPU, a runtime that forbids allocation where it calls in): inputs and
outputs are device buffers the caller already holds, and the solver's scratch
is a fixed device array inside the library.

Checked against the allocating m2cg_riemann_batch on the same problems, on
two calls in a row (the second smaller, so it runs over scratch the first
left behind; one pair uses the largest allowed size, which fills the last
scratch slot), at the tolerance of the other FP64 tests (1e-12 relative;
integer outputs exact), with and without the optional warm-start and
iteration arrays. The device's free memory is the same before and after a
call (after the first call on the device, which sets up the scratch).
Also: sizes above the maximum are refused with a message, and an
out-of-range material id is flagged per problem. The limits are read from
include/m2c_gpu.h, so the test follows the header.

Named to be collected last: device buffers here come from torch.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

from m2c_b200 import abi, cases

pytestmark = pytest.mark.gpu


def _header_define(name):
    h = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "m2c_gpu.h")
    m = re.search(r"#define\s+" + name + r"\s+(\d+)", open(h).read())
    assert m, name
    return int(m.group(1))


MAX_PROBLEMS = _header_define("M2CG_NOALLOC_MAX_PROBLEMS")
ERR_MATERIAL_ID = _header_define("M2CG_RIEMANN_ERR_MATERIAL_ID")


def _bind(L):
    f = L.m2cg_riemann_batch_noalloc
    f.argtypes = [C.POINTER(abi.Scheme), C.POINTER(abi.Material), C.c_int, C.c_int] + [C.c_void_p] * 13
    f.restype = C.c_int
    return f


def _noalloc(gpu, s, mats, VL, idl, VR, idr, dirs, warm=None, with_iters=True, free_mem=None):
    """Copies the problems to torch device tensors, calls the entry point on
    torch's current stream and returns host copies of its outputs (iters is
    None when with_iters is False). free_mem, a list, receives the device's
    free bytes just before and just after the call."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    n = len(idl)
    t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    dVL, dVR, ddir = t(VL, torch.float64), t(VR, torch.float64), t(dirs, torch.float64)
    didl, didr = t(idl, torch.int32), t(idr, torch.int32)
    dwarm = None if warm is None else t(warm, torch.float64)
    Vs, Vsm, Vsp = (torch.full((n, 5), -1.0, dtype=torch.float64, device=dev) for _ in range(3))
    mid, it, err = (torch.full((n,), -7, dtype=torch.int32, device=dev) for _ in range(3))
    arr = (abi.Material * len(mats))(*mats)
    stream = torch.cuda.current_stream(dev)
    p = lambda x: None if x is None else C.c_void_p(x.data_ptr())
    torch.cuda.synchronize(dev)
    if free_mem is not None:
        free_mem.append(torch.cuda.mem_get_info(dev)[0])
    st = _bind(gpu.lib())(C.byref(s), arr, len(mats), n, p(dVL), p(didl), p(dVR), p(didr), p(ddir), p(dwarm),
                          p(Vs), p(mid), p(Vsm), p(Vsp), p(it) if with_iters else None, p(err),
                          C.c_void_p(stream.cuda_stream))
    gpu.check(st)
    stream.synchronize()
    if free_mem is not None:
        free_mem.append(torch.cuda.mem_get_info(dev)[0])
    out = [x.cpu().numpy() for x in (Vs, mid, Vsm, Vsp, it, err)]
    if not with_iters:
        out[4] = None
    return tuple(out)


def _rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


@pytest.mark.parametrize("sizes", [(1000, 700), (MAX_PROBLEMS, 700)])
def test_noalloc_matches_allocating_entry_point(gpu, sizes):
    s = abi.scheme()
    for call, n in enumerate(sizes):
        mats, VL, idl, VR, idr, dirs = cases.riemann_problems(n, seed=40 + call)
        want = gpu.riemann_batch(s, mats, VL, idl, VR, idr, dirs)
        got = _noalloc(gpu, s, mats, VL, idl, VR, idr, dirs)
        Vs, mid, Vsm, Vsp, it, err = got
        wVs, wmid, wVsm, wVsp, wit, werr = want
        np.testing.assert_array_equal(err, werr)
        np.testing.assert_array_equal(mid, wmid)
        np.testing.assert_array_equal(it, wit)
        for a, b in ((Vs, wVs), (Vsm, wVsm), (Vsp, wVsp)):
            assert _rel(a, b).max() <= 1e-12, (call, _rel(a, b).max())
        assert (err == 0).mean() >= 0.95


def test_noalloc_with_warm_start_and_no_iteration_array(gpu):
    """Optional arguments: a warm-start array (some entries NaN, which means
    no proposal) and iters = NULL, against the allocating entry point with
    the same warm array."""
    s = abi.scheme()
    n = 600
    mats, VL, idl, VR, idr, dirs = cases.riemann_problems(n, seed=61)
    cold = gpu.riemann_batch(s, mats, VL, idl, VR, idr, dirs)
    warm = np.where(cold[5] == 0, cold[2][:, 4] * 1.05, np.nan)
    warm[::7] = np.nan
    want = gpu.riemann_batch(s, mats, VL, idl, VR, idr, dirs, warm=warm)
    Vs, mid, Vsm, Vsp, it, err = _noalloc(gpu, s, mats, VL, idl, VR, idr, dirs, warm=warm, with_iters=False)
    assert it is None
    wVs, wmid, wVsm, wVsp, wit, werr = want
    np.testing.assert_array_equal(err, werr)
    np.testing.assert_array_equal(mid, wmid)
    for a, b in ((Vs, wVs), (Vsm, wVsm), (Vsp, wVsp)):
        assert _rel(a, b).max() <= 1e-12, _rel(a, b).max()


def test_noalloc_allocates_nothing(gpu):
    """After the first call on the device (which sets up the scratch), a
    call leaves the device's free memory unchanged."""
    s = abi.scheme()
    mats, VL, idl, VR, idr, dirs = cases.riemann_problems(MAX_PROBLEMS, seed=70)
    _noalloc(gpu, s, mats, VL, idl, VR, idr, dirs)  # first call: set-up and the kernel's first launch
    free = []
    _noalloc(gpu, s, mats, VL, idl, VR, idr, dirs, free_mem=free)
    assert free[0] == free[1], free


def test_noalloc_limits(gpu):
    import torch
    s = abi.scheme()
    mats, VL, idl, VR, idr, dirs = cases.riemann_problems(1, seed=9)
    dev = torch.device("cuda", torch.cuda.current_device())
    big = torch.zeros((MAX_PROBLEMS + 1) * 5, dtype=torch.float64, device=dev)
    ibig = torch.zeros(MAX_PROBLEMS + 1, dtype=torch.int32, device=dev)
    arr = (abi.Material * len(mats))(*mats)
    vp, ip = C.c_void_p(big.data_ptr()), C.c_void_p(ibig.data_ptr())
    st = _bind(gpu.lib())(C.byref(s), arr, len(mats), MAX_PROBLEMS + 1, vp, ip, vp, ip, vp, None, vp, ip, vp, vp,
                          ip, ip, None)
    assert st == abi.ERR_ARG
    assert b"maximum" in gpu.lib().m2cg_last_error()
    # a material id outside [0, nmat) is flagged for that problem only
    VL2, VR2 = np.repeat(VL, 2, 0), np.repeat(VR, 2, 0)
    Vs, mid, Vsm, Vsp, it, err = _noalloc(gpu, s, mats, VL2, [0, 0], VR2, [1, 5], np.repeat(dirs, 2, 0))
    assert err[1] == ERR_MATERIAL_ID and mid[1] == -1 and np.isnan(Vs[1]).all()
    assert err[0] == 0 and mid[0] in (0, 1)
