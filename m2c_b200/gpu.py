"""Python handle on the CUDA library (libm2c_gpu.so) through its C ABI.

The host-side mirror of the reference's interface for this path:
``Solver`` plays the role of SpaceOperator + TimeIntegrator on one
subdomain (SpaceOperator.h:103-140, TimeIntegrator.h:66-73) and exposes
``compute_residual`` / ``compute_dt`` / ``advance`` / ``run`` with the
reference's ghosted array layout. There is no CPU fallback: if the CUDA
library cannot be loaded or no device is present, construction raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libm2c_gpu.so")

_lib = None


class M2CError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"m2cg status {status}: {msg}")
        self.status = status


class Counters(C.Structure):
    _fields_ = [(n, C.c_longlong) for n in (
        "steps", "cells_updated", "riemann_calls", "riemann_iterations", "riemann_errors",
        "clipped_cells", "reinit_calls", "kernel_launches", "unresolved_cells", "riemann_evaluations",
        "failsafe_cells", "riemann_nontrivial", "wall_riemann_calls")]


class BatchTuning(C.Structure):
    _fields_ = [("cells_per_block", C.c_int), ("threads_per_block", C.c_int), ("use_graph", C.c_int)]


def lib():
    """Load libm2c_gpu.so (fails loudly when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"CUDA library not built: {LIB_PATH} (run m2c_b200/build.py)")
    L = C.CDLL(LIB_PATH)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
    L.m2cg_last_error.restype = C.c_char_p
    L.m2cg_create.argtypes = [C.POINTER(abi.Grid), C.POINTER(abi.Scheme), C.POINTER(abi.Material), C.c_int,
                              C.POINTER(abi.LevelSet), C.c_int, C.POINTER(vp)]
    L.m2cg_destroy.argtypes = [vp]
    L.m2cg_upload_state.argtypes = [vp, dp, dp, dp]
    L.m2cg_download_state.argtypes = [vp, dp, dp, dp]
    L.m2cg_compute_dt.argtypes = [vp, dp]
    L.m2cg_compute_residual.argtypes = [vp, dp]
    L.m2cg_advance.argtypes = [vp, C.c_double, C.c_double, C.c_int]
    L.m2cg_run.argtypes = [vp, C.c_int, C.c_double, dp, ip]
    L.m2cg_get_counters.argtypes = [vp, C.POINTER(Counters)]
    L.m2cg_time_steps.argtypes = [vp, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_longlong)]
    L.m2cg_get_stream.argtypes = [vp, C.POINTER(vp)]
    L.m2cg_profile_stages.argtypes = [vp, C.c_int, C.POINTER(C.c_float), ip, C.POINTER(C.c_float)]
    L.m2cg_riemann_batch.argtypes = [C.POINTER(abi.Scheme), C.POINTER(abi.Material), C.c_int, C.c_int, dp, ip, dp,
                                     ip, dp, dp, dp, ip, dp, dp, ip, ip]
    L.m2cg_riemann_batch.restype = C.c_int
    L.m2cg_riemann_batch_pairs.argtypes = [C.POINTER(abi.Scheme), C.POINTER(abi.Material), C.c_int, dp, dp, dp, dp,
                                           dp, ip, dp, dp, ip, ip, ip]
    L.m2cg_riemann_batch_pairs.restype = C.c_int
    L.m2cg_riemann_wall_batch.argtypes = [C.POINTER(abi.Scheme), C.POINTER(abi.Material), C.c_int, C.c_int, dp, ip,
                                          dp, dp, dp, ip, dp, ip, ip]
    L.m2cg_riemann_wall_batch.restype = C.c_int
    L.m2cg_set_wall_faces.argtypes = [vp, C.c_int, ip, dp, dp, dp, dp]
    L.m2cg_batch_create.argtypes = [C.POINTER(abi.Scheme), C.c_int, ip, C.POINTER(abi.Material), dp, dp,
                                    C.POINTER(BatchTuning), C.POINTER(vp)]
    L.m2cg_batch_run.argtypes = [vp, C.c_int]
    L.m2cg_batch_download.argtypes = [vp, dp, ip, dp]
    L.m2cg_batch_get_tuning.argtypes = [vp, C.POINTER(BatchTuning)]
    L.m2cg_batch_get_counters.argtypes = [vp, C.POINTER(Counters)]
    L.m2cg_batch_tube_errors.argtypes = [vp, ip]
    L.m2cg_batch_time_steps.argtypes = [vp, C.c_int, C.POINTER(C.c_float)]
    L.m2cg_batch_destroy.argtypes = [vp]
    L.m2cg_batch_set_mlp.argtypes = [vp, vp]
    L.m2cg_set_mlp.argtypes = [vp, vp]
    L.m2cg_set_probes.argtypes = [vp, C.c_int, dp, C.c_int, C.c_int]
    L.m2cg_sample_probes.argtypes = [vp]
    L.m2cg_read_probes.argtypes = [vp, dp, ip]
    fp = C.POINTER(C.c_float)
    L.m2cg_mlp_create.argtypes = [C.c_ulonglong, C.POINTER(vp)]
    L.m2cg_mlp_destroy.argtypes = [vp]
    L.m2cg_mlp_get_params.argtypes = [vp, fp, fp]
    L.m2cg_mlp_set_params.argtypes = [vp, fp, fp]
    L.m2cg_mlp_loss_grad.argtypes = [vp, fp, fp, C.c_int, fp, fp]
    L.m2cg_mlp_train.argtypes = [vp, fp, fp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_ulonglong, fp]
    L.m2cg_mlp_features_pairs.argtypes = [C.POINTER(abi.Material), C.c_int, dp, dp, dp, fp, dp, ip]
    L.m2cg_mlp_infer.argtypes = [vp, fp, ip, C.c_int, fp]
    L.m2cg_mlp_predict_pairs.argtypes = [vp, C.POINTER(abi.Material), C.c_int, dp, dp, dp, dp]
    L.m2cg_set_device.argtypes = [C.c_int]
    L.m2cg_set_device.restype = C.c_int
    L.m2cg_default_scheme.argtypes = [C.POINTER(abi.Scheme)]
    L.m2cg_default_material.argtypes = [C.POINTER(abi.Material)]
    L.m2cg_default_levelset.argtypes = [C.POINTER(abi.LevelSet)]
    for name in ("m2cg_create", "m2cg_destroy", "m2cg_upload_state", "m2cg_download_state", "m2cg_compute_dt",
                 "m2cg_compute_residual", "m2cg_advance", "m2cg_run", "m2cg_get_counters", "m2cg_time_steps",
                 "m2cg_get_stream", "m2cg_profile_stages", "m2cg_batch_create", "m2cg_batch_run",
                 "m2cg_batch_download", "m2cg_batch_get_tuning", "m2cg_batch_get_counters",
                 "m2cg_batch_tube_errors", "m2cg_batch_time_steps", "m2cg_batch_destroy", "m2cg_batch_set_mlp",
                 "m2cg_set_mlp", "m2cg_set_probes", "m2cg_sample_probes", "m2cg_read_probes",
                 "m2cg_mlp_create", "m2cg_mlp_destroy", "m2cg_mlp_get_params", "m2cg_mlp_set_params",
                 "m2cg_mlp_loss_grad", "m2cg_mlp_train", "m2cg_mlp_features_pairs", "m2cg_mlp_infer",
                 "m2cg_mlp_predict_pairs"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def riemann_batch(s, mats, VL, idl, VR, idr, dirs, warm=None):
    """Exact two-material Riemann problems on the GPU
    (ExactRiemannSolverBase::ComputeRiemannSolution, one problem per thread).
    Returns Vs, id, Vsm, Vsp, iterations, err."""
    n = len(idl)
    VL, VR, dirs = (np.ascontiguousarray(a, np.float64) for a in (VL, VR, dirs))
    idl, idr = np.ascontiguousarray(idl, np.int32), np.ascontiguousarray(idr, np.int32)
    warm = None if warm is None else np.ascontiguousarray(warm, np.float64)
    Vs, Vsm, Vsp = np.zeros((n, 5)), np.zeros((n, 5)), np.zeros((n, 5))
    mid, it, err = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, np.int32)
    arr = (abi.Material * len(mats))(*mats)
    check(lib().m2cg_riemann_batch(C.byref(s), arr, len(mats), n, abi.dptr(VL), abi.iptr(idl), abi.dptr(VR),
                                   abi.iptr(idr), abi.dptr(dirs), abi.dptr(warm), abi.dptr(Vs), abi.iptr(mid),
                                   abi.dptr(Vsm), abi.dptr(Vsp), abi.iptr(it), abi.iptr(err)))
    return Vs, mid, Vsm, Vsp, it, err


def riemann_wall_batch(s, mats, Vm, idm, uwall, dirs):
    """One-sided (wall) Riemann problems on the GPU
    (ExactRiemannSolverBase::ComputeOneSidedRiemannSolution): fluid state
    Vm[q] of material idm[q] against a wall moving with velocity uwall[q],
    dirs[q] the unit normal from the fluid to the wall. Returns Vs (zero
    where id = -1), id, Vsm, iterations, err."""
    n = len(idm)
    Vm, uwall, dirs = (np.ascontiguousarray(a, np.float64) for a in (Vm, uwall, dirs))
    idm = np.ascontiguousarray(idm, np.int32)
    Vs, Vsm = np.zeros((n, 5)), np.zeros((n, 5))
    mid, it, err = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, np.int32)
    arr = (abi.Material * len(mats))(*mats)
    check(lib().m2cg_riemann_wall_batch(C.byref(s), arr, len(mats), n, abi.dptr(Vm), abi.iptr(idm),
                                        abi.dptr(uwall), abi.dptr(dirs), abi.dptr(Vs), abi.iptr(mid),
                                        abi.dptr(Vsm), abi.iptr(it), abi.iptr(err)))
    return Vs, mid, Vsm, it, err


def riemann_batch_pairs(s, mats, VL, VR, dirs, warm=None):
    """Exact Riemann problems where problem q has material mats[2q] on the
    left and mats[2q+1] on the right. Returns Vs, id (0 left, 1 right), Vsm,
    Vsp, iterations, evaluations, err."""
    n = len(VL)
    VL, VR, dirs = (np.ascontiguousarray(a, np.float64) for a in (VL, VR, dirs))
    warm = None if warm is None else np.ascontiguousarray(warm, np.float64)
    Vs, Vsm, Vsp = np.zeros((n, 5)), np.zeros((n, 5)), np.zeros((n, 5))
    mid, it, ev, err = (np.zeros(n, np.int32) for _ in range(4))
    arr = abi.material_array(mats)
    check(lib().m2cg_riemann_batch_pairs(C.byref(s), arr, n, abi.dptr(VL), abi.dptr(VR), abi.dptr(dirs),
                                         abi.dptr(warm), abi.dptr(Vs), abi.iptr(mid), abi.dptr(Vsm), abi.dptr(Vsp),
                                         abi.iptr(it), abi.iptr(ev), abi.iptr(err)))
    return Vs, mid, Vsm, Vsp, it, ev, err


def tube_rejects(s):
    """reject() for cases.tubes: tubes whose initial interface Riemann problem
    the solver reports as failed or path-overflowing are redrawn."""
    def reject(mats, VL, VR):
        dirs = np.zeros((len(VL), 3))
        dirs[:, 0] = 1.0
        err = riemann_batch_pairs(s, mats, VL, VR, dirs)[6]
        return err != 0
    return reject


def set_device(device):
    check(lib().m2cg_set_device(device))


def check(st):
    if st != 0:
        raise M2CError(st, lib().m2cg_last_error().decode())


class Solver:
    """One structured subdomain advanced on the GPU (FP64 or mixed precision)."""

    def __init__(self, g, s, mats, ls=None):
        L = lib()
        self.g, self.s = g, s
        self.nls = 0 if ls is None else 1
        arr = (abi.Material * len(mats))(*mats)
        h = C.c_void_p()
        check(L.m2cg_create(C.byref(g), C.byref(s), arr, len(mats), C.byref(ls) if ls is not None else None,
                            self.nls, C.byref(h)))
        self.h = h
        self.t = 0.0
        self.step = 0

    def upload(self, V, ID=None, phi=None):
        V = np.ascontiguousarray(V, np.float64)
        ID = None if ID is None else np.ascontiguousarray(ID, np.float64)
        phi = None if phi is None else np.ascontiguousarray(phi, np.float64)
        check(lib().m2cg_upload_state(self.h, abi.dptr(V), abi.dptr(ID), abi.dptr(phi)))

    def download(self, out_V=None, out_ID=None, out_phi=None, with_id=True):
        """Host copies of V (and of the material IDs unless with_id is False,
        and of phi when there is a level set), ghosted layout."""
        V = out_V if out_V is not None else np.empty(abi.ghosted_shape(self.g, 5))
        ID = out_ID if out_ID is not None else (np.empty(abi.ghosted_shape(self.g)) if with_id else None)
        phi = out_phi if out_phi is not None else (np.empty(abi.ghosted_shape(self.g)) if self.nls else None)
        check(lib().m2cg_download_state(self.h, abi.dptr(V), abi.dptr(ID), abi.dptr(phi)))
        return V, ID, phi

    def compute_dt(self):
        dt = C.c_double()
        check(lib().m2cg_compute_dt(self.h, C.byref(dt)))
        return dt.value

    def residual(self):
        R = np.empty(abi.ghosted_shape(self.g, 5))
        check(lib().m2cg_compute_residual(self.h, abi.dptr(R)))
        return R

    def advance(self, dt):
        """One step of size dt (the reference passes the updated time t+dt)."""
        self.t += dt
        self.step += 1
        check(lib().m2cg_advance(self.h, self.t, dt, self.step))

    def run(self, nsteps, t_max=float("inf")):
        t = C.c_double(self.t)
        n = C.c_int()
        check(lib().m2cg_run(self.h, nsteps, t_max, C.byref(t), C.byref(n)))
        self.t = t.value
        self.step += n.value
        return n.value, self.t

    def time_steps(self, nsteps):
        ms = C.c_float()
        launches = C.c_longlong()
        check(lib().m2cg_time_steps(self.h, nsteps, C.byref(ms), C.byref(launches)))
        return ms.value, launches.value

    def profile_stages(self, nsteps):
        ms, n, step = C.c_float(), C.c_int(), C.c_float()
        check(lib().m2cg_profile_stages(self.h, nsteps, C.byref(ms), C.byref(n), C.byref(step)))
        return ms.value, n.value, step.value

    def counters(self):
        c = Counters()
        check(lib().m2cg_get_counters(self.h, C.byref(c)))
        return {n: getattr(c, n) for n, _ in Counters._fields_}

    def update_states_after_motion(self, IDn, use_stored_riemann_solutions=False):
        """UpdateStateVariablesAfterInterfaceMotion on the resident state
        against the step-start IDs IDn (ghosted layout); returns the number of
        cells handed to FixUnresolvedNodes."""
        IDn = np.ascontiguousarray(IDn, dtype=np.float64)
        n = C.c_int()
        check(lib().m2cg_update_states_after_interface_motion(self.h, abi.dptr(IDn),
                                                              int(bool(use_stored_riemann_solutions)),
                                                              C.byref(n)))
        return n.value

    def set_probes(self, xyz, every=1, capacity=1024):
        """Sample the primitive state at the points xyz [n][3] on the device
        after every `every`-th step (ProbeOutput's interpolation)."""
        self._probe_xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        self._probe_cap = capacity
        check(lib().m2cg_set_probes(self.h, len(self._probe_xyz), abi.dptr(self._probe_xyz), every, capacity))

    def sample_probes(self):
        check(lib().m2cg_sample_probes(self.h))

    def read_probes(self):
        """Records since the last read, [nrec][2 + 5n]: t, step, then rho, u,
        v, w, p of each probe."""
        n = len(self._probe_xyz)
        out = np.empty((self._probe_cap, 2 + 5 * n))
        cnt = C.c_int()
        check(lib().m2cg_read_probes(self.h, abi.dptr(out), C.byref(cnt)))
        return out[:cnt.value]

    def set_wall_faces(self, faces, nwall_fwd=None, uwall_fwd=None, nwall_bwd=None, uwall_bwd=None):
        """Faces cut by an embedded surface for the following stages
        (m2cg_set_wall_faces): faces [n][4] = (axis, i, j, k), the face
        between cell (i, j, k) and its low neighbour; the surface's unit
        normal and velocity seen from the low cell (fwd) and from the high
        cell (bwd), [n][3] each (velocities default to zero, normals to the
        face normal). An empty list removes the walls."""
        faces = np.ascontiguousarray(np.asarray(faces, np.int32).reshape(-1, 4))
        n = len(faces)
        def arr(a, default):
            return np.ascontiguousarray(default if a is None else np.asarray(a, np.float64).reshape(n, 3))
        en = np.zeros((n, 3))
        en[np.arange(n), faces[:, 0]] = 1.0
        nf, uf = arr(nwall_fwd, en), arr(uwall_fwd, np.zeros((n, 3)))
        nb, ub = arr(nwall_bwd, en), arr(uwall_bwd, np.zeros((n, 3)))
        check(lib().m2cg_set_wall_faces(self.h, n, abi.iptr(faces), abi.dptr(nf), abi.dptr(uf), abi.dptr(nb),
                                        abi.dptr(ub)))

    def set_mlp(self, mlp):
        """Start every interface Riemann solve of the steps from the
        network's proposal (None detaches; two materials only)."""
        check(lib().m2cg_set_mlp(self.h, mlp.h if mlp is not None else None))
        self._mlp = mlp  # keep it alive while attached

    def stream(self):
        p = C.c_void_p()
        check(lib().m2cg_get_stream(self.h, C.byref(p)))
        return p.value

    def close(self):
        if getattr(self, "h", None):
            lib().m2cg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Batched 1D two-material shock tubes advanced together on the GPU
    (m2cg_batch_*): tube t has len[t] cells on [0, 1], materials mats[2t]
    (left, phi > 0) and mats[2t+1] (right), left/right states VL[t], VR[t],
    INLET/OUTLET ghosts holding those states. Each tube is what one reference
    run of the same setup computes (TimeIntegratorRK2/RK3, MultiPhaseOperator)."""

    def __init__(self, s, lens, mats, VL, VR, cells_per_block=0, threads_per_block=0, use_graph=-1):
        L = lib()
        self.lens = np.ascontiguousarray(lens, np.int32)
        self.ntubes = len(self.lens)
        self.ncell = int(self.lens.sum())
        VL = np.ascontiguousarray(VL, np.float64)
        VR = np.ascontiguousarray(VR, np.float64)
        arr = (abi.Material * len(mats))(*mats)
        tun = BatchTuning(cells_per_block, threads_per_block, use_graph)
        h = C.c_void_p()
        check(L.m2cg_batch_create(C.byref(s), self.ntubes, abi.iptr(self.lens), arr, abi.dptr(VL), abi.dptr(VR),
                                  C.byref(tun), C.byref(h)))
        self.h = h

    def run(self, nsteps):
        check(lib().m2cg_batch_run(self.h, nsteps))

    def time_steps(self, nsteps, check_errors=True):
        """Device time (ms) of nsteps steps. With check_errors=False a tube
        error does not raise: the time is returned and tube_errors() tells
        which tubes failed."""
        ms = C.c_float(-1.0)
        st = lib().m2cg_batch_time_steps(self.h, nsteps, C.byref(ms))
        if st and (check_errors or ms.value < 0):
            check(st)
        return ms.value

    def download(self, check_errors=True):
        """Returns (list of per-tube V arrays [len, 5], list of ID arrays, t per
        tube). With check_errors=False a tube error does not raise (the
        failed tubes' states are not defined; tube_errors() tells which)."""
        V = np.empty((self.ncell, 5))
        ID = np.empty(self.ncell, np.int32)
        t = np.empty(self.ntubes)
        st = lib().m2cg_batch_download(self.h, abi.dptr(V), abi.iptr(ID), abi.dptr(t))
        if st and (check_errors or st == 2):  # 2: CUDA error (nothing copied)
            check(st)
        cuts = np.cumsum(self.lens)[:-1]
        return np.split(V, cuts), np.split(ID, cuts), t

    def tuning(self):
        tun = BatchTuning()
        check(lib().m2cg_batch_get_tuning(self.h, C.byref(tun)))
        return {n: getattr(tun, n) for n, _ in BatchTuning._fields_}

    def counters(self):
        c = Counters()
        check(lib().m2cg_batch_get_counters(self.h, C.byref(c)))
        return {n: getattr(c, n) for n, _ in Counters._fields_}

    def set_mlp(self, mlp):
        """Start every interface Riemann solve from the network's proposal
        (None detaches)."""
        check(lib().m2cg_batch_set_mlp(self.h, mlp.h if mlp is not None else None))
        self._mlp = mlp  # keep it alive while attached

    def tube_errors(self):
        codes = np.zeros(self.ntubes, np.int32)
        check(lib().m2cg_batch_tube_errors(self.h, abi.iptr(codes)))
        return codes

    def close(self):
        if getattr(self, "h", None):
            lib().m2cg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _fptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


class Mlp:
    """The learned warm start of the interface Riemann solve: a
    16 -> 64 -> 64 -> 64 -> 1 tanh network proposing log(p*/pac) (pac the
    acoustic estimate) from
    dimensionless problem features (m2cg_mlp_*). Trained on the GPU by the
    library's own FP32 forward/backward kernels; inference is BF16 on tensor
    cores."""
    NPARAM = 9473
    NIN = 16
    NNORM = 34

    def __init__(self, seed=0):
        h = C.c_void_p()
        check(lib().m2cg_mlp_create(seed, C.byref(h)))
        self.h = h

    def params(self):
        p = np.empty(self.NPARAM, np.float32)
        n = np.empty(self.NNORM, np.float32)
        check(lib().m2cg_mlp_get_params(self.h, _fptr(p), _fptr(n)))
        return p, n

    def set_params(self, params=None, norm=None):
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        n = None if norm is None else np.ascontiguousarray(norm, np.float32)
        check(lib().m2cg_mlp_set_params(self.h, _fptr(p), _fptr(n)))

    def loss_grad(self, Xn, yn):
        Xn = np.ascontiguousarray(Xn, np.float32)
        yn = np.ascontiguousarray(yn, np.float32)
        loss = np.zeros(1, np.float32)
        g = np.zeros(self.NPARAM, np.float32)
        check(lib().m2cg_mlp_loss_grad(self.h, _fptr(Xn), _fptr(yn), len(yn), _fptr(loss), _fptr(g)))
        return float(loss[0]), g

    def train(self, X, y, steps=3000, batch=8192, lr=2e-3, seed=0):
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = np.zeros(1, np.float32)
        check(lib().m2cg_mlp_train(self.h, _fptr(X), _fptr(y), len(y), steps, batch, lr, seed, _fptr(loss)))
        return float(loss[0])

    def infer(self, X, valid=None):
        X = np.ascontiguousarray(X, np.float32)
        valid = np.ones(len(X), np.int32) if valid is None else np.ascontiguousarray(valid, np.int32)
        y = np.zeros(len(X), np.float32)
        check(lib().m2cg_mlp_infer(self.h, _fptr(X), abi.iptr(valid), len(X), _fptr(y)))
        return y

    def predict_pairs(self, mats, VL, VR, dirs):
        VL, VR, dirs = (np.ascontiguousarray(a, np.float64) for a in (VL, VR, dirs))
        p = np.empty(len(VL))
        check(lib().m2cg_mlp_predict_pairs(self.h, abi.material_array(mats), len(VL), abi.dptr(VL), abi.dptr(VR),
                                           abi.dptr(dirs), abi.dptr(p)))
        return p

    def close(self):
        if getattr(self, "h", None):
            lib().m2cg_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mlp_features_pairs(mats, VL, VR, dirs):
    """Network input features of per-pair problems: X [n, 16] (float32),
    scale [n, 2] = (base B, shift S) of the target log((p* + S) / B),
    valid [n]."""
    VL, VR, dirs = (np.ascontiguousarray(a, np.float64) for a in (VL, VR, dirs))
    n = len(VL)
    X = np.zeros((n, 16), np.float32)
    P = np.zeros((n, 2))
    valid = np.zeros(n, np.int32)
    check(lib().m2cg_mlp_features_pairs(abi.material_array(mats), n, abi.dptr(VL), abi.dptr(VR), abi.dptr(dirs),
                                        _fptr(X), abi.dptr(P), abi.iptr(valid)))
    return X, P, valid
