"""Python handle on the CPU oracles (TEST INFRASTRUCTURE ONLY).

  * ``RefCase``/``RefPoint`` over oracle/_ref/libm2c_ref.so: the unmodified
    reference M2C sources compiled in place with single-rank shims
    (oracle/Makefile, target ``ref``), driven like Main.cpp.
  * ``RefCaseCR``/``RefPointCR`` over oracle/_ref/libm2c_ref_crpow.so
    (target ``refcr``): the same reference build with pow(x, 0.25) and
    pow(x, 0.2) correctly rounded (oracle/ref_shim/crpow_interpose.cpp), as
    the GPU's Riemann solver computes them; every other operation is the
    unmodified reference's.
  * ``DropinCase`` over oracle/_ref/libm2c_dropin.so (target ``dropin``):
    the same reference driver with its RK integrator replaced by the GPU
    drop-in m2c_b200/adapter/TimeIntegratorGPU.h. This one runs the product
    (the GPU library) inside the reference's own loop; tests compare it with
    RefCase to show the drop-in boundary works.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this module, and only as the checker.
"""
import ctypes as C
import os

import numpy as np

from m2c_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libm2c_ref.so")
DROPIN_SO = os.path.join(HERE, "_ref", "libm2c_dropin.so")
CR_SO = os.path.join(HERE, "_ref", "libm2c_ref_crpow.so")

_libs = {}


def _load(path, prefix):
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    lib = C.CDLL(path)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
    f = lambda n: getattr(lib, prefix + n)
    f("create").restype = vp
    f("create").argtypes = [C.POINTER(abi.Grid), C.POINTER(abi.Scheme), C.POINTER(abi.Material), C.c_int,
                            C.POINTER(abi.LevelSet), C.c_int]
    f("set_state").argtypes = [vp, dp, dp, dp]
    f("get_state").argtypes = [vp, dp, dp, dp]
    f("update_states_after_motion").restype = C.c_int
    f("update_states_after_motion").argtypes = [vp, dp]
    f("compute_dt").restype = C.c_double
    f("compute_dt").argtypes = [vp]
    f("compute_residual").argtypes = [vp, dp]
    f("compute_residual_walls").argtypes = [vp, C.c_int, ip, dp, dp, dp, dp, dp]
    f("run_walls").argtypes = [vp, C.c_int, ip, dp, dp, dp, dp, C.c_int, dp]
    f("run_walls").restype = C.c_int
    f("advance").argtypes = [vp, C.c_double]
    f("run").restype = C.c_int
    f("run").argtypes = [vp, C.c_int, C.c_double, dp]
    f("seconds").restype = C.c_double
    f("seconds").argtypes = [vp]
    f("destroy").argtypes = [vp]
    f("point_create").restype = vp
    f("point_create").argtypes = [C.POINTER(abi.Scheme), C.POINTER(abi.Material), C.c_int]
    f("point_flux").argtypes = [vp, C.c_int, C.c_int, dp, dp, ip, dp]
    f("point_c2p").argtypes = [vp, C.c_int, dp, ip, dp]
    f("point_p2c").argtypes = [vp, C.c_int, dp, ip, dp]
    f("point_riemann").restype = C.c_int
    f("point_riemann").argtypes = [vp, C.c_int, dp, dp, ip, dp, ip, dp, ip, dp, dp, ip]
    f("point_riemann_wall").argtypes = [vp, C.c_int, dp, dp, ip, dp, dp, ip, dp, ip]
    f("point_destroy").argtypes = [vp]
    _libs[path] = lib
    return lib


def available(which="ref"):
    return os.path.exists({"ref": REF_SO, "crpow": CR_SO, "dropin": DROPIN_SO}[which])


class _Case:
    def __init__(self, lib, prefix, g, s, mats, ls=None):
        self.lib, self.p = lib, prefix
        self.g = g
        mats_arr = (abi.Material * len(mats))(*mats)
        nls = 0 if ls is None else 1
        lsp = C.byref(ls) if ls is not None else None
        self.h = getattr(lib, prefix + "create")(C.byref(g), C.byref(s), mats_arr, len(mats), lsp, nls)
        self.nls = nls

    def _f(self, n):
        return getattr(self.lib, self.p + n)

    def set_state(self, V, ID=None, phi=None):
        V = np.ascontiguousarray(V, dtype=np.float64)
        ID = None if ID is None else np.ascontiguousarray(ID, dtype=np.float64)
        phi = None if phi is None else np.ascontiguousarray(phi, dtype=np.float64)
        self._f("set_state")(self.h, abi.dptr(V), abi.dptr(ID), abi.dptr(phi))

    def get_state(self):
        V = np.zeros(abi.ghosted_shape(self.g, 5))
        ID = np.zeros(abi.ghosted_shape(self.g))
        phi = np.zeros(abi.ghosted_shape(self.g)) if self.nls else None
        self._f("get_state")(self.h, abi.dptr(V), abi.dptr(ID), abi.dptr(phi))
        return V, ID, phi

    def compute_dt(self):
        return self._f("compute_dt")(self.h)

    def update_states_after_motion(self, IDn):
        """UpdateStateVariablesAfterInterfaceMotion against the step-start IDs
        IDn (ghosted layout), no stored Riemann solutions; returns the number
        of cells still unresolved."""
        IDn = np.ascontiguousarray(IDn, dtype=np.float64)
        return self._f("update_states_after_motion")(self.h, abi.dptr(IDn))

    def residual(self):
        R = np.zeros(abi.ghosted_shape(self.g, 5))
        self._f("compute_residual")(self.h, abi.dptr(R))
        return R

    def residual_walls(self, faces, nwall_fwd, uwall_fwd, nwall_bwd, uwall_bwd):
        """SpaceOperator::ComputeResidual with an embedded surface cutting the
        listed faces (the arguments of Solver.set_wall_faces, all given)."""
        faces = np.ascontiguousarray(np.asarray(faces, np.int32).reshape(-1, 4))
        arrs = [np.ascontiguousarray(np.asarray(a, np.float64).reshape(-1, 3))
                for a in (nwall_fwd, uwall_fwd, nwall_bwd, uwall_bwd)]
        R = np.zeros(abi.ghosted_shape(self.g, 5))
        self._f("compute_residual_walls")(self.h, len(faces), abi.iptr(faces), *[abi.dptr(a) for a in arrs],
                                          abi.dptr(R))
        return R

    def run_walls(self, faces, nwall_fwd, uwall_fwd, nwall_bwd, uwall_bwd, nsteps):
        """nsteps CFL steps of one material (RK2 / RK3 as the reference's
        integrator takes them) with an embedded surface cutting the listed
        faces; returns (steps, t)."""
        faces = np.ascontiguousarray(np.asarray(faces, np.int32).reshape(-1, 4))
        arrs = [np.ascontiguousarray(np.asarray(a, np.float64).reshape(-1, 3))
                for a in (nwall_fwd, uwall_fwd, nwall_bwd, uwall_bwd)]
        t = C.c_double(0.0)
        n = self._f("run_walls")(self.h, len(faces), abi.iptr(faces), *[abi.dptr(a) for a in arrs], nsteps,
                                 C.byref(t))
        if n < 0:
            raise ValueError("run_walls: one material without level sets only")
        return n, t.value

    def advance(self, dt):
        self._f("advance")(self.h, dt)

    def run(self, nsteps, t_max=float("inf")):
        t = C.c_double(0.0)
        n = self._f("run")(self.h, nsteps, t_max, C.byref(t))
        return n, t.value

    def seconds(self):
        return self._f("seconds")(self.h)

    def close(self):
        if self.h:
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Point:
    def __init__(self, lib, prefix, s, mats):
        self.lib, self.p = lib, prefix
        mats_arr = (abi.Material * len(mats))(*mats)
        self.h = getattr(lib, prefix + "point_create")(C.byref(s), mats_arr, len(mats))

    def _f(self, n):
        return getattr(self.lib, self.p + n)

    def flux(self, direction, Vm, Vp, ids):
        Vm, Vp = np.ascontiguousarray(Vm, np.float64), np.ascontiguousarray(Vp, np.float64)
        ids = np.ascontiguousarray(ids, np.int32)
        F = np.zeros_like(Vm)
        self._f("point_flux")(self.h, len(ids), direction, abi.dptr(Vm), abi.dptr(Vp), abi.iptr(ids), abi.dptr(F))
        return F

    def c2p(self, U, ids):
        U = np.ascontiguousarray(U, np.float64)
        ids = np.ascontiguousarray(ids, np.int32)
        V = np.zeros_like(U)
        self._f("point_c2p")(self.h, len(ids), abi.dptr(U), abi.iptr(ids), abi.dptr(V))
        return V

    def p2c(self, V, ids):
        V = np.ascontiguousarray(V, np.float64)
        ids = np.ascontiguousarray(ids, np.int32)
        U = np.zeros_like(V)
        self._f("point_p2c")(self.h, len(ids), abi.dptr(V), abi.iptr(ids), abi.dptr(U))
        return U

    def riemann(self, dirs, VL, idl, VR, idr):
        n = len(idl)
        dirs, VL, VR = (np.ascontiguousarray(a, np.float64) for a in (dirs, VL, VR))
        idl, idr = np.ascontiguousarray(idl, np.int32), np.ascontiguousarray(idr, np.int32)
        Vs, Vsm, Vsp = np.zeros((n, 5)), np.zeros((n, 5)), np.zeros((n, 5))
        mid, err = np.zeros(n, np.int32), np.zeros(n, np.int32)
        self._f("point_riemann")(self.h, n, abi.dptr(dirs), abi.dptr(VL), abi.iptr(idl), abi.dptr(VR),
                                 abi.iptr(idr), abi.dptr(Vs), abi.iptr(mid), abi.dptr(Vsm), abi.dptr(Vsp),
                                 abi.iptr(err))
        return Vs, mid, Vsm, Vsp, err

    def riemann_wall(self, dirs, Vm, idm, uwall):
        """ExactRiemannSolverBase::ComputeOneSidedRiemannSolution per problem:
        returns (Vs, id, Vsm, err); Vs is zero where id = -1."""
        n = len(idm)
        dirs, Vm, uwall = (np.ascontiguousarray(a, np.float64) for a in (dirs, Vm, uwall))
        idm = np.ascontiguousarray(idm, np.int32)
        Vs, Vsm = np.zeros((n, 5)), np.zeros((n, 5))
        mid, err = np.zeros(n, np.int32), np.zeros(n, np.int32)
        self._f("point_riemann_wall")(self.h, n, abi.dptr(dirs), abi.dptr(Vm), abi.iptr(idm), abi.dptr(uwall),
                                      abi.dptr(Vs), abi.iptr(mid), abi.dptr(Vsm), abi.iptr(err))
        return Vs, mid, Vsm, err

    def close(self):
        if self.h:
            self._f("point_destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def RefCase(g, s, mats, ls=None):
    return _Case(_load(REF_SO, "m2cref_"), "m2cref_", g, s, mats, ls)


def RefPoint(s, mats):
    return _Point(_load(REF_SO, "m2cref_"), "m2cref_", s, mats)


def RefCaseCR(g, s, mats, ls=None):
    return _Case(_load(CR_SO, "m2cref_"), "m2cref_", g, s, mats, ls)


def RefPointCR(s, mats):
    return _Point(_load(CR_SO, "m2cref_"), "m2cref_", s, mats)


def DropinCase(g, s, mats, ls=None):
    return _Case(_load(DROPIN_SO, "m2cref_"), "m2cref_", g, s, mats, ls)


def _tube_worker(args):
    """One tube as one reference run (process-pool worker: a reference abort
    ends only this process). args = (scheme field dict, n, two material field
    tuples, VL, VR, nsteps, crpow); returns (V [n, 5], ID [n], t)."""
    sd, n, mt, VL, VR, nsteps, crpow = args
    from m2c_b200 import cases
    s = abi.scheme(**sd)
    mats = [abi.Material(*m) for m in mt]
    g, ls, V, ID, PHI = cases.tube_case(n, VL, VR)
    c = (RefCaseCR if crpow else RefCase)(g, s, mats, ls)
    c.set_state(V, ID, PHI)
    _, t = c.run(nsteps)
    Vr, IDr, _ = c.get_state()
    c.close()
    return Vr[1, 1, 1:-1].copy(), IDr[1, 1, 1:-1].astype(np.int32), t


def tubes(s, lens, mats, VL, VR, nsteps, which, processes=8, crpow=False):
    """Reference runs of the selected tubes (indices `which`) of a batch, in
    a spawned process pool (crpow: the build with correctly rounded
    step-control pow). Returns a list of (V, ID, t) or None where the
    reference process failed."""
    import multiprocessing as mp
    sd = {f: getattr(s, f) for f, _ in abi.Scheme._fields_}
    field = lambda m: tuple(getattr(m, f) for f, _ in abi.Material._fields_)
    jobs = [(sd, int(lens[t]), (field(mats[2 * t]), field(mats[2 * t + 1])), tuple(VL[t]), tuple(VR[t]), nsteps,
             crpow) for t in which]
    out = []
    with mp.get_context("spawn").Pool(min(processes, len(jobs))) as pool:
        res = [pool.apply_async(_tube_worker, (j,)) for j in jobs]
        for r in res:
            try:
                out.append(r.get(timeout=600))
            except Exception:
                out.append(None)
    return out
