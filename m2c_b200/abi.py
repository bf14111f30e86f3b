"""ctypes mirror of the C structs in include/m2c_gpu.h.

The defaults are the reference's IoData defaults:
MaterialModelData (IoData.cpp:860-871), StiffenedGasModelData (598-612),
ReconstructionData (1049-1058), SchemeData (1154-1160),
LevelSetSchemeData/LevelSetReinitializationData (1205-1265),
ExactRiemannSolverData (1345-1357), MultiPhaseData (1400-1417).
"""
import ctypes as C
import sys

import numpy as np

DBL_MAX = sys.float_info.max

BC_NONE, BC_INLET, BC_OUTLET, BC_SLIPWALL, BC_STICKWALL, BC_SYMMETRY = 0, 1, 2, 3, 4, 5
BC_PERIODIC = 100
EOS_SG, EOS_NASG = 0, 1
FLUX_ROE, FLUX_LLF, FLUX_HLLC = 0, 1, 2
REC_CONSTANT, REC_LINEAR = 0, 1
LIM_NONE, LIM_GENMINMOD, LIM_VANALBADA = 0, 1, 2
RECVAR_PRIMITIVE, RECVAR_CONSERVATIVE, RECVAR_PRIM_CHAR, RECVAR_CONS_CHAR = 0, 1, 2, 3
PREC_FP64, PREC_MIXED = 0, 1
MPFLUX_EXACT, MPFLUX_NUMERICAL, MPFLUX_LLF = 0, 1, 2
RIEMANN_NORMAL_LEVEL_SET, RIEMANN_NORMAL_MESH, RIEMANN_NORMAL_AVERAGE = 0, 1, 2
PHASECHANGE_RIEMANN_SOLUTION, PHASECHANGE_EXTRAPOLATION = 0, 1
PHASECHANGE_ALL, PHASECHANGE_UPWIND = 0, 1
OK, ERR_ARG, ERR_CUDA, ERR_STATE, ERR_RIEMANN, ERR_REINIT, ERR_ITER_CAP, ERR_NOMEM, ERR_UNSUPPORTED = range(9)
LSBC_NONE, LSBC_ZERO_NEUMANN, LSBC_LINEAR_EXTRAPOLATION, LSBC_NON_NEGATIVE = 0, 1, 2, 3

_dp = C.POINTER(C.c_double)


class Grid(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("x0", C.c_double), ("xmax", C.c_double), ("y0", C.c_double), ("ymax", C.c_double),
        ("z0", C.c_double), ("zmax", C.c_double),
        ("xc", _dp), ("dx", _dp), ("yc", _dp), ("dy", _dp), ("zc", _dp), ("dz", _dp),
        ("bc", C.c_int * 6),
        ("inlet", C.c_double * 5), ("outlet", C.c_double * 5),
    ]


class Material(C.Structure):
    _fields_ = [
        ("eos", C.c_int), ("gamma", C.c_double), ("p_c", C.c_double), ("b", C.c_double), ("q", C.c_double),
        ("rhomin", C.c_double), ("pmin", C.c_double), ("rhomax", C.c_double), ("pmax", C.c_double),
        ("failsafe_density", C.c_double), ("mu", C.c_double), ("mu_bulk", C.c_double),
        ("heat_diffusivity", C.c_double), ("cv", C.c_double), ("T0", C.c_double), ("e0", C.c_double),
        ("cp", C.c_double), ("h0", C.c_double),
    ]


class Scheme(C.Structure):
    _fields_ = [
        ("flux", C.c_int), ("roe_delta", C.c_double), ("rec_type", C.c_int), ("limiter", C.c_int),
        ("minmod_coeff", C.c_double), ("slope_near_interface", C.c_int), ("rec_var", C.c_int),
        ("rk_order", C.c_int), ("cfl", C.c_double), ("precision", C.c_int),
        ("mp_flux", C.c_int), ("mp_recon", C.c_int), ("mp_phasechange_type", C.c_int),
        ("mp_phasechange_dir", C.c_int), ("mp_apply_failsafe_density", C.c_int),
        ("riem_maxits_main", C.c_int), ("riem_maxits_bracket", C.c_int), ("riem_maxits_shock", C.c_int),
        ("riem_nsteps_rarefaction", C.c_int),
        ("riem_tol_main", C.c_double), ("riem_tol_shock", C.c_double), ("riem_tol_rarefaction", C.c_double),
        ("riem_min_pressure", C.c_double), ("riem_failure_threshold", C.c_double),
        ("riem_pressure_at_failure", C.c_double), ("riem_warm_delta", C.c_double),
        ("mp_riemann_normal", C.c_int), ("riem_warm_gate", C.c_double),
        ("ebm_riemann_normal", C.c_int), ("ebm_recon", C.c_int),
        ("inactive_density", C.c_double), ("inactive_pressure", C.c_double), ("inactive_energy", C.c_double),
    ]


class LevelSet(C.Structure):
    _fields_ = [
        ("material_id", C.c_int), ("bc", C.c_int * 6), ("reinit_frequency", C.c_int),
        ("reinit_maxits", C.c_int), ("reinit_cfl", C.c_double), ("reinit_tol", C.c_double),
        ("reinit_first_layer", C.c_int), ("solver", C.c_int), ("flux", C.c_int), ("delta", C.c_double),
        ("rec_type", C.c_int), ("limiter", C.c_int), ("minmod_coeff", C.c_double),
    ]


def material(gamma=1.4, p_c=0.0, eos=EOS_SG, b=0.0, q=0.0, rhomin=0.0, pmin=-DBL_MAX,
             rhomax=DBL_MAX, pmax=DBL_MAX, failsafe_density=1.0e-10, mu=0.0, mu_bulk=0.0, heat_diffusivity=0.0,
             cv=0.0, T0=0.0, e0=0.0, cp=0.0, h0=0.0):
    return Material(eos, gamma, p_c, b, q, rhomin, pmin, rhomax, pmax, failsafe_density, mu, mu_bulk,
                    heat_diffusivity, cv, T0, e0, cp, h0)


# EmbeddedBoundaryMethodData::RiemannNormal (IoData.h:1345)
EBM_NORMAL_SURFACE, EBM_NORMAL_MESH, EBM_NORMAL_AVERAGE = 0, 1, 2


def scheme(**kw):
    s = Scheme()
    s.flux = FLUX_HLLC
    s.roe_delta = 0.2
    s.rec_type = REC_LINEAR
    s.limiter = LIM_NONE
    s.minmod_coeff = 1.2
    s.slope_near_interface = 1
    s.rec_var = RECVAR_PRIMITIVE
    s.rk_order = 2
    s.cfl = 0.5
    s.precision = PREC_FP64
    s.mp_flux = MPFLUX_NUMERICAL
    s.mp_recon = 0
    s.mp_phasechange_type = 0
    s.mp_phasechange_dir = 1
    s.mp_apply_failsafe_density = 1
    s.riem_maxits_main = 200
    s.riem_maxits_bracket = 100
    s.riem_maxits_shock = 200
    s.riem_nsteps_rarefaction = 200
    s.riem_tol_main = 1.0e-4
    s.riem_tol_shock = 1.0e-12
    s.riem_tol_rarefaction = 1.0e-8
    s.riem_min_pressure = -1.0e8
    s.riem_failure_threshold = 0.2
    s.riem_pressure_at_failure = 1.0e-8
    s.riem_warm_delta = 3.0e-4
    s.mp_riemann_normal = RIEMANN_NORMAL_MESH
    s.ebm_riemann_normal = EBM_NORMAL_MESH
    s.ebm_recon = 0
    s.inactive_density = 1.0e-6
    s.inactive_pressure = 0.0
    s.inactive_energy = 0.0
    for k, v in kw.items():
        if not hasattr(s, k):
            raise AttributeError(k)
        setattr(s, k, v)
    return s


LS_FINITE_VOLUME, LS_FINITE_DIFFERENCE = 0, 1
LSFLUX_ROE, LSFLUX_LLF, LSFLUX_UPWIND = 0, 1, 2


def levelset(material_id=1, bc=(LSBC_ZERO_NEUMANN,) * 6, reinit_frequency=-1, reinit_maxits=30,
             reinit_cfl=0.8, reinit_tol=2.0e-4, reinit_first_layer=0, solver=LS_FINITE_DIFFERENCE,
             flux=LSFLUX_ROE, delta=0.2, rec_type=1, limiter=0, minmod_coeff=1.2):
    return LevelSet(material_id, (C.c_int * 6)(*bc), reinit_frequency, reinit_maxits, reinit_cfl,
                    reinit_tol, reinit_first_layer, solver, flux, delta, rec_type, limiter, minmod_coeff)


def grid(nx, ny, nz, x=(0.0, 1.0), y=(0.0, 1.0), z=(0.0, 1.0), bc=(BC_SYMMETRY,) * 6,
         inlet=(1.0, 0.0, 0.0, 0.0, 1.0), outlet=(1.0, 0.0, 0.0, 0.0, 1.0)):
    g = Grid()
    g.nx, g.ny, g.nz = nx, ny, nz
    g.x0, g.xmax = x
    g.y0, g.ymax = y
    g.z0, g.zmax = z
    g.bc = (C.c_int * 6)(*bc)
    g.inlet = (C.c_double * 5)(*inlet)
    g.outlet = (C.c_double * 5)(*outlet)
    return g


def ghosted_shape(g, dof=None):
    s = (g.nz + 2, g.ny + 2, g.nx + 2)
    return s + (dof,) if dof else s


def set_mesh(g, axis, widths):
    """Give axis 0/1/2 of g a non-uniform mesh: cell widths `widths` (length
    n) laid end to end from the axis' lower bound; the centres and widths
    are kept alive on g and passed through m2cg_grid's xc/dx (yc/dy, zc/dz)."""
    w = np.ascontiguousarray(widths, dtype=np.float64)
    lo = (g.x0, g.y0, g.z0)[axis]
    faces = lo + np.concatenate(([0.0], np.cumsum(w)))
    c = np.ascontiguousarray(0.5 * (faces[:-1] + faces[1:]))
    keep = getattr(g, "_mesh", {})
    keep[axis] = (c, w)
    g._mesh = keep
    pc, pw = c.ctypes.data_as(C.POINTER(C.c_double)), w.ctypes.data_as(C.POINTER(C.c_double))
    if axis == 0:
        g.xc, g.dx, g.xmax = pc, pw, float(faces[-1])
    elif axis == 1:
        g.yc, g.dy, g.ymax = pc, pw, float(faces[-1])
    else:
        g.zc, g.dz, g.zmax = pc, pw, float(faces[-1])


def cell_centres(g):
    """Cell centres as MeshGenerator::ComputeMesh1DUniform (MeshGenerator.cpp:146-158),
    or the ones given with set_mesh."""
    out = []
    mesh = getattr(g, "_mesh", {})
    for axis, (n, a, b) in enumerate(((g.nx, g.x0, g.xmax), (g.ny, g.y0, g.ymax), (g.nz, g.z0, g.zmax))):
        if axis in mesh:
            out.append(mesh[axis][0].copy())
            continue
        h = (b - a) / n
        out.append(np.array([a + 0.5 * h + i * h for i in range(n)]))
    return out


def dptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def iptr(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int))


# numpy mirror of m2cg_material (C layout: int, padding, nine doubles)
MATERIAL_DTYPE = np.dtype([("eos", "<i4"), ("gamma", "<f8"), ("p_c", "<f8"), ("b", "<f8"), ("q", "<f8"),
                           ("rhomin", "<f8"), ("pmin", "<f8"), ("rhomax", "<f8"), ("pmax", "<f8"),
                           ("failsafe_density", "<f8"), ("mu", "<f8"), ("mu_bulk", "<f8"),
                           ("heat_diffusivity", "<f8"), ("cv", "<f8"), ("T0", "<f8"), ("e0", "<f8"), ("cp", "<f8"),
                           ("h0", "<f8")], align=True)


def material_table(gamma, p_c):
    """Stiffened-gas materials as a MATERIAL_DTYPE array (fast path for
    large per-problem material tables), with the IoData defaults."""
    gamma = np.asarray(gamma, np.float64)
    t = np.zeros(len(gamma), MATERIAL_DTYPE)
    t["eos"] = EOS_SG
    t["gamma"] = gamma
    t["p_c"] = p_c
    t["pmin"] = -DBL_MAX
    t["rhomax"] = DBL_MAX
    t["pmax"] = DBL_MAX
    t["failsafe_density"] = 1.0e-10
    return t


def material_array(mats):
    """Pointer to a C array of m2cg_material from a list of Material or a
    MATERIAL_DTYPE numpy array (kept alive by the caller)."""
    if isinstance(mats, np.ndarray):
        assert mats.dtype == MATERIAL_DTYPE and mats.flags.c_contiguous
        assert MATERIAL_DTYPE.itemsize == C.sizeof(Material)
        return mats.ctypes.data_as(C.POINTER(Material))
    return (Material * len(mats))(*mats)
