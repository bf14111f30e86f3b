"""Parity of the single-material GPU path against the reference oracle
(the unmodified reference sources built with single-rank shims).

Bar: the FP64 path is compiled without FMA contraction and keeps the
reference's operation order, so results are expected to be bit-identical;
the asserted tolerance is 1e-12 relative (per variable, max norm).
The mixed path (FP32 reconstruction/flux, FP64 state) is checked against the
FP64 path with a stated L1 tolerance.
"""
import numpy as np
import pytest

from m2c_b200 import abi, cases
from tests.helpers import face_ghosts_mask, inner, l1_rel, rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_L1_TOL = 1e-5


def run_both(gpu, ref, g, s, mats, V, nsteps=None, t_max=float("inf"), dts=None):
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    if dts is not None:
        for dt in dts:
            sol.advance(dt)
            rc.advance(dt)
    else:
        sol.run(nsteps, t_max)
        rc.run(nsteps, t_max)
    Vg, _, _ = sol.download()
    Vr, _, _ = rc.get_state()
    return Vg, Vr, sol, rc


def test_sod_fp64_matches_reference(gpu, ref):
    g, s, mats, V = cases.sod(400)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    n, t = sol.run(100000, 0.2)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    nr, tr = rc.run(100000, 0.2)
    assert n == nr and t == tr
    Vg, _, _ = sol.download()
    Vr, _, _ = rc.get_state()
    assert rel_err(inner(Vg), inner(Vr)) <= FP64_TOL
    # star-state plateau of the exact solution (p* = 0.30313)
    p = inner(Vr)[0, 0, :, 4]
    assert abs(np.median(p[250:290]) - 0.30313) < 2e-3


def test_initial_dt_matches_reference(gpu, ref):
    g, s, mats, V = cases.random_box(20, 12, 9, seed=3)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    assert sol.compute_dt() == rc.compute_dt()


@pytest.mark.parametrize("flux", [abi.FLUX_HLLC, abi.FLUX_ROE, abi.FLUX_LLF])
@pytest.mark.parametrize("limiter", [abi.LIM_NONE, abi.LIM_GENMINMOD, abi.LIM_VANALBADA])
def test_residual_matches_reference(gpu, ref, flux, limiter):
    bc = (abi.BC_INLET, abi.BC_OUTLET, abi.BC_SLIPWALL, abi.BC_STICKWALL, abi.BC_SYMMETRY, abi.BC_SYMMETRY)
    g, s, mats, V = cases.random_box(37, 11, 10, seed=11 + flux * 3 + limiter, bc=bc, flux=flux, limiter=limiter)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    Rg, Rr = sol.residual(), rc.residual()
    assert rel_err(inner(Rg), inner(Rr)) <= FP64_TOL


@pytest.mark.parametrize("rk", [1, 2, 3])
def test_steps_match_reference(gpu, ref, rk):
    bc = (abi.BC_SYMMETRY, abi.BC_OUTLET, abi.BC_SYMMETRY, abi.BC_SLIPWALL, abi.BC_STICKWALL, abi.BC_INLET)
    g, s, mats, V = cases.random_box(40, 17, 12, seed=5, bc=bc, rk=rk, limiter=abi.LIM_VANALBADA)
    Vg, Vr, _, _ = run_both(gpu, ref, g, s, mats, V, nsteps=6)
    m = face_ghosts_mask(Vg.shape)
    assert rel_err(Vg[m], Vr[m]) <= FP64_TOL


def test_water_stiffened_gas_matches_reference(gpu, ref):
    bc = (abi.BC_INLET, abi.BC_OUTLET) + (abi.BC_SYMMETRY,) * 4
    g, s, mats, V = cases.random_box(33, 9, 9, seed=21, bc=bc, water=True, rk=3)
    Vg, Vr, _, _ = run_both(gpu, ref, g, s, mats, V, nsteps=5)
    assert rel_err(inner(Vg), inner(Vr)) <= FP64_TOL


@pytest.mark.parametrize("flux", [abi.FLUX_HLLC, abi.FLUX_ROE, abi.FLUX_LLF])
def test_nasg_water_matches_reference(gpu, ref, flux):
    """Noble-Abel stiffened gas (VarFcnNASG.h): residual and RK3 steps."""
    bc = (abi.BC_INLET, abi.BC_OUTLET) + (abi.BC_SYMMETRY,) * 4
    g, s, mats, V = cases.random_box(30, 9, 8, seed=23 + flux, bc=bc, nasg=True, rk=3, flux=flux)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    assert rel_err(inner(sol.residual()), inner(rc.residual())) <= FP64_TOL
    Vg, Vr, _, _ = run_both(gpu, ref, g, s, mats, V, nsteps=5)
    assert rel_err(inner(Vg), inner(Vr)) <= FP64_TOL


@pytest.mark.parametrize("rec_var", [abi.RECVAR_CONSERVATIVE, abi.RECVAR_PRIM_CHAR, abi.RECVAR_CONS_CHAR])
@pytest.mark.parametrize("flux", [abi.FLUX_HLLC, abi.FLUX_ROE, abi.FLUX_LLF])
@pytest.mark.parametrize("limiter", [abi.LIM_GENMINMOD, abi.LIM_VANALBADA])
def test_nonprimitive_reconstruction_matches_reference(gpu, ref, flux, limiter, rec_var):
    """Reconstruction in conservative, primitive-characteristic and
    conservative-characteristic variables (ReconstructionData::VariableType,
    FluxFcnBase.h:309-500), including the fall-back to primitive variables
    for cells with a non-physical face (Reconstructor.cpp:719-775): residual
    and RK3 steps."""
    bc = (abi.BC_INLET, abi.BC_OUTLET, abi.BC_SLIPWALL, abi.BC_STICKWALL, abi.BC_SYMMETRY, abi.BC_SYMMETRY)
    g, s, mats, V = cases.random_box(31, 10, 9, seed=41 + flux * 3 + limiter, bc=bc, flux=flux, limiter=limiter)
    s.rec_var = rec_var
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    assert rel_err(inner(sol.residual()), inner(rc.residual())) <= FP64_TOL
    Vg, Vr, _, _ = run_both(gpu, ref, g, s, mats, V, nsteps=4)
    m = face_ghosts_mask(Vg.shape)
    assert rel_err(Vg[m], Vr[m]) <= FP64_TOL


@pytest.mark.parametrize("rec_var", [abi.RECVAR_CONSERVATIVE, abi.RECVAR_PRIM_CHAR, abi.RECVAR_CONS_CHAR])
def test_nonprimitive_reconstruction_water_matches_reference(gpu, ref, rec_var):
    bc = (abi.BC_INLET, abi.BC_OUTLET) + (abi.BC_SYMMETRY,) * 4
    g, s, mats, V = cases.random_box(33, 9, 9, seed=29, bc=bc, water=True, rk=3)
    s.rec_var = rec_var
    Vg, Vr, _, _ = run_both(gpu, ref, g, s, mats, V, nsteps=5)
    assert rel_err(inner(Vg), inner(Vr)) <= FP64_TOL


def test_periodic_box_matches_tiled_reference(gpu, ref):
    """The reference has no periodic boundary: it runs a 3x3x3 tiled copy, whose
    central tile evolves as the periodic box for 2 RK3 steps (reach 6 cells/step)."""
    g, s, mats, V = cases.fourier_box(16, shape=(16, 16, 16), seed=9)
    dt = gpu.Solver(g, s, mats)
    dt.upload(V)
    dt0 = dt.compute_dt()
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    G, W = cases.tile_periodic(g, V, (3, 3, 3))
    rc = ref.RefCase(G, s, mats)
    rc.set_state(W)
    for _ in range(2):
        sol.advance(dt0)
        rc.advance(dt0)
    Vg, _, _ = sol.download()
    Vr, _, _ = rc.get_state()
    centre = inner(Vr)[16:32, 16:32, 16:32]
    assert rel_err(inner(Vg), centre) <= FP64_TOL


def test_mixed_precision_close_to_fp64(gpu):
    g, s, mats, V = cases.fourier_box(32, shape=(32, 32, 32), seed=4)
    a = gpu.Solver(g, s, mats)
    a.upload(V)
    s2 = abi.scheme(**{n: getattr(s, n) for n, _ in abi.Scheme._fields_})
    s2.precision = abi.PREC_MIXED
    b = gpu.Solver(g, s2, mats)
    b.upload(V)
    a.run(10)
    b.run(10)
    Va, _, _ = a.download()
    Vb, _, _ = b.download()
    assert l1_rel(inner(Vb), inner(Va)) <= MIXED_L1_TOL


def test_nonphysical_state_is_reported_not_trapped(gpu):
    g, s, mats, V = cases.random_box(16, 8, 8, seed=1)
    V[4, 4, 4, 0] = -1.0  # negative density: ClipDensityAndPressure + CheckState fail
    sol = gpu.Solver(g, s, mats)
    with pytest.raises(gpu.M2CError) as e:
        sol.upload(V)
    assert e.value.status == 3
    # the context stays usable
    g2, s2, m2, V2 = cases.random_box(16, 8, 8, seed=2)
    sol2 = gpu.Solver(g2, s2, m2)
    sol2.upload(V2)
    sol2.run(2)


@pytest.mark.parametrize("limiter", [abi.LIM_VANALBADA, abi.LIM_GENMINMOD])
def test_stretched_mesh_matches_reference(gpu, ref, limiter):
    """Non-uniform cell widths on all three axes (geometric growth,
    geometric shrinking, seeded jitter): the limiter coefficients A, B and
    the van Albada exponent of Reconstructor::Setup (Reconstructor.cpp:53-121)
    vary per cell, and the face areas, volumes and CFL widths with them."""
    bc = (abi.BC_INLET, abi.BC_OUTLET, abi.BC_SLIPWALL, abi.BC_SYMMETRY, abi.BC_STICKWALL, abi.BC_SYMMETRY)
    g, s, mats, V = cases.random_box(29, 13, 11, seed=31, bc=bc, limiter=limiter, mesh=cases.stretch)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    assert sol.compute_dt() == rc.compute_dt()
    assert rel_err(inner(sol.residual()), inner(rc.residual())) <= FP64_TOL
    for _ in range(5):
        sol.run(1)
        rc.run(1)
    Vg, _, _ = sol.download()
    Vr, _, _ = rc.get_state()
    assert rel_err(inner(Vg), inner(Vr)) <= FP64_TOL


def test_probes_match_reference_interpolation(gpu):
    """m2cg_set_probes: device samples of the state at fixed points after
    every step equal the reference's probe interpolation (ProbeOutput.cpp:
    219-340, 636-673, restated in oracle/probe_ref.py) applied to the
    downloaded ghosted state, bit for bit; points near the walls use the
    ghost layer, and the ones whose cell touches an edge ghost the reference
    leaves unpopulated use its averaging rule."""
    from oracle import probe_ref
    bc = (abi.BC_INLET, abi.BC_OUTLET, abi.BC_SLIPWALL, abi.BC_SYMMETRY, abi.BC_STICKWALL, abi.BC_SYMMETRY)
    g, s, mats, V = cases.random_box(17, 11, 9, seed=5, bc=bc, mesh=cases.stretch)
    xc, yc, zc = abi.cell_centres(g)
    mesh = getattr(g, "_mesh", {})
    widths = [mesh[a][1] for a in range(3)]
    coords = [probe_ref.ghosted_coords(c, w) for c, w in zip((xc, yc, zc), widths)]
    rng = np.random.default_rng(3)
    pts = [[rng.uniform(coords[a][0], coords[a][-1] - 1e-12) for a in range(3)] for _ in range(40)]
    pts += [[coords[0][0], coords[1][1], coords[2][5]], [coords[0][-2], coords[1][-2], coords[2][-2]],
            [0.5 * (coords[0][0] + coords[0][1]), 0.5 * (coords[1][-2] + coords[1][-1]), coords[2][3]]]
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    sol.set_probes(pts, every=2, capacity=8)
    sol.sample_probes()
    sol.run(4)
    rec = sol.read_probes()
    assert rec.shape == (3, 2 + 5 * len(pts))
    assert list(rec[:, 1]) == [0.0, 2.0, 4.0]
    Vd, _, _ = sol.download()
    setup = probe_ref.setup(pts, coords, (g.nx, g.ny, g.nz))
    want = np.array([[probe_ref.interpolate(Vd, e, c) for c in range(5)] for e in setup]).ravel()
    assert np.array_equal(rec[-1, 2:], want), np.abs(rec[-1, 2:] - want).max()
    assert len(sol.read_probes()) == 0
