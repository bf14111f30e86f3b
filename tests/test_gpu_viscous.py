"""Viscous fluxes of constant-viscosity materials against the reference
oracle (ViscosityOperator::AddDiffusionFluxes with ViscoFcnConstant,
InterpolatorLinear and GradientCalculatorCentral, set up as Main.cpp does).

Bar: the FP64 path adds the viscous face fluxes to each cell's flux sum in
the reference's order, without FMA contraction, so residuals and steps are
expected to be bit-identical; asserted at 1e-12 relative (max norm per
variable). The mixed path is checked against the FP64 path in L1.
"""
import numpy as np
import pytest

from m2c_b200 import abi, cases
from tests.helpers import inner, l1_rel, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12


def viscous_box(bc, mesh=None, precision=abi.PREC_FP64, mu=2.0e-3, bulk=7.0e-4, dims=(14, 11, 9)):
    g, s, mats, V = cases.random_box(*dims, seed=5, bc=bc, rk=3, precision=precision, mesh=mesh)
    mats = [abi.material(1.4, 0.0, mu=mu, mu_bulk=bulk)]
    return g, s, mats, V


BCS = {
    "symmetry": (abi.BC_SYMMETRY,) * 6,
    "inlet_stickwall_slipwall": (abi.BC_INLET, abi.BC_OUTLET, abi.BC_STICKWALL, abi.BC_STICKWALL,
                                 abi.BC_SLIPWALL, abi.BC_SYMMETRY),
}


@pytest.mark.parametrize("dims", [(14, 11, 9), (9, 14, 11)])
@pytest.mark.parametrize("bcname", sorted(BCS))
def test_viscous_residual_matches_reference(gpu, ref, bcname, dims):
    """The residual of one stage (advective + viscous fluxes over -volume) on
    a box with every boundary rule the viscous ghosts take. With ny >= nx the
    reference's ghost test (SpaceVariable.h:150-158, whose x clause reads
    j >= NX) zeroes the velocity derivatives on the top y-ghost row and on the
    z-ghost layers' rows j >= nx; the (9, 14, 11) box has both."""
    g, s, mats, V = viscous_box(BCS[bcname], dims=dims)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    Rg, Rr = inner(sol.residual()), inner(rc.residual())
    assert rel_err(Rg, Rr) <= TOL
    # the viscous part is not negligible: the inviscid residual differs
    g2, s2, _, _ = viscous_box(BCS[bcname], dims=dims)
    inv = gpu.Solver(g2, s2, [abi.material(1.4, 0.0)])
    inv.upload(V)
    assert rel_err(inner(inv.residual()), Rr) > 1e-6
    sol.close()
    inv.close()


@pytest.mark.parametrize("bcname", sorted(BCS))
def test_viscous_steps_match_reference(gpu, ref, bcname):
    g, s, mats, V = viscous_box(BCS[bcname])
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    n, t = sol.run(6)
    nr, tr = rc.run(6)
    assert n == nr and t == tr
    Vg, _, _ = sol.download()
    Vr, _, _ = rc.get_state()
    assert rel_err(inner(Vg), inner(Vr)) <= TOL
    sol.close()


def test_viscous_on_stretched_mesh_matches_reference(gpu, ref):
    """Non-uniform widths: the interpolation weights and the three-point
    derivative coefficients depend on the index (Interpolator.cpp:145-185,
    GradientCalculatorCentral.cpp:226-366)."""
    g, s, mats, V = viscous_box(BCS["inlet_stickwall_slipwall"], mesh=cases.stretch)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    assert rel_err(inner(sol.residual()), inner(rc.residual())) <= TOL
    sol.run(4)
    rc.run(4)
    assert rel_err(inner(sol.download()[0]), inner(rc.get_state()[0])) <= TOL
    sol.close()


def test_viscous_bubble_two_materials_matches_reference(gpu, ref):
    """Water and air with their own viscosities: at faces between the two
    materials each side takes its own material's flux, except on z faces,
    where the reference evaluates both sides with the right cell's
    (ViscosityOperator.cpp:384)."""
    if not ref.available("crpow"):
        pytest.skip("reference oracle with correctly rounded pow not built (make -C oracle refcr)")
    g, s, mats, ls, V, ID, PHI = cases.bubble_case(20, reinit_frequency=-1, radius=4.0e-3)
    mats = [abi.material(mats[0].gamma, mats[0].p_c, mu=1.0e-3, mu_bulk=3.0e-3),
            abi.material(mats[1].gamma, mats[1].p_c, mu=1.8e-5)]
    V[1:-1, 1:-1, 1:-1, 1:4] += np.array([30.0, -20.0, 10.0])
    sol = gpu.Solver(g, s, mats, ls)
    sol.upload(V, ID, PHI)
    rc = ref.RefCaseCR(g, s, mats, ls)
    rc.set_state(V, ID, PHI)
    assert rel_err(inner(sol.residual()), inner(rc.residual())) <= TOL
    for _ in range(3):
        sol.run(1)
        rc.run(1)
    Vg, IDg, Pg = sol.download()
    Vr, IDr, Pr = rc.get_state()
    assert np.array_equal(inner(IDg), inner(IDr))
    assert rel_err(inner(Vg), inner(Vr)) <= TOL
    sol.close()


def test_viscous_mixed_tracks_fp64(gpu):
    bc = BCS["inlet_stickwall_slipwall"]
    out = []
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        g, s, mats, V = viscous_box(bc, precision=prec)
        sol = gpu.Solver(g, s, mats)
        sol.upload(V)
        sol.run(10)
        out.append(inner(sol.download()[0]))
        sol.close()
    assert l1_rel(out[1], out[0]) <= 1e-5


def test_batched_tubes_refuse_viscosity(gpu):
    lens, mats, VL, VR, _ = cases.tubes(2, seed=3)
    mats = list(mats)
    mats[0] = abi.material(mats[0].gamma, mats[0].p_c, mu=1e-3)
    with pytest.raises(gpu.M2CError):
        gpu.Batch(cases.tube_scheme(), lens, mats, VL, VR)


HEAT_BC = (abi.BC_INLET, abi.BC_OUTLET, abi.BC_SYMMETRY, abi.BC_STICKWALL, abi.BC_SLIPWALL, abi.BC_SYMMETRY)


@pytest.mark.parametrize("law", ["cv", "cp"])
@pytest.mark.parametrize("dims", [(14, 11, 9), (9, 14, 11)])
def test_heat_diffusion_matches_reference(gpu, ref, law, dims):
    """HeatDiffusionOperator::AddDiffusionFluxes: the temperature from the
    EOS's law (T0 + (e - e0)/cv, or T0 + (e + p/rho - h0)/cp), the central
    temperature difference across each face times the harmonic mean of the
    two diffusivities, energy only, added after the viscous fluxes; with and
    without viscosity, residual and whole steps."""
    g, s, _, V = cases.random_box(*dims, seed=5, bc=HEAT_BC, rk=3)
    kw = dict(cv=2.5, T0=1.0, e0=0.5) if law == "cv" else dict(cp=3.5, T0=1.0, h0=0.7)
    for mu in (0.0, 2.0e-3):
        # diffusivity 0.02: the explicit step has no diffusive time-step limit
        # (as in the reference); 0.2 drives both codes to a non-physical state
        mats = [abi.material(1.4, 0.0, heat_diffusivity=0.02, mu=mu, **kw)]
        sol = gpu.Solver(g, s, mats)
        sol.upload(V)
        rc = ref.RefCase(g, s, mats)
        rc.set_state(V)
        assert rel_err(inner(sol.residual()), inner(rc.residual())) <= TOL
        sol.run(4)
        rc.run(4)
        assert rel_err(inner(sol.download()[0]), inner(rc.get_state()[0])) <= TOL
        sol.close()


def test_heat_diffusion_two_materials_matches_reference(gpu, ref):
    """Different diffusivities on the two sides of the bubble (harmonic mean
    at the interface, the y and z faces reusing the x face's denominator as
    the reference does), with a NASG liquid's temperature law on one side."""
    if not ref.available("crpow"):
        pytest.skip("reference oracle with correctly rounded pow not built (make -C oracle refcr)")
    g, s, mats, ls, V, ID, PHI = cases.bubble_case(20, reinit_frequency=-1, radius=4.0e-3)
    mats = [abi.material(mats[0].gamma, mats[0].p_c, heat_diffusivity=0.6, cv=4180.0, T0=293.0, e0=0.0,
                         mu=1.0e-3),
            abi.material(mats[1].gamma, mats[1].p_c, heat_diffusivity=0.026, cv=718.0, T0=293.0, e0=2.1e5)]
    sol = gpu.Solver(g, s, mats, ls)
    sol.upload(V, ID, PHI)
    rc = ref.RefCaseCR(g, s, mats, ls)
    rc.set_state(V, ID, PHI)
    assert rel_err(inner(sol.residual()), inner(rc.residual())) <= TOL
    for _ in range(3):
        sol.run(1)
        rc.run(1)
    Vg, IDg, _ = sol.download()
    Vr, IDr, _ = rc.get_state()
    assert np.array_equal(inner(IDg), inner(IDr))
    assert rel_err(inner(Vg), inner(Vr)) <= TOL
    sol.close()


def test_heat_diffusion_nasg_matches_reference(gpu, ref):
    g, s, _, V = cases.random_box(12, 10, 8, seed=9, bc=HEAT_BC, rk=3, nasg=True)
    mats = [abi.material(1.19, 7.028e8, eos=abi.EOS_NASG, b=6.61e-4, q=-1.177788e6, heat_diffusivity=0.6,
                         cv=3610.0)]
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    assert rel_err(inner(sol.residual()), inner(rc.residual())) <= TOL
    sol.close()
