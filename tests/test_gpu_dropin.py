"""The drop-in boundary at work: the reference's own driver (the unmodified
M2C sources built in place, oracle/ref_harness.cpp mirroring Main.cpp) with
its TimeIntegratorRK2/RK3 replaced by the GPU integrator a maintainer adds
(m2c_b200/adapter/TimeIntegratorGPU.h: AdvanceOneTimeStep over the C-ABI).
The reference still computes the CFL time step on the CPU from the state
the GPU wrote back into its SpaceVariable3D arrays. Results must equal the
pure reference run at the parity bars of the other tests (1e-12 single
material, 1e-10 two materials with identical IDs)."""
import numpy as np
import pytest

from m2c_b200 import abi, cases
from tests.helpers import face_ghosts_mask, inner, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dropin(gpu):
    from oracle import ref
    if not ref.available("ref") or not ref.available("dropin"):
        pytest.skip("reference / drop-in builds not present (make -C oracle ref dropin)")
    return ref


def test_dropin_sod_matches_reference(dropin):
    g, s, mats, V = cases.sod(400)
    a = dropin.RefCase(g, s, mats)
    b = dropin.DropinCase(g, s, mats)
    for c in (a, b):
        c.set_state(V)
    na, ta = a.run(100000, 0.2)
    nb, tb = b.run(100000, 0.2)
    assert na == nb and ta == tb
    Va, Vb = a.get_state()[0], b.get_state()[0]
    assert rel_err(inner(Vb), inner(Va)) <= 1e-12


def test_dropin_box_rk3_with_ghosts_matches_reference(dropin):
    bc = (abi.BC_SYMMETRY, abi.BC_OUTLET, abi.BC_SYMMETRY, abi.BC_SLIPWALL, abi.BC_STICKWALL, abi.BC_INLET)
    g, s, mats, V = cases.random_box(24, 11, 9, seed=5, bc=bc, rk=3, limiter=abi.LIM_VANALBADA)
    a = dropin.RefCase(g, s, mats)
    b = dropin.DropinCase(g, s, mats)
    for c in (a, b):
        c.set_state(V)
        c.run(5)
    Va, Vb = a.get_state()[0], b.get_state()[0]
    m = face_ghosts_mask(Va.shape)  # ghost layers as the reference's boundary conditions left them
    assert rel_err(Vb[m], Va[m]) <= 1e-12


def test_dropin_bubble_matches_reference(dropin):
    g, s, mats, ls, V, ID, PHI = cases.bubble_case(16)
    a = dropin.RefCase(g, s, mats, ls)
    b = dropin.DropinCase(g, s, mats, ls)
    for c in (a, b):
        c.set_state(V, ID, PHI)
        c.run(4)
    Va, IDa, Pa = a.get_state()
    Vb, IDb, Pb = b.get_state()
    assert np.array_equal(inner(IDb), inner(IDa))
    assert rel_err(inner(Vb), inner(Va)) <= 1e-10
    assert rel_err(inner(Pb), inner(Pa), axis_last=False) <= 1e-10
