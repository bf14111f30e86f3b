"""The oracle's RK loop with an embedded surface (oracle/ref_harness.cpp,
m2cref_run_walls: the statements of TimeIntegratorRK2 / RK3::
AdvanceOneTimeStep with a hand-written EmbeddedBoundaryDataSet) is pinned
against the reference's own integrator: with a surface that cuts no face the
two runs agree bit for bit, for RK2 and RK3 and for several boundary rules.
CPU only."""
import numpy as np
import pytest

from m2c_b200 import abi, cases


@pytest.mark.parametrize("rk", [2, 3])
@pytest.mark.parametrize("bc", [(abi.BC_SYMMETRY,) * 6,
                                (abi.BC_INLET, abi.BC_OUTLET, abi.BC_STICKWALL, abi.BC_SLIPWALL, abi.BC_SYMMETRY,
                                 abi.BC_SYMMETRY)])
def test_oracle_wall_loop_equals_reference_integrator_without_cuts(ref, rk, bc):
    g, s, mats, V = cases.random_box(12, 10, 8, seed=3, rk=rk, bc=bc)
    none = np.zeros((0, 3))
    a = ref.RefCase(g, s, mats)
    a.set_state(V)
    na, ta = a.run_walls(np.zeros((0, 4), np.int32), none, none, none, none, 5)
    b = ref.RefCase(g, s, mats)
    b.set_state(V)
    nb, tb = b.run(5)
    assert na == nb == 5 and ta == tb
    assert np.array_equal(a.get_state()[0], b.get_state()[0])


def test_oracle_wall_residual_without_cuts_equals_plain_residual(ref):
    g, s, mats, V = cases.random_box(12, 10, 8, seed=3)
    none = np.zeros((0, 3))
    a = ref.RefCase(g, s, mats)
    a.set_state(V)
    assert np.array_equal(a.residual_walls(np.zeros((0, 4), np.int32), none, none, none, none), a.residual())
