"""GPU parity against the golden fixtures (reference outputs committed
under tests/golden/), so parity is checked on machines where the reference
cannot be built. Bars as in the oracle-driven tests: FP64 single material
1e-12 relative, two materials 1e-10 with identical material IDs, exact
Riemann problems within the pow()-rounding statistics of test_gpu_riemann."""
import os

import numpy as np
import pytest

from m2c_b200 import abi, cases
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name))


def inner(A):
    return A[1:-1, 1:-1, 1:-1]


def test_sod_matches_golden(gpu):
    d = load("sod400.npz")
    g, s, mats, V = cases.sod(400)
    sol = gpu.Solver(g, s, mats)
    sol.upload(d["V0"])
    n, t = sol.run(100000, 0.2)
    assert n == int(d["steps"]) and t == float(d["t"])
    assert rel_err(inner(sol.download()[0]), inner(d["V"])) <= 1e-12


def test_residuals_match_golden(gpu):
    d = load("residual_10x6x5.npz")
    bc = (abi.BC_INLET, abi.BC_OUTLET, abi.BC_SLIPWALL, abi.BC_STICKWALL, abi.BC_SYMMETRY, abi.BC_SYMMETRY)
    for flux in (abi.FLUX_HLLC, abi.FLUX_ROE, abi.FLUX_LLF):
        for lim in (abi.LIM_NONE, abi.LIM_GENMINMOD, abi.LIM_VANALBADA):
            g, s, mats, _ = cases.random_box(10, 6, 5, seed=11 + flux * 3 + lim, bc=bc, flux=flux, limiter=lim)
            sol = gpu.Solver(g, s, mats)
            sol.upload(d[f"V_{flux}_{lim}"])
            assert rel_err(inner(sol.residual()), d[f"R_{flux}_{lim}"]) <= 1e-12, (flux, lim)
            sol.close()


def test_steps_match_golden(gpu):
    d = load("steps_12x7x5.npz")
    bc = (abi.BC_SYMMETRY, abi.BC_OUTLET, abi.BC_SYMMETRY, abi.BC_SLIPWALL, abi.BC_STICKWALL, abi.BC_INLET)
    for rk in (1, 2, 3):
        g, s, mats, _ = cases.random_box(12, 7, 5, seed=5, bc=bc, rk=rk, limiter=abi.LIM_VANALBADA)
        sol = gpu.Solver(g, s, mats)
        sol.upload(d[f"V0_{rk}"])
        sol.run(6)
        assert rel_err(inner(sol.download()[0]), d[f"V_{rk}"]) <= 1e-12, rk
        sol.close()


def test_riemann_matches_golden(gpu):
    d = load("riemann400.npz")
    mats = [abi.material(g, p) for g, p in d["mats"]]
    Vs, mid, Vsm, Vsp, it, err = gpu.riemann_batch(abi.scheme(), mats, d["VL"], d["idl"], d["VR"], d["idr"], d["dirs"])
    both = (err == 0) & (d["err"] == 0)
    assert both.mean() >= 0.95
    for a, k in ((Vs, "Vs"), (Vsm, "Vsm"), (Vsp, "Vsp")):
        b = d[k]
        rel = (np.abs(a - b) / np.maximum(np.abs(b), 1e-300))[both].max(axis=1)
        assert (rel <= 1e-12).mean() >= 0.95, k
        assert rel.max() <= abi.scheme().riem_tol_main, k


def test_bubble_matches_golden(gpu):
    d = load("bubble16.npz")
    g, s, mats, ls, V, ID, PHI = cases.bubble_case(16)
    sol = gpu.Solver(g, s, mats, ls)
    sol.upload(V, ID, PHI)
    sol.run(3)
    Vg, IDg, Pg = sol.download()
    assert np.array_equal(inner(IDg), d["ID"])
    assert rel_err(inner(Vg), d["V"]) <= 1e-10
    assert rel_err(inner(Pg), d["PHI"], axis_last=False) <= 1e-10


def test_tube_matches_golden(gpu):
    d = load("tube137.npz")
    mats = [abi.material(g, p) for g, p in d["mats"]]
    b = gpu.Batch(cases.tube_scheme(), [137], mats, d["VL"][None, :], d["VR"][None, :])
    b.run(20)
    V, ID, t = b.download()
    assert np.array_equal(ID[0], d["ID"])
    assert rel_err(V[0], d["V"]) <= 1e-10
    assert abs(t[0] - float(d["t"])) <= 1e-12 * abs(float(d["t"]))
