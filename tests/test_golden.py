"""Golden fixtures (tests/golden/, written by make_golden.py from the
reference built in place): they load, and — where the reference oracle is
built on this machine — the oracle reproduces them bit for bit, which pins
the oracle build to the fixtures the GPU tests use. No GPU."""
import os

import numpy as np
import pytest

from m2c_b200 import abi, cases

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = ["sod400.npz", "residual_10x6x5.npz", "steps_12x7x5.npz", "riemann400.npz", "bubble16.npz", "tube137.npz"]


def load(name):
    return np.load(os.path.join(GOLD, name))


def inner(A):
    return A[1:-1, 1:-1, 1:-1]


@pytest.mark.parametrize("name", FILES)
def test_fixture_loads_and_is_finite(name):
    d = load(name)
    for k in d.files:
        assert np.all(np.isfinite(d[k])), (name, k)


def test_sod_fixture_has_the_exact_star_plateau():
    d = load("sod400.npz")
    p = inner(d["V"])[0, 0, :, 4]
    assert abs(np.median(p[250:290]) - 0.30313) < 2e-3  # exact p* of the Sod problem
    assert abs(float(d["t"]) - 0.2) < 1e-14


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as r
    if not r.available("ref"):
        pytest.skip("reference oracle not built (make -C oracle ref)")
    return r


def test_oracle_reproduces_sod(ref):
    d = load("sod400.npz")
    g, s, mats, V = cases.sod(400)
    assert np.array_equal(V, d["V0"])
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    n, t = rc.run(100000, 0.2)
    assert n == int(d["steps"]) and t == float(d["t"])
    assert np.array_equal(inner(rc.get_state()[0]), inner(d["V"]))


def test_oracle_reproduces_residuals(ref):
    d = load("residual_10x6x5.npz")
    bc = (abi.BC_INLET, abi.BC_OUTLET, abi.BC_SLIPWALL, abi.BC_STICKWALL, abi.BC_SYMMETRY, abi.BC_SYMMETRY)
    for flux in (abi.FLUX_HLLC, abi.FLUX_ROE, abi.FLUX_LLF):
        for lim in (abi.LIM_NONE, abi.LIM_GENMINMOD, abi.LIM_VANALBADA):
            g, s, mats, V = cases.random_box(10, 6, 5, seed=11 + flux * 3 + lim, bc=bc, flux=flux, limiter=lim)
            rc = ref.RefCase(g, s, mats)
            rc.set_state(d[f"V_{flux}_{lim}"])
            assert np.array_equal(inner(rc.residual()), d[f"R_{flux}_{lim}"]), (flux, lim)


def test_oracle_reproduces_riemann(ref):
    d = load("riemann400.npz")
    mats = [abi.material(g, p) for g, p in d["mats"]]
    Vs, mid, Vsm, Vsp, err = ref.RefPoint(abi.scheme(), mats).riemann(d["dirs"], d["VL"], d["idl"], d["VR"], d["idr"])
    for a, k in ((Vs, "Vs"), (mid, "id"), (Vsm, "Vsm"), (Vsp, "Vsp"), (err, "err")):
        assert np.array_equal(a, d[k]), k


def test_oracle_reproduces_bubble(ref):
    d = load("bubble16.npz")
    g, s, mats, ls, V, ID, PHI = cases.bubble_case(16)
    rc = ref.RefCase(g, s, mats, ls)
    rc.set_state(V, ID, PHI)
    rc.run(3)
    Vr, IDr, Pr = rc.get_state()
    assert np.array_equal(inner(Vr), d["V"]) and np.array_equal(inner(IDr), d["ID"])
    assert np.array_equal(inner(Pr), d["PHI"])
