"""Regenerate the golden fixtures of this directory from the reference.

The reference ships no golden vectors for this path, so these fixtures are
outputs of the reference itself: its unmodified C++ sources built in place
with single-rank shims (oracle/Makefile, target `ref`), run through
oracle/ref.py on seeded inputs from m2c_b200/cases.py. Each fixture stores
its inputs and the reference's outputs, so GPU parity can be checked where
the reference cannot be built (tests/test_gpu_golden.py).

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from m2c_b200 import abi, cases  # noqa: E402
from oracle import ref  # noqa: E402


def inner(A):
    return A[1:-1, 1:-1, 1:-1]


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name), **arrays)
    print("wrote", name)


def main():
    assert ref.available("ref"), "build the reference oracle first: make -C oracle ref"
    # Sod shock tube to t = 0.2 (400 cells, HLLC, van Albada, RK2, CFL 0.5)
    g, s, mats, V = cases.sod(400)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    n, t = rc.run(100000, 0.2)
    Vr, _, _ = rc.get_state()
    save("sod400.npz", V0=V, V=Vr, steps=n, t=t)
    # residuals: 3 fluxes x 3 limiters on a 10x6x5 box with mixed boundaries
    bc = (abi.BC_INLET, abi.BC_OUTLET, abi.BC_SLIPWALL, abi.BC_STICKWALL, abi.BC_SYMMETRY, abi.BC_SYMMETRY)
    out = {}
    for flux in (abi.FLUX_HLLC, abi.FLUX_ROE, abi.FLUX_LLF):
        for lim in (abi.LIM_NONE, abi.LIM_GENMINMOD, abi.LIM_VANALBADA):
            g, s, mats, V = cases.random_box(10, 6, 5, seed=11 + flux * 3 + lim, bc=bc, flux=flux, limiter=lim)
            rc = ref.RefCase(g, s, mats)
            rc.set_state(V)
            out[f"V_{flux}_{lim}"] = V
            out[f"R_{flux}_{lim}"] = inner(rc.residual())
    save("residual_10x6x5.npz", **out)
    # 6 steps of RK1/2/3 on a 12x7x5 box
    out = {}
    bc = (abi.BC_SYMMETRY, abi.BC_OUTLET, abi.BC_SYMMETRY, abi.BC_SLIPWALL, abi.BC_STICKWALL, abi.BC_INLET)
    for rk in (1, 2, 3):
        g, s, mats, V = cases.random_box(12, 7, 5, seed=5, bc=bc, rk=rk, limiter=abi.LIM_VANALBADA)
        rc = ref.RefCase(g, s, mats)
        rc.set_state(V)
        rc.run(6)
        out[f"V0_{rk}"] = V
        out[f"V_{rk}"] = inner(rc.get_state()[0])
    save("steps_12x7x5.npz", **out)
    # exact two-material Riemann problems
    mats, VL, idl, VR, idr, dirs = cases.riemann_problems(400, seed=3)
    Vs, mid, Vsm, Vsp, err = ref.RefPoint(abi.scheme(), mats).riemann(dirs, VL, idl, VR, idr)
    save("riemann400.npz", VL=VL, VR=VR, idl=idl, idr=idr, dirs=dirs, Vs=Vs, id=mid, Vsm=Vsm, Vsp=Vsp, err=err,
         mats=np.array([[m.gamma, m.p_c] for m in mats]))
    # air bubble in water, 16^3, 3 RK3 steps (two materials, level set)
    g, s, mats, ls, V, ID, PHI = cases.bubble_case(16)
    rc = ref.RefCase(g, s, mats, ls)
    rc.set_state(V, ID, PHI)
    rc.run(3)
    Vr, IDr, Pr = rc.get_state()
    save("bubble16.npz", V=inner(Vr), ID=inner(IDr), PHI=inner(Pr))
    # one two-material shock tube, 20 RK2 steps
    lens, tmats, TVL, TVR, _ = cases.tubes(6, seed=5)
    r = ref.tubes(cases.tube_scheme(), np.array([137] * 6, np.int32), tmats, TVL, TVR, 20, [1])[0]
    save("tube137.npz", V=r[0], ID=r[1], t=r[2], VL=TVL[1], VR=TVR[1],
         mats=np.array([[tmats[2].gamma, tmats[2].p_c], [tmats[3].gamma, tmats[3].p_c]]))


if __name__ == "__main__":
    main()
