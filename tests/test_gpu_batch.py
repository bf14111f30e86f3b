"""Batched 1D two-material shock tubes (m2cg_batch_*) against one reference
run per tube (TimeIntegratorRK2::AdvanceOneTimeStep with the two-material
machinery on an n x 1 x 1 grid), and against this library's own 3D path on
the same tube.

Bars: material IDs identical; states within 1e-10 relative of the reference
(the FP64 two-material bar of the 3D path; the exact Riemann solver's pow()
rounding keeps some interface states from being bit-identical); the per-tube
time identical to the reference's to 1e-12. Tunings (autotuned, fixed,
graph or direct launches) give bit-identical results.
"""
import numpy as np
import pytest

from m2c_b200 import abi, cases
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu

LENS = [100, 137, 211, 160, 333, 101]
STEPS = 20


def _batch_case(seed=5):
    rng = np.random.default_rng(seed)
    lens, mats, VL, VR, _ = cases.tubes(len(LENS), seed=seed)
    return np.array(LENS, np.int32), mats, VL, VR


def test_batch_tubes_match_reference(gpu, ref):
    lens, mats, VL, VR = _batch_case()
    s = cases.tube_scheme()
    b = gpu.Batch(s, lens, mats, VL, VR)
    b.run(STEPS)
    Vg, IDg, tg = b.download()
    assert (b.tube_errors() == 0).all()
    refs = ref.tubes(s, lens, mats, VL, VR, STEPS, range(len(lens)))
    checked = 0
    for t, r in enumerate(refs):
        assert r is not None, f"reference run of tube {t} failed"
        Vr, IDr, t_ref = r
        assert np.array_equal(IDg[t], IDr), t
        assert rel_err(Vg[t], Vr) <= 1e-10, (t, rel_err(Vg[t], Vr))
        assert abs(tg[t] - t_ref) <= 1e-12 * abs(t_ref), (t, tg[t], t_ref)
        checked += 1
    assert checked == len(lens)
    c = b.counters()
    assert c["riemann_calls"] >= STEPS * 2 * len(lens)


def test_batch_matches_3d_path(gpu):
    """Every tube of the batch equals the library's 3D solver run on the
    same n x 1 x 1 grid (which is itself parity-checked against the
    reference)."""
    lens, mats, VL, VR = _batch_case(seed=8)
    s = cases.tube_scheme()
    b = gpu.Batch(s, lens, mats, VL, VR)
    b.run(STEPS)
    Vg, IDg, tg = b.download()
    for t in range(len(lens)):
        g, ls, V, ID, PHI = cases.tube_case(int(lens[t]), VL[t], VR[t])
        sol = gpu.Solver(g, s, [mats[2 * t], mats[2 * t + 1]], ls)
        sol.upload(V, ID, PHI)
        sol.run(STEPS)
        V3, ID3, _ = sol.download()
        sol.close()
        assert np.array_equal(IDg[t], ID3[1, 1, 1:-1].astype(np.int32)), t
        assert rel_err(Vg[t], V3[1, 1, 1:-1]) <= 1e-10, (t, rel_err(Vg[t], V3[1, 1, 1:-1]))


def test_batch_tunings_agree(gpu):
    """Autotuned, fixed-shape, graph and direct-launch runs give the same bits."""
    lens, mats, VL, VR = _batch_case(seed=9)
    s = cases.tube_scheme()
    outs = []
    for kw in (dict(), dict(cells_per_block=128, threads_per_block=128), dict(cells_per_block=512,
               threads_per_block=256, use_graph=0)):
        b = gpu.Batch(s, lens, mats, VL, VR, **kw)
        b.run(7)  # odd count: exercises the single-step graph
        b.run(4)
        outs.append(b.download())
        tun = b.tuning()
        if kw.get("cells_per_block"):
            assert tun["cells_per_block"] == kw["cells_per_block"]
        b.close()
    for V, ID, t in outs[1:]:
        for a, c in zip(V, outs[0][0]):
            assert np.array_equal(a, c)
        for a, c in zip(ID, outs[0][1]):
            assert np.array_equal(a, c)
        assert np.array_equal(t, outs[0][2])
