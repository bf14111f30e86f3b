"""The tubes of the batched-tube workload that fail on the GPU fail in the
reference too.

tests/golden/failed_tubes4.npz holds the 4 tubes (of 4096, seed 11) that
report an error within 200 RK2 steps on the GPU (made by
tests/golden/make_failed_tubes.py): three CheckState failures (a
non-hyperbolic state at the interface) and one whose interface list
overflowed first. Run alone, the reference aborts on every one of them with
"State variables ... violate hyperbolicity" (SpaceOperator.cpp:618-635,
exit(-1)), a few cells from the interface; so these are failures of the
problem, not of the GPU path, and the workload counts them instead of
redrawing them."""
import os
import multiprocessing as mp

import numpy as np
import pytest

from m2c_b200 import abi, cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIXTURE = os.path.join(ROOT, "tests", "golden", "failed_tubes4.npz")


def load_failed():
    d = np.load(FIXTURE)
    fields = [str(f) for f in d["fields"]]
    types = dict(abi.Material._fields_)
    mats = []
    for row in d["mats"]:
        m = abi.Material()
        for f, v in zip(fields, row):
            setattr(m, f, int(v) if types[f] is abi.C.c_int else float(v))
        mats.append(m)
    return d["which"], d["lens"].astype(np.int32), mats, d["VL"], d["VR"]


def _reference_tube(args, path):
    """Child process: one tube through the reference, stdout to path."""
    fd = os.open(path, os.O_WRONLY | os.O_CREAT | os.O_TRUNC)
    os.dup2(fd, 1)
    from oracle import ref
    ref._tube_worker(args)


def test_reference_aborts_on_the_tubes_that_fail_on_the_gpu(ref, tmp_path):
    which, lens, mats, VL, VR = load_failed()
    s = cases.tube_scheme()
    sd = {f: getattr(s, f) for f, _ in abi.Scheme._fields_}
    field = lambda m: tuple(getattr(m, f) for f, _ in abi.Material._fields_)
    crpow = ref.available("crpow")
    ctx = mp.get_context("spawn")
    procs = []
    for q in range(len(which)):
        args = (sd, int(lens[q]), (field(mats[2 * q]), field(mats[2 * q + 1])), tuple(VL[q]), tuple(VR[q]), 200,
                crpow)
        path = str(tmp_path / f"tube{q}.log")
        p = ctx.Process(target=_reference_tube, args=(args, path))
        p.start()
        procs.append((p, path))
    for p, path in procs:
        p.join(300)
        if p.is_alive():
            p.kill()
            p.join()
            pytest.fail("reference tube run did not end within 300 s")
        assert p.exitcode != 0
        assert "violate hyperbolicity" in open(path, errors="replace").read()


@pytest.mark.gpu
def test_gpu_reports_the_failed_tubes_and_stops_them(gpu):
    """The same tubes on the GPU, with two healthy tubes of the workload
    beside them: the four report an error within 200 steps, the healthy
    ones none, and a failed tube stops advancing (its clock stops)."""
    which, lens, mats, VL, VR = load_failed()
    hl, hm, hVL, hVR, _ = cases.tubes(2, seed=3)
    b = gpu.Batch(cases.tube_scheme(), np.concatenate([lens, hl]), list(mats) + list(hm),
                  np.concatenate([VL, hVL]), np.concatenate([VR, hVR]))
    b.time_steps(200, check_errors=False)
    errs = b.tube_errors()
    assert (errs[:4] != 0).all() and (errs[4:] == 0).all()
    _, _, t1 = b.download(check_errors=False)
    b.time_steps(5, check_errors=False)
    _, _, t2 = b.download(check_errors=False)
    assert np.array_equal(t1[:4], t2[:4]) and (t2[4:] > t1[4:]).all()
    b.close()
