"""Generate tests/golden/failed_tubes4.npz (needs a GPU): the tubes of the
batched-tube workload (4096 tubes, seed 11, tubes whose initial interface
problem fails redrawn) that report an error within 200 RK2 steps on the
GPU. The file holds their index in the batch, length, material pair (the
m2cg_material fields, by name), and left/right states. The reference aborts
on each of them too (tests/test_failed_tubes.py).

    python tests/golden/make_failed_tubes.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def main():
    from m2c_b200 import abi, cases, gpu
    s = cases.tube_scheme()
    lens, mats, VL, VR, _ = cases.tubes(4096, seed=11, reject=gpu.tube_rejects(s))
    b = gpu.Batch(s, lens, mats, VL, VR)
    b.time_steps(200, check_errors=False)
    errs = b.tube_errors()
    b.close()
    bad = np.nonzero(errs)[0]
    fields = [f for f, _ in abi.Material._fields_]
    M = np.array([[getattr(mats[2 * t + m], f) for f in fields] for t in bad for m in (0, 1)])
    out = os.path.join(ROOT, "tests", "golden", "failed_tubes4.npz")
    np.savez(out, which=bad, lens=lens[bad], mats=M, VL=VL[bad], VR=VR[bad], fields=np.array(fields))
    print(f"{len(bad)} failed tubes: {bad.tolist()} codes {errs[bad].tolist()} -> {out}")


if __name__ == "__main__":
    main()
