"""The CPU oracle of the warm-start network pinned by central finite
differences (no GPU)."""
import numpy as np

from oracle import mlp_ref


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.3, mlp_ref.NPARAM)
    X = rng.normal(size=(40, 16))
    y = rng.normal(size=40)
    _, g = mlp_ref.loss_grad(p, X, y)
    idx = rng.choice(mlp_ref.NPARAM, 60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (mlp_ref.loss_grad(p + e, X, y)[0] - mlp_ref.loss_grad(p - e, X, y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_parameter_count_matches_header():
    import re
    from pathlib import Path
    hdr = (Path(__file__).resolve().parents[1] / "include" / "m2c_gpu.h").read_text()
    assert int(re.search(r"#define M2CG_MLP_NPARAMS (\d+)", hdr).group(1)) == mlp_ref.NPARAM
