"""Training data and training of the learned Riemann warm start.

The network learns the star pressure of two-material interface Riemann
problems drawn from the batched-tube state distribution (stiffened-gas
pairs with gamma in [1.2, 7] and p_inf 0 w.p. 1/4 else log-uniform in
1e6..1e9 Pa; densities log-uniform in 1..1000 kg/m^3, pressures log-uniform
in 1e4..1e9 Pa, velocities uniform in +-200 m/s). Targets come from the
library's own exact solver (m2cg_riemann_batch_pairs, the restated
ExactRiemannSolverBase::ComputeRiemannSolution); training runs on the GPU
through m2cg_mlp_train.
"""
import numpy as np

from . import abi, gpu


def sample_problems(n, seed):
    """n seeded problems: (materials [2n] as a MATERIAL_DTYPE table, VL, VR, dirs)."""
    rng = np.random.default_rng(seed)
    gam = rng.uniform(1.2, 7.0, 2 * n)
    zero = rng.uniform(size=2 * n) < 0.25
    pinf = np.where(zero, 0.0, 10.0 ** rng.uniform(6.0, 9.0, 2 * n))
    mats = abi.material_table(gam, pinf)
    VL = np.zeros((n, 5))
    VR = np.zeros((n, 5))
    for V in (VL, VR):
        V[:, 0] = 10.0 ** rng.uniform(0.0, 3.0, n)
        V[:, 1] = rng.uniform(-200.0, 200.0, n)
        V[:, 4] = 10.0 ** rng.uniform(4.0, 9.0, n)
    dirs = np.zeros((n, 3))
    dirs[:, 0] = 1.0
    return mats, VL, VR, dirs


def sample_cluster_problems(n, seed):
    """n seeded interface problems of the bubble-cluster kind: water
    (stiffened gas gamma 6.12, p_inf 3.43e8 Pa, density log-uniform in
    990..1400 kg/m^3) against air (gamma 1.4, density log-uniform in
    1..300 kg/m^3), on either side; both sides near one base state (pressure
    log-uniform in 1e5..3e9 Pa, velocity uniform in +-700 m/s) with relative
    pressure and velocity departures log-uniform in 1e-4..0.5, so that the
    set runs from near-acoustic problems (most of the cluster's interface
    faces) to strong waves (the collapse)."""
    rng = np.random.default_rng(seed)
    water_left = rng.uniform(size=n) < 0.5
    gam = np.empty(2 * n)
    pinf = np.empty(2 * n)
    gam[0::2] = np.where(water_left, 6.12, 1.4)
    gam[1::2] = np.where(water_left, 1.4, 6.12)
    pinf[0::2] = np.where(water_left, 3.43e8, 0.0)
    pinf[1::2] = np.where(water_left, 0.0, 3.43e8)
    mats = abi.material_table(gam, pinf)
    p0 = 10.0 ** rng.uniform(5.0, np.log10(3e9), n)
    u0 = rng.uniform(-700.0, 700.0, n)
    rw = 10.0 ** rng.uniform(np.log10(990.0), np.log10(1400.0), n)
    ra = 10.0 ** rng.uniform(0.0, np.log10(300.0), n)
    VL = np.zeros((n, 5))
    VR = np.zeros((n, 5))
    VL[:, 0] = np.where(water_left, rw, ra)
    VR[:, 0] = np.where(water_left, ra, rw)
    for V in (VL, VR):
        dp = 10.0 ** rng.uniform(-4.0, np.log10(0.5), n) * rng.choice([-1.0, 1.0], n)
        du = 10.0 ** rng.uniform(-4.0, np.log10(0.5), n) * rng.choice([-1.0, 1.0], n)
        V[:, 4] = p0 * (1.0 + dp)
        V[:, 1] = u0 + du * np.maximum(np.abs(u0), 10.0)
    dirs = np.zeros((n, 3))
    dirs[:, 0] = 1.0
    return mats, VL, VR, dirs


def solve(s, mats, VL, VR, dirs, warm=None, chunk=250_000):
    """Exact solves in chunks; returns dict of arrays (Vs, id, Vsm, Vsp, iters, evals, err)."""
    out = {k: [] for k in ("Vs", "id", "Vsm", "Vsp", "iters", "evals", "err")}
    for a in range(0, len(VL), chunk):
        b = min(len(VL), a + chunk)
        r = gpu.riemann_batch_pairs(s, mats[2 * a:2 * b], VL[a:b], VR[a:b], dirs[a:b],
                                    None if warm is None else warm[a:b])
        for k, v in zip(out, r):
            out[k].append(v)
    return {k: np.concatenate(v) for k, v in out.items()}


def training_set(n, seed, s=None, cluster_fraction=0.25):
    """Features X [m, 16] and targets y = log((p* + S) / B) (B, S: the base
    and shift the features return; B is the shifted acoustic estimate) of
    the solvable problems (solver OK, features valid) among n samples, a
    fraction cluster_fraction of them of the bubble-cluster kind."""
    s = s or abi.scheme()
    nc = int(round(n * cluster_fraction))
    mats, VL, VR, dirs = sample_problems(n - nc, seed)
    if nc:
        parts = [(mats, VL, VR, dirs), sample_cluster_problems(nc, seed + 1)]
        mats = np.concatenate([q[0] for q in parts])
        VL, VR, dirs = (np.concatenate([q[k] for q in parts]) for k in (1, 2, 3))
    r = solve(s, mats, VL, VR, dirs)
    X, P, valid = gpu.mlp_features_pairs(mats, VL, VR, dirs)
    q = r["Vsm"][:, 4] + P[:, 1]
    keep = (r["err"] == 0) & (q > 0) & (valid != 0)
    y = np.log(q[keep] / P[keep, 0]).astype(np.float32)
    return X[keep], y, keep.mean()


def train(n=2_000_000, steps=6000, batch=8192, lr=2e-3, seed=0, s=None):
    """Generate n problems, solve them, train a network on the GPU. Returns
    (Mlp, info)."""
    X, y, frac = training_set(n, seed, s)
    net = gpu.Mlp(seed=seed)
    loss = net.train(X, y, steps=steps, batch=batch, lr=lr, seed=seed)
    return net, {"samples": int(len(y)), "kept_fraction": float(frac), "final_loss": loss}


def save(net, path):
    p, nrm = net.params()
    np.savez(path, params=p, norm=nrm)


def load(path):
    d = np.load(path)
    net = gpu.Mlp()
    net.set_params(d["params"], d["norm"])
    return net


if __name__ == "__main__":
    import argparse
    import os
    ap = argparse.ArgumentParser(description="train the learned Riemann warm start on the GPU")
    ap.add_argument("--n", type=int, default=2_000_000, help="sampled problems (solved on the GPU for targets)")
    ap.add_argument("--steps", type=int, default=20_000)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--seed", type=int, default=21)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                                                   "warmstart_mlp.npz"))
    a = ap.parse_args()
    net, info = train(n=a.n, steps=a.steps, batch=a.batch, lr=a.lr, seed=a.seed)
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    save(net, a.out)
    print({**info, "out": a.out})
