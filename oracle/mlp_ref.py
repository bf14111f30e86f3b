"""CPU oracle of the learned warm start's network (TEST INFRASTRUCTURE ONLY).

A float64 numpy restatement of the 16 -> 64 -> 64 -> 64 -> 1 tanh network
with the parameter layout of include/m2c_gpu.h (W1[64][16] b1 W2[64][64] b2
W3[64][64] b3 w4[64] b4) and its mean-squared-error loss, used to check the
GPU training kernels' gradients and the BF16 inference. The network has no
counterpart in the reference; its backward pass here is the textbook
chain rule, itself pinned by finite differences in tests/test_mlp_oracle.py.
"""
import numpy as np

NIN, NH = 16, 64
SIZES = [("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NH, NH)), ("b3", (NH,)),
         ("w4", (NH,)), ("b4", (1,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    p = np.asarray(p, np.float64)
    out, o = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = p[o:o + k].reshape(shape)
        o += k
    return out


def forward(p, X):
    """Network output for normalised inputs X [n, 16]; returns (out, cache)."""
    w = unpack(p)
    X = np.asarray(X, np.float64)
    h1 = np.tanh(X @ w["W1"].T + w["b1"])
    h2 = np.tanh(h1 @ w["W2"].T + w["b2"])
    h3 = np.tanh(h2 @ w["W3"].T + w["b3"])
    out = h3 @ w["w4"] + w["b4"][0]
    return out, (X, h1, h2, h3, w)


def loss_grad(p, X, y):
    """Mean squared error and its gradient (flat, parameter layout order)."""
    out, (X, h1, h2, h3, w) = forward(p, X)
    n = len(out)
    e = out - np.asarray(y, np.float64)
    loss = float(np.mean(e * e))
    dout = 2.0 * e / n
    g = {}
    g["w4"] = h3.T @ dout
    g["b4"] = np.array([dout.sum()])
    g3 = np.outer(dout, w["w4"]) * (1 - h3 ** 2)
    g["W3"] = g3.T @ h2
    g["b3"] = g3.sum(0)
    g2 = (g3 @ w["W3"]) * (1 - h2 ** 2)
    g["W2"] = g2.T @ h1
    g["b2"] = g2.sum(0)
    g1 = (g2 @ w["W2"]) * (1 - h1 ** 2)
    g["W1"] = g1.T @ X
    g["b1"] = g1.sum(0)
    flat = np.concatenate([g[name].ravel() for name, _ in SIZES])
    return loss, flat


def predict(p, norm, X):
    """Output in target units for raw features X (normalisation blob
    xmean[16] xstd[16] ymean ystd)."""
    norm = np.asarray(norm, np.float64)
    Xn = (np.asarray(X, np.float64) - norm[:NIN]) / norm[NIN:2 * NIN]
    out, _ = forward(p, Xn)
    return out * norm[2 * NIN + 1] + norm[2 * NIN]
