"""Learned screen of the Monte Carlo driver: fitting and evaluation.

The screen predicts per-atom GAP energies from the normalised SOAP vector:
    z = P (q - mean)                  P: n_pca x dim (PCA directions, scaled to unit variance)
    e = w3 . silu(W2 silu(W1 z + b1) + b2) + b3
`fit` computes the PCA on the host (an SVD of at most 20,000 centred rows, a one-off
preprocessing step), then trains the network on the device with the library's own forward and
backward kernels and Adam (tgap_screen_train) on the mean squared error of standardised targets;
the target scale is folded into (w3, b3) at the end. `predict` runs the device kernel the Monte
Carlo driver uses (tgap_screen_eval: bf16 weights, FP32 sums).
"""
import ctypes as C

import numpy as np

from . import native


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def init_params(n_pca, hidden, seed=0):
    """He-normal W1 and W2, zero biases, N(0, 1/hidden) w3: the starting point of `fit`."""
    rng = np.random.default_rng(seed)
    return {"w1": (rng.normal(size=(hidden, n_pca)) * np.sqrt(2.0 / n_pca)).astype(np.float32),
            "b1": np.zeros(hidden, np.float32),
            "w2": (rng.normal(size=(hidden, hidden)) * np.sqrt(2.0 / hidden)).astype(np.float32),
            "b2": np.zeros(hidden, np.float32),
            "w3": (rng.normal(size=hidden) * np.sqrt(1.0 / hidden)).astype(np.float32),
            "b3": np.float32(0.0)}


def grad(ctx, p, z, t):
    """Loss (1/n) sum (out - t)^2 of the network part on rows z (n, n_pca) and its gradients,
    computed on the device as one batch (n <= 16384)."""
    z, t = _f32(z), _f32(t)
    n, K = z.shape
    H = len(p["b1"])
    w = {k: _f32(p[k]) for k in ("w1", "b1", "w2", "b2", "w3")}
    g = {k: np.zeros_like(v) for k, v in w.items()}
    gb3 = np.zeros(1, np.float32)
    loss = C.c_double()
    native.check(native.lib().tgap_screen_grad(
        ctx.h, n, K, H, native.ptr(z), native.ptr(t), *[native.ptr(w[k]) for k in ("w1", "b1", "w2", "b2", "w3")],
        float(p["b3"]), *[native.ptr(g[k]) for k in ("w1", "b1", "w2", "b2", "w3")], native.ptr(gb3),
        C.byref(loss)), ctx.h, "tgap_screen_grad")
    g["b3"] = float(gb3[0])
    return loss.value, g


def train(ctx, p, z, t, order, epochs, batch, lr):
    """Minibatch Adam on the device from the starting point p; order: (epochs, n) row visits.
    Returns the trained parameters and each epoch's mean squared error."""
    z, t = _f32(z), _f32(t)
    n, K = z.shape
    H = len(p["b1"])
    order = np.ascontiguousarray(order, dtype=np.int32)
    if order.shape != (epochs, n):
        raise ValueError("order must be (epochs, n)")
    w = {k: _f32(p[k]).copy() for k in ("w1", "b1", "w2", "b2", "w3")}
    b3 = np.array([p["b3"]], np.float32)
    log = np.zeros(epochs)
    native.check(native.lib().tgap_screen_train(
        ctx.h, n, K, H, native.ptr(z), native.ptr(t), int(epochs), int(batch), float(lr), native.ptr(order),
        *[native.ptr(w[k]) for k in ("w1", "b1", "w2", "b2", "w3")], native.ptr(b3), native.ptr(log)),
        ctx.h, "tgap_screen_train")
    w["b3"] = np.float32(b3[0])
    return w, log


def fit(ctx, q, e, n_pca=64, hidden=128, epochs=40, batch=512, lr=3e-3, seed=0, return_log=False):
    """Fits the screen to per-atom energies e (n,) of descriptors q (n, dim). Returns the weights
    in the layout tgap_mc_set_screen takes (float32; the device rounds the matrices to bf16)."""
    rng = np.random.default_rng(seed)
    q = np.asarray(q, dtype=np.float64)
    e = np.asarray(e, dtype=np.float64)
    mean = q.mean(0)
    X = q - mean
    sub = X[rng.choice(len(X), size=min(len(X), 20000), replace=False)]
    _, _, vt = np.linalg.svd(sub, full_matrices=False)
    P = vt[:n_pca]
    Z = X @ P.T
    zs = Z.std(0) + 1e-12
    P = P / zs[:, None]
    Z = (Z / zs).astype(np.float32)
    e_mu, e_sd = e.mean(), e.std() + 1e-30
    t = ((e - e_mu) / e_sd).astype(np.float32)
    p0 = init_params(n_pca, hidden, seed=int(rng.integers(1 << 31)))
    order = np.stack([rng.permutation(len(Z)) for _ in range(epochs)]).astype(np.int32)
    p, log = train(ctx, p0, Z, t, order, epochs, batch, lr)
    w = {"mean": mean.astype(np.float32), "pca": P.astype(np.float32), "w1": p["w1"], "b1": p["b1"],
         "w2": p["w2"], "b2": p["b2"], "w3": (p["w3"] * e_sd).astype(np.float32),
         "b3": float(p["b3"] * e_sd + e_mu)}
    return (w, log * e_sd ** 2) if return_log else w


def predict(ctx, w, q):
    """Screen energies of descriptor rows q (n, dim), evaluated on the device."""
    q = _f32(q)
    n, dim = q.shape
    pca = _f32(w["pca"])
    n_pca = pca.shape[0]
    hidden = len(w["b1"])
    keep = [_f32(w[k]) for k in ("mean", "pca", "w1", "b1", "w2", "b2", "w3")]
    out = np.zeros(n)
    native.check(native.lib().tgap_screen_eval(ctx.h, n, dim, n_pca, hidden, *[native.ptr(a) for a in keep],
                                               float(w["b3"]), native.ptr(q), native.ptr(out)),
                 ctx.h, "tgap_screen_eval")
    return out
