"""Learned screen of the Monte Carlo driver: fitting on the host (numpy) and a numpy restatement
of the device evaluation (bf16-rounded weights, FP32 arithmetic).

The screen predicts per-atom GAP energies from the normalised SOAP vector:
    z = P (q - mean)                  P: n_pca x dim (PCA directions, scaled to unit variance)
    e = w3 . silu(W2 silu(W1 z + b1) + b2) + b3
It is trained on (q, e) pairs of GAP-evaluated configurations with Adam on the mean squared error
of standardised targets; the target scale is folded into (w3, b3) at the end.
"""
import numpy as np


def bf16_round(x):
    """Round-to-nearest-even to bfloat16, returned as float32 (the device stores bf16 weights)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(x.shape)


def _silu(x):
    return x / (1.0 + np.exp(-x))


def predict(w, q):
    """Screen energies of descriptor rows q (n, dim), as the device evaluates them."""
    q = np.asarray(q, dtype=np.float32)
    z = (q - w["mean"].astype(np.float32)) @ bf16_round(w["pca"]).T
    h1 = _silu(z @ bf16_round(w["w1"]).T + w["b1"].astype(np.float32))
    h2 = _silu(h1 @ bf16_round(w["w2"]).T + w["b2"].astype(np.float32))
    return (h2 @ bf16_round(w["w3"]) + np.float32(w["b3"])).astype(np.float64)


def fit(q, e, n_pca=64, hidden=128, epochs=40, batch=512, lr=3e-3, seed=0):
    """Fits the screen to per-atom energies e (n,) of descriptors q (n, dim). Returns the weights
    (float32 arrays; `predict` and the device round the matrices to bf16)."""
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

    def init(o, i):
        return (rng.normal(size=(o, i)) * np.sqrt(2.0 / i)).astype(np.float32)

    params = {"w1": init(hidden, n_pca), "b1": np.zeros(hidden, np.float32), "w2": init(hidden, hidden),
              "b2": np.zeros(hidden, np.float32), "w3": (rng.normal(size=hidden) * np.sqrt(1.0 / hidden)).astype(np.float32),
              "b3": np.zeros(1, np.float32)}
    m = {k: np.zeros_like(v) for k, v in params.items()}
    v = {k: np.zeros_like(v) for k, v in params.items()}
    b1_, b2_, eps = 0.9, 0.999, 1e-8
    step = 0
    n = len(Z)
    for ep in range(epochs):
        perm = rng.permutation(n)
        lr_ep = lr * 0.5 * (1.0 + np.cos(np.pi * ep / epochs))
        for s in range(0, n, batch):
            idx = perm[s:s + batch]
            x, y = Z[idx], t[idx]
            a1 = x @ params["w1"].T + params["b1"]
            s1 = 1.0 / (1.0 + np.exp(-a1))
            h1 = a1 * s1
            a2 = h1 @ params["w2"].T + params["b2"]
            s2 = 1.0 / (1.0 + np.exp(-a2))
            h2 = a2 * s2
            out = h2 @ params["w3"] + params["b3"][0]
            g_out = (2.0 / len(idx)) * (out - y)
            grads = {"w3": h2.T @ g_out, "b3": np.array([g_out.sum()], np.float32)}
            g_h2 = np.outer(g_out, params["w3"])
            g_a2 = g_h2 * (s2 * (1.0 + a2 * (1.0 - s2)))
            grads["w2"] = g_a2.T @ h1
            grads["b2"] = g_a2.sum(0)
            g_h1 = g_a2 @ params["w2"]
            g_a1 = g_h1 * (s1 * (1.0 + a1 * (1.0 - s1)))
            grads["w1"] = g_a1.T @ x
            grads["b1"] = g_a1.sum(0)
            step += 1
            for k in params:
                m[k] = b1_ * m[k] + (1 - b1_) * grads[k]
                v[k] = b2_ * v[k] + (1 - b2_) * grads[k] ** 2
                mh = m[k] / (1 - b1_ ** step)
                vh = v[k] / (1 - b2_ ** step)
                params[k] = (params[k] - lr_ep * mh / (np.sqrt(vh) + eps)).astype(np.float32)
    return {"mean": mean.astype(np.float32), "pca": P.astype(np.float32), "w1": params["w1"], "b1": params["b1"],
            "w2": params["w2"], "b2": params["b2"], "w3": (params["w3"] * e_sd).astype(np.float32),
            "b3": float(params["b3"][0] * e_sd + e_mu)}
