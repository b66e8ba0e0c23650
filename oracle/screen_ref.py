"""CPU reference of the Monte Carlo screen network (numpy). Test infrastructure: only tests/ import
it, as the checker of the device trainer (tgap_screen_grad / tgap_screen_train) and of the device
screen evaluation (tgap_screen_eval and the driver's stage-1 energies).

The screen is the project's own addition (the reference's MC, src/mc/mc_interface.f90:183-449,
has no surrogate); there is no reference algorithm to follow, so this file restates the network
and its training exactly as the device code defines them:
    z = P (q - mean)                  P: n_pca x dim
    out = w3 . silu(W2 silu(W1 z + b1) + b2) + b3
    loss = (1/B) sum_r (out_r - t_r)^2 over a batch of B rows
    Adam: m = b1 m + (1 - b1) g, v = b2 v + (1 - b2) g^2,
          w -= lr (m / (1 - b1^s)) / (sqrt(v / (1 - b2^s)) + eps),  b1 0.9, b2 0.999, eps 1e-8
    epoch e learning rate lr (1 + cos(pi e / epochs)) / 2
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
    """Screen energies of descriptor rows q (n, dim) in the device's arithmetic: bf16-rounded
    matrices, FP32 sums."""
    q = np.asarray(q, dtype=np.float32)
    z = (q - w["mean"].astype(np.float32)) @ bf16_round(w["pca"]).T
    h1 = _silu(z @ bf16_round(w["w1"]).T + w["b1"].astype(np.float32))
    h2 = _silu(h1 @ bf16_round(w["w2"]).T + w["b2"].astype(np.float32))
    return (h2 @ bf16_round(w["w3"]) + np.float32(w["b3"])).astype(np.float64)


def loss_and_grad(p, z, t, dtype=np.float64):
    """Loss (1/n) sum (out - t)^2 over all rows and its gradients; p holds w1 (H x K), b1, w2
    (H x H), b2, w3 (H), b3 (scalar)."""
    z = np.asarray(z, dtype)
    t = np.asarray(t, dtype)
    P = {k: np.asarray(v, dtype) for k, v in p.items()}
    a1 = z @ P["w1"].T + P["b1"]
    s1 = 1.0 / (1.0 + np.exp(-a1))
    h1 = a1 * s1
    a2 = h1 @ P["w2"].T + P["b2"]
    s2 = 1.0 / (1.0 + np.exp(-a2))
    h2 = a2 * s2
    out = h2 @ P["w3"] + P["b3"]
    err = out - t
    g_out = (2.0 / len(t)) * err
    g = {"w3": h2.T @ g_out, "b3": g_out.sum()}
    g_a2 = np.outer(g_out, P["w3"]) * (s2 * (1.0 + a2 * (1.0 - s2)))
    g["w2"] = g_a2.T @ h1
    g["b2"] = g_a2.sum(0)
    g_a1 = (g_a2 @ P["w2"]) * (s1 * (1.0 + a1 * (1.0 - s1)))
    g["w1"] = g_a1.T @ z
    g["b1"] = g_a1.sum(0)
    return float(np.mean(err ** 2)), g


def adam_train(p, z, t, order, epochs, batch, lr):
    """The device trainer's minibatch Adam in FP32: epoch e visits rows order[e] in order."""
    p = {k: np.array(v, np.float32) for k, v in p.items()}
    p["b3"] = np.float32(p["b3"])
    m = {k: np.zeros_like(v) for k, v in p.items()}
    v = {k: np.zeros_like(x) for k, x in p.items()}
    z = np.asarray(z, np.float32)
    t = np.asarray(t, np.float32)
    n = len(t)
    step = 0
    for ep in range(epochs):
        lr_ep = np.float32(lr * 0.5 * (1.0 + np.cos(np.pi * ep / epochs)))
        for s in range(0, n, batch):
            idx = order[ep][s:s + batch]
            _, g = loss_and_grad(p, z[idx], t[idx], np.float32)
            step += 1
            bc1 = np.float32(1.0 - 0.9 ** step)
            bc2 = np.float32(1.0 - 0.999 ** step)
            for k in p:
                gk = np.asarray(g[k], np.float32)
                m[k] = np.float32(0.9) * m[k] + np.float32(0.1) * gk
                v[k] = np.float32(0.999) * v[k] + np.float32(0.001) * gk * gk
                p[k] = (p[k] - lr_ep * (m[k] / bc1) / (np.sqrt(v[k] / bc2) + np.float32(1e-8))).astype(np.float32)
    return p
