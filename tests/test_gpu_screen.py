"""The Monte Carlo screen's network on the device: gradients, Adam training and evaluation against
the numpy reference (oracle/screen_ref.py), fitting through the public API, and what the trained
screen buys the Monte Carlo driver over plain GAP MC.

Tolerances: gradients and loss are FP32 sums against an FP64 reference (max error over a tensor
within 1e-4 of its largest entry); after a few Adam steps the FP32 weights agree within
1e-5 + 1e-3 |w|; the evaluation, bf16 weights and FP32 sums in both, within 1e-5 of the energies'
scale.
"""
import numpy as np
import pytest

import helpers
import screen_ref

pytestmark = pytest.mark.gpu

KB = float(np.float32(8.617333262e-5))


@pytest.fixture(scope="module")
def ctx(tg):
    import torch
    assert torch.cuda.is_available()
    c = tg.Context(0)
    yield c
    c.close()


def _params(rng, K, H, scale=1.0):
    return {"w1": (rng.normal(size=(H, K)) * np.sqrt(2.0 / K) * scale).astype(np.float32),
            "b1": (rng.normal(size=H) * 0.1).astype(np.float32),
            "w2": (rng.normal(size=(H, H)) * np.sqrt(2.0 / H) * scale).astype(np.float32),
            "b2": (rng.normal(size=H) * 0.1).astype(np.float32),
            "w3": (rng.normal(size=H) * np.sqrt(1.0 / H)).astype(np.float32),
            "b3": np.float32(0.3)}


@pytest.mark.parametrize("n,K,H", [(1000, 16, 32), (517, 64, 128)])
def test_screen_gradients_match_reference(ctx, tg, n, K, H):
    rng = np.random.default_rng(K + H)
    z = rng.normal(size=(n, K)).astype(np.float32)
    t = rng.normal(size=n).astype(np.float32)
    p = _params(rng, K, H)
    loss, g = tg.screen.grad(ctx, p, z, t)
    loss_ref, g_ref = screen_ref.loss_and_grad(p, z, t)
    assert abs(loss - loss_ref) < 1e-5 * loss_ref
    for k in ("w1", "b1", "w2", "b2", "w3", "b3"):
        ref = np.asarray(g_ref[k])
        err = np.max(np.abs(np.asarray(g[k], np.float64) - ref))
        assert err <= 1e-4 * np.max(np.abs(ref)), (k, err, np.max(np.abs(ref)))


def test_screen_adam_training_matches_reference(ctx, tg):
    """Three epochs of minibatch Adam (batch 128 over 600 rows: a short last batch each epoch)."""
    rng = np.random.default_rng(3)
    n, K, H, epochs = 600, 16, 32, 3
    z = rng.normal(size=(n, K)).astype(np.float32)
    t = np.tanh(z[:, 0] + 0.5 * z[:, 1] * z[:, 2]).astype(np.float32)
    p0 = _params(rng, K, H)
    order = np.stack([rng.permutation(n) for _ in range(epochs)])
    p, log = tg.screen.train(ctx, p0, z, t, order, epochs, 128, 3e-3)
    p_ref = screen_ref.adam_train(p0, z, t, order, epochs, 128, 3e-3)
    for k in ("w1", "b1", "w2", "b2", "w3", "b3"):
        a, b = np.asarray(p[k], np.float64), np.asarray(p_ref[k], np.float64)
        assert np.all(np.abs(a - b) <= 1e-5 + 1e-3 * np.abs(b)), (k, np.max(np.abs(a - b)))
    # the logged loss falls and the first epoch's matches the reference's start
    assert log[-1] < log[0]
    l0, _ = screen_ref.loss_and_grad(p0, z, t)
    assert log[0] < 1.05 * l0


def test_screen_evaluation_matches_reference(ctx, tg):
    rng = np.random.default_rng(5)
    dim, K, H, n = 324, 64, 128, 1003
    q = np.abs(rng.normal(size=(n, dim)))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    p = _params(rng, K, H)
    w = dict(mean=q.mean(0).astype(np.float32), pca=(rng.normal(size=(K, dim)) * 3).astype(np.float32), **p)
    w["b3"] = float(p["b3"])
    e = tg.screen.predict(ctx, w, q)
    e_ref = screen_ref.predict(w, q)
    assert np.max(np.abs(e - e_ref)) < 1e-5 * max(1.0, np.max(np.abs(e_ref)))


def test_screen_fit_learns_a_smooth_target(ctx, tg):
    """PCA on the host, network trained on the device: a smooth function of the leading
    directions is learned to a small fraction of its spread."""
    rng = np.random.default_rng(0)
    q = rng.normal(size=(4000, 40)) * np.r_[np.full(4, 4.0), np.ones(36)]  # leading directions dominate
    q /= np.linalg.norm(q, axis=1)[:, None]
    e = np.sin(3 * q[:, 0]) + 0.5 * q[:, 1] ** 2
    w, log = tg.screen.fit(ctx, q, e, n_pca=16, hidden=32, epochs=60, seed=1, return_log=True)
    pred = tg.screen.predict(ctx, w, q)
    assert np.sqrt(np.mean((pred - e) ** 2)) < 0.2 * e.std()
    assert log[-1] < 0.1 * log[0]


def _descriptors_and_energies(ctx, tg, model, snaps, box, sp):
    """(descriptor, per-atom GAP energy) rows of the given position snapshots (device, FP64)."""
    import ctypes as C
    import torch
    from turbogap_b200 import native
    n = len(sp)
    qs, es = [], []
    for p in snaps:
        system = tg.System(ctx, [(p, box, sp)], 3.7)
        e = torch.zeros(n, dtype=torch.float64, device="cuda")
        f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
        v = torch.zeros(9, dtype=torch.float64, device="cuda")
        q = torch.zeros((n, model.dim), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        system.compute_device([model], tg.TGAP_FP64, e.data_ptr(), f.data_ptr(), v.data_ptr())
        nr = C.c_int(0)
        native.check(native.lib().tgap_descriptors(ctx.h, system.h, model.h, 0, C.c_void_p(q.data_ptr()),
                                                   C.byref(nr)), ctx.h, "descriptors")
        ctx.synchronize()
        qs.append(q.cpu().numpy())
        es.append(e.cpu().numpy())
        system.close()
    return np.concatenate(qs), np.concatenate(es)


def test_trained_screen_saves_exact_evaluations(ctx, tg, synth):
    """What the trained network buys. A plain GAP MC chain is equilibrated at a low temperature,
    the screen is trained on snapshots of that chain, and three chains then run the same
    proposals from its end: plain GAP MC (one exact evaluation per proposal), the trained screen,
    and the untrained starting network on the same PCA. The figure of merit of delayed
    acceptance is accepted moves per exact GAP evaluation: the trained screen raises it above
    plain GAP MC's (it settles proposals that would be rejected without the exact energies), the
    untrained one does not. The chain's exactness is checked move by move in test_gpu_mc.py."""
    hyp, m = helpers.carbon_model(synth, 200, seed=5)
    pos, box, sp, _ = synth.random_packing(64, 2.0, 1.2, seed=95)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    T, radius = 2.0, 0.3  # moves below the 0.4 A skin
    rng = np.random.default_rng(96)
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.4)
    mc = tg.MC(ctx, system, [model], T, precision=tg.TGAP_MIXED)
    a, d, u = synth.mc_proposals(len(pos), 3000, radius, seed=97)
    mc.run(a, d, u, logs=False)  # equilibration
    snaps = []
    for k in range(200):
        a, d, u = synth.mc_proposals(len(pos), 10, radius, seed=1000 + k)
        mc.run(a, d, u, logs=False)
        snaps.append(mc.state()["positions"])
    start = mc.state()["positions"]
    mc.close()
    system.close()
    q_tr, e_tr = _descriptors_and_energies(ctx, tg, model, snaps, box, sp)
    w = tg.screen.fit(ctx, q_tr, e_tr, n_pca=32, hidden=64, epochs=60, seed=3)
    n = 1000
    atoms, disp, u1 = synth.mc_proposals(len(pos), n, radius, seed=98)
    u = np.stack([u1, rng.random(n)], 1)
    p0 = tg.screen.init_params(32, 64, seed=3)
    untrained = dict(w, **{k: p0[k] for k in ("w1", "b1", "w2", "b2")}, w3=p0["w3"] * float(np.std(e_tr)), b3=0.0)
    results = {}
    for name, weights in (("plain", None), ("trained", w), ("untrained", untrained)):
        system = tg.System(ctx, [(start, box, sp)], 3.7 + 0.4)
        mc = tg.MC(ctx, system, [model], T, precision=tg.TGAP_MIXED)
        if weights is not None:
            mc.set_screen(weights)
            mc.screen_fallback(window=1 << 40)  # never: measure the screen as it is
            r = mc.run(atoms, disp, u, logs=False)
            _, stage = mc.screen_log(n)
            exact = float(np.mean(stage == 2))
        else:
            r = mc.run(atoms, disp, u1, logs=False)
            exact = 1.0
        results[name] = dict(acc=r["accepted"] / n, exact=exact, acc_per_exact=r["accepted"] / n / exact)
        mc.close()
        system.close()
    print("screen gain:", results)
    plain, tr, un = results["plain"], results["trained"], results["untrained"]
    assert tr["exact"] < 0.9, results  # the trained screen settles proposals on its own
    assert tr["acc_per_exact"] > 1.2 * plain["acc_per_exact"], results
    assert un["acc_per_exact"] < tr["acc_per_exact"], results
