"""Metropolis Monte Carlo with local updates (tgap_mc) against the oracle's full recomputation.

Each proposal's energy change on the device comes from re-evaluating only the sites within the
cutoff of the moved atom; the oracle recomputes the whole structure before and after the move.
FP64: dE within 1e-9 eV, identical decisions (mc_utils.f90:172-180 with the binary32 kB,
get_mc_acceptance min(1, p), accept when p > u), identical final positions. The neighbor skin is
small enough that the lists are rebuilt several times during the run.
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


@pytest.fixture(scope="module")
def carbon(synth):
    return helpers.carbon_model(synth, 200, seed=5)


def _oracle_chain(hyp, models, pos, box, sp, atoms, disp, u, temperature, de_g, acc_g, de_tol):
    """Replays the proposals with full oracle evaluations; returns positions and total energy."""
    p = np.array(pos, dtype=np.float64)
    e_cur = helpers.oracle_structure_eval(hyp, models, p, box, sp, do_forces=False)[0].sum()
    n_border = 0
    for k in range(len(atoms)):
        q = p.copy()
        q[atoms[k]] = q[atoms[k]] + disp[k]
        e_new = helpers.oracle_structure_eval(hyp, models, q, box, sp, do_forces=False)[0].sum()
        de = e_new - e_cur
        assert abs(de - de_g[k]) < de_tol, (k, de, de_g[k])
        pacc = min(1.0, float(np.exp(-de / (KB * temperature))))
        if abs(pacc - u[k]) > 1e-9:
            assert (pacc > u[k]) == bool(acc_g[k]), k
        else:
            n_border += 1
        if acc_g[k]:  # follow the device's chain
            p, e_cur = q, e_new
    return p, e_cur, n_border


def test_mc_fp64_matches_oracle_full_recompute(ctx, tg, synth, carbon):
    hyp, m = carbon
    pos, box, sp, _ = synth.random_packing(64, 2.0, 1.2, seed=70)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.3)
    T = 30.0
    mc = tg.MC(ctx, system, [model], T, precision=tg.TGAP_FP64)
    e0 = mc.state()["e_total"]
    e_o0 = helpers.oracle_structure_eval(hyp, [m], pos, box, sp, do_forces=False)[0].sum()
    assert abs(e0 - e_o0) < 1e-9
    atoms, disp, u = synth.mc_proposals(len(pos), 160, 0.2, seed=71)
    out = mc.run(atoms, disp, u)
    st = mc.state()
    p, e, _ = _oracle_chain(hyp, [m], pos, box, sp, atoms, disp, u, T, out["de"], out["accept"], 1e-9)
    assert 0 < out["accepted"] < len(atoms)
    assert out["accepted"] == int(out["accept"].sum()) == st["accepted"]
    assert st["rebuilds"] >= 2
    assert np.array_equal(st["positions"], p)
    assert abs(st["e_total"] - e) < 1e-9
    # a second run continues the same chain
    atoms2, disp2, u2 = synth.mc_proposals(len(pos), 40, 0.2, seed=72)
    out2 = mc.run(atoms2, disp2, u2)
    p2, e2, _ = _oracle_chain(hyp, [m], p, box, sp, atoms2, disp2, u2, T, out2["de"], out2["accept"], 1e-9)
    st2 = mc.state()
    assert np.array_equal(st2["positions"], p2)
    assert abs(st2["e_total"] - e2) < 1e-9
    mc.close()


def test_mc_two_species_two_models_with_replicas(ctx, tg, synth):
    """SiO2 with one model per centre species; the 9 A cell is smaller than twice the list
    cutoff, so the moved atom's periodic images are in its own list."""
    hyp = synth.sio2_hypers()
    dmin = {("Si", "O"): 1.4, ("O", "O"): 2.2, ("Si", "Si"): 2.5}
    frac = {"Si": 1 / 3, "O": 2 / 3}
    pool = [synth.random_packing(48, 2.2, dmin, frac, seed=50 + k)[:3] for k in range(2)]
    qSi = np.concatenate([helpers.oracle_descriptors(hyp, p, b, s, 1) for p, b, s in pool])
    qO = np.concatenate([helpers.oracle_descriptors(hyp, p, b, s, 2) for p, b, s in pool])
    mSi = synth.gap_model(qSi, 20, seed=1)
    mO = synth.gap_model(qO, 20, seed=2)
    mSi["central_species"], mO["central_species"] = 1, 2
    pos, box, sp, _ = synth.random_packing(48, 2.2, dmin, frac, seed=56)
    models = [tg.Model(ctx, hyp, mm["Qs"], mm["alphas"], 1.0, 4.0, central_species=mm["central_species"])
              for mm in (mSi, mO)]
    system = tg.System(ctx, [(pos, box, sp)], 5.0 + 0.4)
    T = 40.0
    mc = tg.MC(ctx, system, models, T, precision=tg.TGAP_FP64)
    atoms, disp, u = synth.mc_proposals(len(pos), 60, 0.2, seed=57)
    out = mc.run(atoms, disp, u)
    st = mc.state()
    p, e, _ = _oracle_chain(hyp, [mSi, mO], pos, box, sp, atoms, disp, u, T, out["de"], out["accept"], 1e-9)
    assert out["accepted"] > 0
    assert np.array_equal(st["positions"], p)
    assert abs(st["e_total"] - e) < 1e-9
    mc.close()


def test_mc_mixed_tracks_fp64(ctx, tg, synth, carbon):
    hyp, m = carbon
    pos, box, sp, _ = synth.random_packing(96, 2.0, 1.2, seed=73)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    atoms, disp, u = synth.mc_proposals(len(pos), 200, 0.2, seed=74)
    runs = {}
    for prec in (tg.TGAP_FP64, tg.TGAP_MIXED):
        system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.5)
        mc = tg.MC(ctx, system, [model], 30.0, precision=prec)
        runs[prec] = mc.run(atoms, disp, u)
        mc.close()
        system.close()
    d64, d32 = runs[tg.TGAP_FP64]["de"], runs[tg.TGAP_MIXED]["de"]
    a64, a32 = runs[tg.TGAP_FP64]["accept"], runs[tg.TGAP_MIXED]["accept"]
    # identical chains up to the first differing decision; dE agrees to the mixed-path accuracy
    first = np.argmax(a64 != a32) if np.any(a64 != a32) else len(a64)
    assert first > 20
    assert np.max(np.abs(d64[:first] - d32[:first])) < 2e-4


def test_mc_graph_and_eager_agree(ctx, tg, synth, carbon):
    hyp, m = carbon
    pos, box, sp, _ = synth.random_packing(64, 2.0, 1.2, seed=75)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    atoms, disp, u = synth.mc_proposals(len(pos), 100, 0.2, seed=76)
    res = []
    for graph in (True, False):
        system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.3)
        mc = tg.MC(ctx, system, [model], 30.0, precision=tg.TGAP_FP64, use_graph=graph)
        out = mc.run(atoms, disp, u)
        res.append((out, mc.state()))
        mc.close()
        system.close()
    assert np.array_equal(res[0][0]["accept"], res[1][0]["accept"])
    assert np.array_equal(res[0][0]["de"], res[1][0]["de"])
    assert np.array_equal(res[0][1]["positions"], res[1][1]["positions"])


def test_mc_rejects_bad_arguments(ctx, tg, synth, carbon):
    hyp, m = carbon
    pos, box, sp, _ = synth.random_packing(64, 2.0, 1.2, seed=77)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    no_skin = tg.System(ctx, [(pos, box, sp)], 3.7)
    with pytest.raises(tg.TgapError):
        tg.MC(ctx, no_skin, [model], 300.0)
    system = tg.System(ctx, [(pos, box, sp)], 4.0)
    mc = tg.MC(ctx, system, [model], 300.0)
    with pytest.raises(tg.TgapError):
        mc.run(np.array([len(pos)], np.int32), np.zeros((1, 3)), np.zeros(1))
    mc.close()


def _gpu_snapshot_data(ctx, tg, synth, hyp, model, pos, box, sp, n_snap, sigma, seed):
    """(descriptor, per-atom GAP energy) pairs of perturbed copies of a box, from the device (FP64)."""
    import ctypes as C
    import torch
    from turbogap_b200 import native
    rng = np.random.default_rng(seed)
    n = len(pos)
    qs, es = [], []
    for k in range(n_snap):
        p = pos + rng.normal(scale=sigma, size=pos.shape)
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


def test_mc_screen_delayed_acceptance_matches_cpu_chain(ctx, tg, synth, carbon):
    """Delayed acceptance: stage 1 on the learned screen (its dE against the numpy evaluation of
    the same bf16 weights on oracle descriptors), stage 2 on the exact mixed-precision GAP energies
    (against the oracle), same decisions, same final positions."""
    hyp, m = carbon
    pos, box, sp, _ = synth.random_packing(64, 2.0, 1.2, seed=80)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    q_tr, e_tr = _gpu_snapshot_data(ctx, tg, synth, hyp, model, pos, box, sp, 40, 0.08, seed=81)
    w = tg.screen.fit(ctx, q_tr, e_tr, n_pca=32, hidden=64, epochs=40, seed=2)
    T = 30.0
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.4)
    mc = tg.MC(ctx, system, [model], T, precision=tg.TGAP_MIXED)
    mc.set_screen(w)
    atoms, disp, _ = synth.mc_proposals(len(pos), 150, 0.2, seed=82)
    u = np.random.default_rng(83).random((150, 2))
    out = mc.run(atoms, disp, u)
    des_g, stage_g = mc.screen_log(150)
    st = mc.state()
    assert np.all(np.isnan(out["de"][stage_g == 1]))
    assert np.sum(stage_g == 1) > 0 and np.sum(stage_g == 2) > 0
    # CPU replay
    p = np.array(pos, dtype=np.float64)
    es_cur = screen_ref.predict(w, helpers.oracle_descriptors(hyp, p, box, sp))
    e_cur = helpers.oracle_structure_eval(hyp, [m], p, box, sp, do_forces=False)[0].sum()
    for k in range(len(atoms)):
        qn = p.copy()
        qn[atoms[k]] = qn[atoms[k]] + disp[k]
        es_new = screen_ref.predict(w, helpers.oracle_descriptors(hyp, qn, box, sp))
        des = es_new.sum() - es_cur.sum()
        assert abs(des - des_g[k]) < 2e-4, (k, des, des_g[k])
        p1 = min(1.0, float(np.exp(-des / (KB * T))))
        if abs(p1 - u[k, 0]) > 1e-3:
            assert (stage_g[k] == 2) == (p1 > u[k, 0]), k
        if stage_g[k] == 2:
            e_new = helpers.oracle_structure_eval(hyp, [m], qn, box, sp, do_forces=False)[0].sum()
            de = e_new - e_cur
            assert abs(de - out["de"][k]) < 2e-4, (k, de, out["de"][k])
            p2 = min(1.0, float(np.exp(-(out["de"][k] - des_g[k]) / (KB * T))))
            assert (p2 > u[k, 1]) == bool(out["accept"][k]), k
            if out["accept"][k]:
                p, es_cur, e_cur = qn, es_new, e_new
    assert np.array_equal(st["positions"], p)
    mc.close()


def test_mc_screen_fallback_to_plain_when_acceptance_collapses(ctx, tg, synth, carbon):
    """A screen whose energies are noise (large random output weights): the exact stage rejects
    what it lets through, so over the first window the confirmation rate collapses and the driver
    switches to plain GAP MC. Before the switch every decision follows the delayed-acceptance
    rule, after it the plain rule on the first deviate of each pair."""
    hyp, m = carbon
    pos, box, sp, _ = synth.random_packing(64, 2.0, 1.2, seed=90)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    dim = tg.synth.soap_dim(hyp)
    rng = np.random.default_rng(91)
    K, H = 16, 32
    bad = dict(mean=np.zeros(dim), pca=rng.normal(size=(K, dim)), w1=rng.normal(size=(H, K)), b1=np.zeros(H),
               w2=rng.normal(size=(H, H)) * 0.3, b2=np.zeros(H), w3=rng.normal(size=H) * 0.5, b3=0.0)
    T = 300.0
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.4)
    mc = tg.MC(ctx, system, [model], T, precision=tg.TGAP_MIXED)
    mc.set_screen(bad)
    mc.screen_fallback(window=128, min_confirm=0.2, min_pass=0.0)
    n = 512
    atoms, disp, _ = synth.mc_proposals(len(pos), n, 0.2, seed=92)
    u = rng.random((n, 2))
    out = mc.run(atoms, disp, u)
    des, stage = mc.screen_log(n)
    s = mc.screen_stats()
    assert not s["active"] and s["fallbacks"] == 1
    k_fb = s["judged"]
    assert 128 <= k_fb < n  # checked between graph launches, after the first full window
    assert s["passed"] >= 32
    for k in range(n):
        if k < k_fb:
            if stage[k] == 1:
                assert not out["accept"][k]
                continue
            p2 = min(1.0, float(np.exp(-(out["de"][k] - des[k]) / (KB * T))))
            assert (p2 > u[k, 1]) == bool(out["accept"][k]), k
        else:
            assert stage[k] == 2 and np.isfinite(out["de"][k])
            p = min(1.0, float(np.exp(-out["de"][k] / (KB * T))))
            assert (p > u[k, 0]) == bool(out["accept"][k]), k
    mc.close()
    system.close()


def test_mc_rejects_moves_beyond_the_skin(ctx, tg, synth, carbon):
    """A displacement at or above the neighbor skin could bring in a pair no list holds, even
    right after a rebuild: the run refuses it before any work, and the driver stays usable."""
    hyp, m = carbon
    pos, box, sp, _ = synth.random_packing(64, 2.0, 1.2, seed=93)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.3)
    mc = tg.MC(ctx, system, [model], 300.0, precision=tg.TGAP_MIXED)
    atoms = np.array([3, 5], np.int32)
    disp = np.array([[0.1, 0.0, 0.0], [0.0, 0.35, 0.0]])
    with pytest.raises(Exception):
        mc.run(atoms, disp, np.array([0.5, 0.5]))
    r = mc.run(atoms[:1], disp[:1], np.array([0.5]))
    assert r["accepted"] in (0, 1)
    mc.close()
    system.close()


def test_mc_speculative_batch_matches_one_at_a_time(ctx, tg, synth, carbon):
    """Batches of 1, 5 and 16 proposals give the same decisions and the same final positions
    (bitwise), and the same dE to rounding: a batch settles proposals past a deferred one, so a list
    rebuild can fall between other moves than one at a time, and the rebuilt lists sum the FP64
    descriptors in another order. On a box several cutoffs wide a batch settles more than one
    proposal on average."""
    hyp, m = carbon
    pos, box, sp, _ = synth.random_packing(1000, 2.0, 1.2, seed=60)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    atoms, disp, u = synth.mc_proposals(len(pos), 300, 0.2, seed=61)
    runs = {}
    for B in (1, 5, 16):
        system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.5)
        mc = tg.MC(ctx, system, [model], 2000.0, precision=tg.TGAP_FP64)
        mc.set_batch(B)
        out = mc.run(atoms, disp, u)
        runs[B] = (out, mc.state(), mc.batch_stats())
        mc.close()
        system.close()
    ref_out, ref_st, ref_bs = runs[1]
    assert ref_bs["settled"] == 300 and ref_bs["batches"] >= 300
    for B in (5, 16):
        out, st, bs = runs[B]
        assert np.array_equal(out["accept"], ref_out["accept"]), B
        assert np.max(np.abs(out["de"] - ref_out["de"])) < 1e-12, B
        assert np.array_equal(st["positions"], ref_st["positions"]), B
        assert st["accepted"] == ref_st["accepted"]
        assert bs["settled"] == 300
        assert bs["batches"] < 0.75 * 300, (B, bs)


def test_screened_batch_equals_one_at_a_time(ctx, tg, synth, carbon):
    """Delayed acceptance inside the speculative batch (12 slots judged by the screen from the
    state before the batch, exact GAP row tiles of rejected slots skipped, settlement in proposal
    order past deferred slots) makes the same decisions and ends at the same positions as one
    proposal at a time."""
    hyp, m = carbon
    pos, box, sp, _ = synth.random_packing(64, 2.0, 1.2, seed=110)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    q_tr, e_tr = _gpu_snapshot_data(ctx, tg, synth, hyp, model, pos, box, sp, 40, 0.08, seed=111)
    w = tg.screen.fit(ctx, q_tr, e_tr, n_pca=32, hidden=64, epochs=40, seed=2)
    n = 600
    atoms, disp, _ = synth.mc_proposals(len(pos), n, 0.25, seed=112)
    u = np.random.default_rng(113).random((n, 2))
    runs = {}
    for slots in (1, 12):
        system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.4)
        mc = tg.MC(ctx, system, [model], 30.0, precision=tg.TGAP_MIXED)
        mc.set_batch(slots)
        mc.set_screen(w)
        mc.screen_fallback(window=1 << 40)
        out = mc.run(atoms, disp, u)
        des, stage = mc.screen_log(n)
        runs[slots] = (out, des, stage, mc.state(), mc.batch_stats())
        mc.close()
        system.close()
    (o1, d1, s1, st1, _), (o12, d12, s12, st12, bs) = runs[1], runs[12]
    assert np.sum(s1 == 1) > 20 and np.sum(s1 == 2) > 20  # both stages decide proposals
    assert np.array_equal(s1, s12)
    assert np.array_equal(o1["accept"], o12["accept"])
    assert np.max(np.abs(d1 - d12)) < 1e-5  # same screen energies (FP32 rows, FP64 sums)
    ex = s1 == 2
    # exact dE to the mixed path's rounding: a list rebuild can fall between other moves when the
    # batch settles past a deferred slot, and the FP32 descriptors then sum in another order
    assert np.max(np.abs(o1["de"][ex] - o12["de"][ex])) < 1e-6
    assert np.array_equal(st1["positions"], st12["positions"])
    assert bs["settled"] == n  # every proposal was settled by the speculative batch
    model.close()


def test_screened_and_plain_chains_sample_the_same_energies(ctx, tg, synth, carbon):
    """Delayed acceptance leaves the target distribution unchanged: 24 independent replicas of
    plain GAP MC and 24 of screened MC, all started from one equilibrated state with independent
    proposal streams, give final total energies whose two-sample Kolmogorov-Smirnov test does
    not reject equality (p > 1e-3). The replicas are independent, so the test needs no
    decorrelation of a single chain."""
    from scipy import stats
    hyp, m = carbon
    pos, box, sp, _ = synth.random_packing(64, 2.0, 1.2, seed=120)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    T, radius = 300.0, 0.3
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.4)
    mc = tg.MC(ctx, system, [model], T, precision=tg.TGAP_MIXED)
    a, d, u = synth.mc_proposals(len(pos), 4000, radius, seed=121)
    mc.run(a, d, u, logs=False)
    start = mc.state()["positions"]
    mc.close()
    system.close()
    q_tr, e_tr = _gpu_snapshot_data(ctx, tg, synth, hyp, model, start, box, sp, 40, 0.06, seed=122)
    w = tg.screen.fit(ctx, q_tr, e_tr, n_pca=32, hidden=64, epochs=40, seed=4)
    finals = {"plain": [], "screened": []}
    passed = []
    for rep in range(24):
        for name in ("plain", "screened"):
            system = tg.System(ctx, [(start, box, sp)], 3.7 + 0.4)
            mc = tg.MC(ctx, system, [model], T, precision=tg.TGAP_MIXED)
            seed = 1000 + 2 * rep + (name == "screened")
            atoms, disp, u1 = synth.mc_proposals(len(pos), 1500, radius, seed=seed)
            if name == "screened":
                mc.set_screen(w)
                mc.screen_fallback(window=1 << 40)
                u = np.stack([u1, np.random.default_rng(seed + 7).random(len(u1))], axis=1)
                mc.run(atoms, disp, u, logs=False)
                s = mc.screen_stats()
                passed.append(s["passed"] / max(1, s["judged"]))
            else:
                mc.run(atoms, disp, u1, logs=False)
            finals[name].append(mc.state()["e_total"])
            mc.close()
            system.close()
    ks = stats.ks_2samp(finals["plain"], finals["screened"])
    print("KS", ks, "mean plain/screened", np.mean(finals["plain"]), np.mean(finals["screened"]),
          "screen pass rate", np.mean(passed))
    assert np.mean(passed) < 0.99  # the screen did judge proposals on its own
    assert ks.pvalue > 1e-3, ks
    model.close()
