"""The host-buffer entry tgap_calculate_gap_soap (the calculate_gap_soap surface) against the
device-pointer path on the same positions: a rebuild of existing lists runs on the device and its
pair count comes back with the results; without a rebuild the descriptor forward writes the pair
geometry itself. Each call must equal a fresh system (host-built lists, separate geometry pass)
evaluated with tgap_compute: bitwise in FP64 up to the order of FP64 atomic additions, and within
the FP32 accumulation order in the mixed form. A list that outgrows the arrays reserved for it is
rebuilt on the host and the call repeated, with the same results."""
import numpy as np
import pytest

import helpers

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(tg):
    import torch
    assert torch.cuda.is_available()
    c = tg.Context(0)
    yield c
    c.close()


def _fresh(ctx, tg, x, box, sp, model, precision):
    """Energies and forces of a new system at x (lists built on the host) via tgap_compute."""
    import torch
    system = tg.System(ctx, [(x, box, sp)], 3.7 + 0.3)
    n = len(x)
    e = torch.zeros(n, dtype=torch.float64, device="cuda")
    f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    v = torch.zeros(9, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    system.compute_device([model], precision, e.data_ptr(), f.data_ptr(), v.data_ptr())
    ctx.synchronize()
    out = e.cpu().numpy(), f.cpu().numpy().reshape(n, 3), system.n_pairs
    system.close()
    return out


@pytest.mark.parametrize("precision_name", ["TGAP_FP64", "TGAP_MIXED"])
def test_host_entry_steps_match_fresh_systems(ctx, tg, synth, precision_name):
    precision = getattr(tg, precision_name)
    hyp, m = helpers.carbon_model(synth, 200, seed=17)
    pos, box, sp, _ = synth.random_packing(300, 2.5, 1.2, seed=18)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.3)
    rng = np.random.default_rng(19)
    x = pos.copy()
    te, tf = (1e-12, 1e-10) if precision == tg.TGAP_FP64 else (1e-7, 1e-6)
    for k in range(6):
        x = x + rng.normal(scale=0.05, size=x.shape)
        rebuild = k % 2 == 0
        e, f, _ = system.calculate_gap_soap([model], precision, x, rebuild=rebuild)
        e_r, f_r, n_r = _fresh(ctx, tg, x, box, sp, model, precision)
        assert np.max(np.abs(e - e_r)) <= te * max(1.0, np.abs(e_r).max()), k
        assert np.max(np.abs(f - f_r)) <= tf * max(1.0, np.abs(f_r).max()), k
        if rebuild:
            assert system.n_pairs == n_r, k
    system.close()
    model.close()


def test_host_entry_repeats_a_call_whose_lists_outgrew_their_arrays(ctx, tg, synth):
    """Atoms drawn halfway towards the box centre: the device-side rebuild finds more pairs than the
    arrays hold, so the call rebuilds on the host and repeats; the results equal a fresh system's and
    no device check is left behind."""
    hyp, m = helpers.carbon_model(synth, 200, seed=17)
    pos, box, sp, _ = synth.random_packing(128, 2.5, 1.2, seed=20)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.3)
    n0 = system.n_pairs
    c = 0.5 * np.asarray(box).sum(axis=0)
    x = c + 0.5 * (pos - c)
    e, f, _ = system.calculate_gap_soap([model], tg.TGAP_FP64, x, rebuild=True)
    e_r, f_r, n_r = _fresh(ctx, tg, x, box, sp, model, tg.TGAP_FP64)
    assert n_r > 1.25 * n0 + 256  # beyond the reserved arrays
    assert system.n_pairs == n_r
    assert np.max(np.abs(e - e_r)) <= 1e-12 * max(1.0, np.abs(e_r).max())
    assert np.max(np.abs(f - f_r)) <= 1e-10 * max(1.0, np.abs(f_r).max())
    ctx.synchronize()  # no device check pending
    system.close()
    model.close()


def test_registered_arrays_give_the_staged_results(ctx, tg, synth):
    """Positions, energies, forces and virial registered with tgap_host_register are copied to and
    from directly (in the captured call graphs too); each call equals the same call through the
    staging buffers to the order of the mixed path's atomic additions."""
    import ctypes as C
    from turbogap_b200 import native
    L = native.lib()
    hyp, m = helpers.carbon_model(synth, 200, seed=17)
    pos, box, sp, _ = synth.random_packing(300, 2.5, 1.2, seed=21)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    n = len(pos)
    arr = (C.c_void_p * 1)(model.h.value)
    runs = []
    for registered in (False, True):
        system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.3)
        x, e, f, v = pos.copy(), np.zeros(n), np.zeros((n, 3)), np.zeros(9)
        if registered:
            for a in (x, e, f, v):
                ctx.host_register(a)
        out = []
        rng = np.random.default_rng(22)
        for k in range(6):
            x += rng.normal(scale=0.03, size=x.shape)
            st = L.tgap_calculate_gap_soap(ctx.h, system.h, 1, arr, tg.TGAP_MIXED, native.ptr(x), int(k % 2 == 0),
                                           native.ptr(e), native.ptr(f), native.ptr(v))
            native.check(st, ctx.h, "calculate")
            out.append((e.copy(), f.copy(), v.copy()))
        if registered:
            for a in (x, e, f, v):
                ctx.host_unregister(a)
        runs.append(out)
        system.close()
    for (e0, f0, v0), (e1, f1, v1) in zip(*runs):
        assert np.array_equal(e0, e1) or np.max(np.abs(e0 - e1)) <= 1e-7 * np.abs(e0).max()
        assert np.max(np.abs(f0 - f1)) <= 1e-6 * max(1.0, np.abs(f0).max())
        assert np.max(np.abs(v0 - v1)) <= 1e-6 * max(1.0, np.abs(v0).max())
    model.close()


def test_call_graphs_follow_e0_and_site_range_changes(ctx, tg, synth):
    """The host-buffer entry replays captured graphs from its third call on; e0 (tgap_system_set_e0)
    and the site range (tgap_system_set_site_range) set afterwards still apply: each atom's energy
    moves by its e0, and a range leaves the energies outside it at zero and its own unchanged."""
    hyp, m = helpers.carbon_model(synth, 200, seed=17)
    pos, box, sp, _ = synth.random_packing(256, 2.5, 1.2, seed=23)
    n = len(pos)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.3)
    for _ in range(3):  # eager, captured, replayed
        e, f, _ = system.calculate_gap_soap([model], tg.TGAP_FP64, pos, rebuild=False)
    system.set_e0([-1.25])
    e1, f1, _ = system.calculate_gap_soap([model], tg.TGAP_FP64, pos, rebuild=False)
    assert np.max(np.abs(e1 - (e - 1.25))) < 1e-12
    assert np.max(np.abs(f1 - f)) < 1e-12
    system.set_site_range(0, n // 2)
    e2, _, _ = system.calculate_gap_soap([model], tg.TGAP_FP64, pos, rebuild=False)
    assert np.all(e2[n // 2:] == 0.0)
    assert np.max(np.abs(e2[:n // 2] - e1[:n // 2])) < 1e-12
    system.set_site_range(0)
    e3, _, _ = system.calculate_gap_soap([model], tg.TGAP_FP64, pos, rebuild=False)
    assert np.max(np.abs(e3 - e1)) < 1e-12
    system.close()
    model.close()


def test_call_graphs_follow_staging_growth(ctx, tg, synth):
    """A larger system on the same context grows the pinned staging buffers that a smaller system's
    captured call graph reads and writes; the smaller system's next call runs with the new buffers
    and gives the results it gave before, and the larger one equals a fresh system."""
    hyp, m = helpers.carbon_model(synth, 200, seed=17)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    pa, ba, sa, _ = synth.random_packing(128, 2.5, 1.2, seed=24)
    pb, bb, sb, _ = synth.random_packing(640, 2.5, 1.2, seed=25)
    sys_a = tg.System(ctx, [(pa, ba, sa)], 3.7 + 0.3)
    sys_b = tg.System(ctx, [(pb, bb, sb)], 3.7 + 0.3)
    for _ in range(3):  # eager, captured, replayed
        ea, fa, _ = sys_a.calculate_gap_soap([model], tg.TGAP_FP64, pa, rebuild=False)
    eb, fb, _ = sys_b.calculate_gap_soap([model], tg.TGAP_FP64, pb, rebuild=False)
    for _ in range(3):
        ea2, fa2, _ = sys_a.calculate_gap_soap([model], tg.TGAP_FP64, pa, rebuild=False)
        # the same to the order of the FP64 force atomics
        assert np.max(np.abs(ea2 - ea)) <= 1e-12 * max(1.0, np.abs(ea).max())
        assert np.max(np.abs(fa2 - fa)) <= 1e-12 * max(1.0, np.abs(fa).max())
    eb_r, fb_r, _ = _fresh(ctx, tg, pb, bb, sb, model, tg.TGAP_FP64)
    assert np.max(np.abs(eb - eb_r)) <= 1e-12 * max(1.0, np.abs(eb_r).max())
    assert np.max(np.abs(fb - fb_r)) <= 1e-10 * max(1.0, np.abs(fb_r).max())
    sys_a.close()
    sys_b.close()
    model.close()
