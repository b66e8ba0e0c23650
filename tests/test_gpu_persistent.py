"""Persistent work-queue form of the descriptor kernels: on a batch of cells of uneven atom and
neighbor counts (atom counts 8..400, densities 1.5..3.5 g/cm^3, triclinic strain) evaluated in one
launch, the warps take sites from a queue until it runs dry. Each site is still computed by one
warp, so the descriptors are the same as in the one-site-per-warp form; what can differ is the order
of atomic additions (FP64 forces and virial; in the mixed path also the FP32 dE/dq the fused GAP
kernel accumulates), with the tolerances of the autotuner test. The persistent form agrees with the
oracle on two cells."""
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
    c.autotune_clear()
    c.close()


def _eval(system, model, precision, n, nst):
    import torch
    e = torch.zeros(n, dtype=torch.float64, device="cuda")
    f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    v = torch.zeros(9 * nst, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    system.compute_device([model], precision, e.data_ptr(), f.data_ptr(), v.data_ptr())
    system.ctx.synchronize()
    return e.cpu().numpy(), f.cpu().numpy().reshape(n, 3), v.cpu().numpy().reshape(nst, 3, 3)


@pytest.mark.parametrize("precision_name", ["TGAP_MIXED", "TGAP_FP64"])
def test_persistent_matches_one_site_per_warp(ctx, tg, synth, precision_name):
    precision = getattr(tg, precision_name)
    hyp, m = helpers.carbon_model(synth, 300, seed=21)
    rng = np.random.default_rng(77)
    nst = 40
    sizes = np.exp(rng.uniform(np.log(8), np.log(400), nst)).astype(int)
    dens = rng.uniform(1.5, 3.5, nst)
    structs = [synth.random_packing(int(n), float(d), 1.1, seed=500 + k, strain=0.05)[:3]
               for k, (n, d) in enumerate(zip(sizes, dens))]
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, structs, 3.7)
    n = int(sizes.sum())
    ctx.autotune_clear()
    e1, f1, v1 = _eval(system, model, precision, n, nst)      # default: persistent
    ctx.autotune_set("*/persist", 0)
    e0, f0, v0 = _eval(system, model, precision, n, nst)      # one site per warp
    ctx.autotune_set("*/persist", 1)
    e2, f2, v2 = _eval(system, model, precision, n, nst)
    ctx.autotune_clear()
    te, tf = (1e-6, 1e-6) if precision == tg.TGAP_MIXED else (1e-12, 1e-9)
    for e, f, v in ((e1, f1, v1), (e2, f2, v2)):
        assert np.max(np.abs(e - e0)) <= te * np.abs(e0).max() + 1e-15
        assert np.max(np.abs(f - f0)) <= tf * np.abs(f0).max()
        assert np.max(np.abs(v - v0)) <= tf * np.abs(v0).max()
    if precision == tg.TGAP_FP64:
        off = np.concatenate([[0], np.cumsum(sizes)])
        for b in (int(np.argmin(sizes)), int(np.argmax(dens * (sizes < 120)))):
            pos, box, sp = structs[b]
            e_o, f_o, v_o = helpers.oracle_structure_eval(hyp, [m], pos, box, sp)
            assert np.max(np.abs(e1[off[b]:off[b + 1]] - e_o)) < 1e-10, b
            assert np.max(np.abs(f1[off[b]:off[b + 1]] - f_o)) < 1e-8, b
            assert np.max(np.abs(v1[b] - v_o)) < 1e-8, b
    system.close()
    model.close()


def test_fused_gap_single_cta_and_cta_pair_forms_agree(ctx, tg, synth):
    """The fused GAP kernel in its single-CTA form and in its CTA-pair form (tcgen05 cta_group::2,
    each CTA of a 2-CTA cluster loading half of every sparse slice) give the same energies and
    forces to FP32 accumulation order, on a system with an odd number of 128-row tiles (600 sites:
    5 tiles, the last pair's second tile is padding)."""
    hyp, m = helpers.carbon_model(synth, 300, seed=13)
    pos, box, sp, _ = synth.random_packing(600, 2.5, 1.2, seed=14)
    n = len(pos)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7)
    out = {}
    for form in (0, 1):
        ctx.autotune_set("*/pair", form)
        out[form] = _eval(system, model, tg.TGAP_MIXED, n, 1)
    ctx.autotune_clear()
    (e0, f0, v0), (e1, f1, v1) = out[0], out[1]
    assert np.max(np.abs(e1 - e0)) <= 1e-6 * np.abs(e0).max() + 1e-15
    assert np.max(np.abs(f1 - f0)) <= 1e-6 * np.abs(f0).max()
    assert np.max(np.abs(v1 - v0)) <= 1e-6 * np.abs(v0).max()
    e_d, f_d, _ = _eval(system, model, tg.TGAP_FP64, n, 1)
    assert np.max(np.abs(e1 - e_d)) <= 1e-5  # eV per atom, far inside the 0.5 meV/atom bar
    system.close()
    model.close()
