"""Autotuner: it finds the tunable launches of an evaluation (descriptor forward and adjoint
sites per CTA and persistent or one-site form, fused GAP kernel chunks), keeps for each the fastest candidate (never slower than
the built-in default, which is among the candidates), and the tuned launches give the same
energies and forces. FP64: only the order of FP64 atomic additions can change (energies 1e-12,
forces and virial 1e-9 relative to their largest entry). Mixed: the fused GAP kernel's chunking
also regroups its FP32 partial sums (1e-6 relative)."""
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


def _eval(system, model, tg, precision, n):
    import torch
    e = torch.zeros(n, dtype=torch.float64, device="cuda")
    f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    v = torch.zeros(9, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    system.compute_device([model], precision, e.data_ptr(), f.data_ptr(), v.data_ptr())
    system.ctx.synchronize()
    return e.cpu().numpy(), f.cpu().numpy(), v.cpu().numpy()


@pytest.mark.parametrize("precision_name", ["TGAP_MIXED", "TGAP_FP64"])
def test_autotune_keeps_results_and_reports_choices(ctx, tg, synth, precision_name):
    precision = getattr(tg, precision_name)
    hyp, m = helpers.carbon_model(synth, 300, seed=11)
    pos, box, sp, _ = synth.random_packing(1000, 2.5, 1.2, seed=12)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7)
    e0, f0, v0 = _eval(system, model, tg, precision, len(pos))
    lines = system.autotune([model], precision, reps=3)
    kinds = {ln.split("/")[0] for ln in lines}
    assert {"soap_fwd", "soap_bwd"} <= kinds, lines
    if precision == tg.TGAP_MIXED:
        assert any(k.startswith("gap_fused") for k in kinds), lines  # single-CTA or CTA-pair form
    for ln in lines:
        parts = ln.split()
        best, best_us, dflt_us = int(parts[1]), float(parts[2]), float(parts[-2])
        assert best >= (0 if parts[0].endswith(("/persist", "/pair")) else 1) and best_us > 0.0
        assert best_us <= dflt_us * (1.0 + 1e-9), ln  # the default is a candidate
    e1, f1, v1 = _eval(system, model, tg, precision, len(pos))
    te, tf = (1e-6, 1e-6) if precision == tg.TGAP_MIXED else (1e-12, 1e-9)
    assert np.max(np.abs(e1 - e0)) <= te * np.max(np.abs(e0)) + 1e-15
    assert np.max(np.abs(f1 - f0)) <= tf * np.max(np.abs(f0))
    assert np.max(np.abs(v1 - v0)) <= tf * np.max(np.abs(v0))
    from turbogap_b200 import native
    native.check(native.lib().tgap_autotune_clear(ctx.h), ctx.h, "clear")
    e2, _, _ = _eval(system, model, tg, precision, len(pos))
    assert np.max(np.abs(e2 - e0)) <= 1e-12 * np.max(np.abs(e0)) + 1e-15  # the default shapes again
    system.close()
    model.close()
