"""Atom decomposition on the device, one GPU: site ranges (tgap_system_set_site_range) that
partition the atoms give partial energies, forces and virials whose sums equal the whole-system
evaluation, each range's energies are zero outside it, and the e0 of each atom is counted by the
range that owns it; the sharded MD driver with a single rank follows the library's MD step for step.
The exchange step between ranks is tested with gloo ranks on the CPU (test_decomposition_gloo.py)."""
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


def _compute(ctx, system, models, precision):
    import torch
    n, nst = system.n_atoms, system.n_structures
    e = torch.zeros(n, dtype=torch.float64, device="cuda")
    f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    v = torch.zeros(9 * nst, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    system.compute_device(models, precision, e.data_ptr(), f.data_ptr(), v.data_ptr())
    ctx.synchronize()
    return e.cpu().numpy(), f.cpu().numpy().reshape(n, 3), v.cpu().numpy()


def test_site_ranges_sum_to_the_whole_system(ctx, tg, synth):
    from turbogap_b200 import decomposition as dc
    hyp, m = helpers.carbon_model(synth, 100, seed=5)
    pos, box, sp, _ = synth.random_packing(300, 2.5, 1.2, seed=31)
    n = len(pos)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7)
    system.set_e0([-1.25])
    for prec, tol in ((tg.TGAP_FP64, 1e-12), (tg.TGAP_MIXED, 1e-6)):
        e_all, f_all, v_all = _compute(ctx, system, [model], prec)
        e_sum, f_sum, v_sum = np.zeros(n), np.zeros((n, 3)), np.zeros(9)
        for r in range(3):
            beg, end = dc.split_tasks(n, 3, r)
            system.set_site_range(beg, end)
            e, f, v = _compute(ctx, system, [model], prec)
            outside = np.ones(n, bool)
            outside[beg:end] = False
            assert np.all(e[outside] == 0.0)
            e_sum += e
            f_sum += f
            v_sum += v
        system.set_site_range(0)
        assert np.max(np.abs(e_sum - e_all)) < tol
        assert np.max(np.abs(f_sum - f_all)) < tol
        assert np.max(np.abs(v_sum - v_all)) < tol * 100
    system.close()
    model.close()


def test_sharded_md_with_one_rank_follows_the_library_md(ctx, tg, synth):
    from turbogap_b200 import decomposition as dc
    hyp, m = helpers.carbon_model(synth, 100, seed=5)
    pos, box, sp, masses = synth.random_packing(128, 2.5, 1.2, seed=32)
    vel = synth.maxwell_boltzmann(masses, 1000.0, seed=2)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 4.0)
    md = tg.MD(ctx, system, [model], masses, 1.0, rebuild_every=5, precision=tg.TGAP_FP64, use_graph=False)
    md.set_velocities(vel)
    md.run(12)
    ref = md.state()
    md.close()
    system.close()
    system = tg.System(ctx, [(pos, box, sp)], 4.0)
    sh = dc.ShardedMD(ctx, system, [model], masses, 1.0, rebuild_every=5, precision=tg.TGAP_FP64)
    assert sh.range == (0, len(pos))
    sh.set_velocities(vel)
    sh.run(12)
    st = sh.state()
    assert np.max(np.abs(st["positions"] - ref["positions"])) < 1e-9
    assert np.max(np.abs(st["velocities"] - ref["velocities"])) < 1e-9
    assert np.max(np.abs(st["forces"] - ref["forces"])) < 1e-8
    assert abs(st["e_pot"] - ref["e_pot"]) < 1e-8
    system.close()
    model.close()
