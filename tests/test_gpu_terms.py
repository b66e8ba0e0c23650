"""Resident pair and triplet terms (tgap_terms): the 2b, core_pot and 3b terms on a system's own
neighbor list added to the outputs, against the sum of the oracle's routines on the same list
(1e-10 eV/atom, 1e-8 eV/A), and an NVE run of a full production-style model (soap_turbo + 2b +
3b + core_pot) whose energy stays conserved."""
import numpy as np
import pytest

import helpers
import oracle_lib as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(tg):
    import torch
    assert torch.cuda.is_available()
    c = tg.Context(0)
    yield c
    c.close()


def _sio2(synth, n=192, seed=47):
    return synth.random_packing(n, 2.2, {("Si", "O"): 1.4, ("O", "O"): 2.2, ("Si", "Si"): 2.5},
                                {"Si": 1 / 3, "O": 2 / 3}, seed=seed)[:3]


def _terms_spec(rng):
    M = 10
    t2 = dict(alphas=rng.normal(size=M) * 0.05, cutoff=rng.uniform(0.5, 1.0, M), Qs=np.linspace(1.3, 3.8, M),
              rcut=4.0, buffer=0.6, delta=1.1, sigma=0.4, e0=0.01)
    x = np.linspace(0.8, 3.5, 30)
    V = 5.0 * np.exp(-2.0 * x) * (1.0 - x / 3.5) ** 2
    y2 = orc.spline_second_derivatives(x, V, -12.0, 0.0)
    Q3 = np.stack([rng.uniform(3.0, 6.5, M), rng.uniform(0.0, 2.0, M), rng.uniform(2.0, 5.5, M)], axis=1)
    t3 = dict(alphas=rng.normal(size=M) * 0.02, cutoff=rng.uniform(0.5, 1.0, M), Qs=Q3, rcut=3.5, buffer=0.5,
              delta=0.9, sigma=np.array([1.0, 1.0, 1.2]), e0=0.005)
    return t2, (x, V, -12.0, 0.0, y2), t3


def _device_terms(tg, ctx, t2, cp, t3):
    T = tg.Terms(ctx)
    T.add_2b(1, 2, t2["alphas"], t2["cutoff"], t2["Qs"], t2["rcut"], t2["buffer"], t2["delta"], t2["sigma"], t2["e0"])
    T.add_core_pot(1, 2, *cp)
    T.add_3b(2, 1, 2, t3["alphas"], t3["cutoff"], t3["Qs"], t3["rcut"], t3["sigma"], t3["buffer"], t3["delta"],
             t3["e0"], "exp")
    return T


def test_resident_terms_match_oracle(ctx, tg, synth):
    import torch
    pos, box, sp = _sio2(synth)
    n = len(pos)
    t2, cp, t3 = _terms_spec(np.random.default_rng(1))
    system = tg.System(ctx, [(pos, box, sp)], 4.0)
    T = _device_terms(tg, ctx, t2, cp, t3)
    e = torch.zeros(n, dtype=torch.float64, device="cuda")
    f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    v = torch.zeros(9, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    T.compute_device(system, e.data_ptr(), f.data_ptr(), v.data_ptr())
    ctx.synchronize()
    nb = orc.build_neighbors(pos, n, *box, 4.0, sp, False)
    e2, f2, v2 = orc.get_2b_energy_and_forces(nb, sp, 1, 2, **t2)
    ec, fc, vc = orc.get_core_pot_energy_and_forces(nb, sp, 1, 2, *cp)
    e3, f3, v3 = orc.get_3b_energy_and_forces(nb, sp, 2, 1, 2, **t3)
    assert np.max(np.abs(e.cpu().numpy() - (e2 + ec + e3))) < 1e-10
    assert np.max(np.abs(f.cpu().numpy().reshape(n, 3) - (f2 + fc + f3))) < 1e-8
    assert np.max(np.abs(v.cpu().numpy().reshape(3, 3, order="F") - (v2 + vc + v3))) < 1e-8
    T.close()
    system.close()


def test_md_with_soap_and_terms_conserves_energy(ctx, tg, synth):
    """NVE with a SiO2 SOAP model per centre species plus 2b, 3b and core_pot terms (FP64, 0.5 fs,
    40 steps): the total energy stays within 2e-3 of the starting kinetic energy (a force that
    disagreed with its energy would drift by a sizeable fraction of it)."""
    hyp = synth.sio2_hypers()
    pos, box, sp = _sio2(synth, 192, seed=49)
    q1 = helpers.oracle_descriptors(hyp, pos, box, sp, 1)
    q2 = helpers.oracle_descriptors(hyp, pos, box, sp, 2)
    mSi, mO = synth.gap_model(q1, 20, seed=3), synth.gap_model(q2, 20, seed=4)
    models = [tg.Model(ctx, hyp, mSi["Qs"], mSi["alphas"], 1.0, 4.0, central_species=1),
              tg.Model(ctx, hyp, mO["Qs"], mO["alphas"], 1.0, 4.0, central_species=2)]
    t2, cp, t3 = _terms_spec(np.random.default_rng(2))
    system = tg.System(ctx, [(pos, box, sp)], 5.0 + 0.3)
    T = _device_terms(tg, ctx, t2, cp, t3)
    masses = np.where(np.asarray(sp) == 1, 28.085, 15.999)
    md = tg.MD(ctx, system, models, masses, 0.5, rebuild_every=10, precision=tg.TGAP_FP64)
    md.set_terms(T)
    rng = np.random.default_rng(5)
    vel = rng.normal(size=(len(pos), 3)) * 0.002
    md.set_velocities(vel)
    energies, kin = [], []
    for _ in range(20):
        md.run(2)
        st = md.state()
        energies.append(st["e_pot"] + st["e_kin"])
        kin.append(st["e_kin"])
    energies = np.array(energies)
    drift = np.max(np.abs(energies - energies[0]))
    assert drift < 2e-3 * kin[0], (drift, kin[0], energies)
    assert abs(energies[-1] - energies[0]) < 2e-3 * kin[0]
    md.close()
    T.close()
    system.close()
