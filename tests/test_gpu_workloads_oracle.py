"""The single-point and two-species workloads checked against the CPU oracle at their real model
sizes, and the per-species isolated-atom energies (calculate_e0) on the resident path.

* predict: 216-atom carbon, 3x3x3 cubic diamond (a = 3.567 A) with every atom displaced by
  uniform +-0.15 A per axis; SOAP poly3 n_max = l_max = 8, rcut 3.7 / 3.2 A, sigma 0.5 A; GAP
  zeta = 4, delta = 1 eV, 1000 sparse points = normalised descriptors of random atoms of 10
  further perturbed supercells, alphas ~ N(0, 1e-6), e0 = 0. FP64 energies, forces and virial
  against the oracle (1e-10 eV/atom, 1e-8 eV/A), mixed precision against FP64 (0.5 meV/atom,
  5 meV/A RMSE).
* two species: amorphous SiO2 (Si:O = 1:2) at 2.2 g/cm^3 with the scale workload's descriptor
  (species-resolved n_max 8 + 8, l_max 6, rcut 5.0 / 4.5 A: 952 components) and model sizes (one
  GAP per centre species with 4,000 sparse points drawn from further boxes), on a 1,536-atom box
  so the oracle's materialised dq/dr stays near a gigabyte; same bars.
* e0: energies of tgap_compute, the host-buffer calculate_gap_soap entry, the MD potential energy
  and the MC state include each atom's species e0, as turbogap adds calculate_e0's energies to
  the total (turbogap_main.f90:993-994).
"""
import ctypes as C

import numpy as np
import pytest

import helpers
import oracle_lib as orc

pytestmark = pytest.mark.gpu

E_TOL = 1e-10   # eV / atom
F_TOL = 1e-8    # eV / A
V_TOL = 1e-8    # eV
E_RMSE = 0.5e-3  # eV / atom, mixed vs FP64
F_RMSE = 5e-3    # eV / A

SIO2_DMIN = {("Si", "O"): 1.4, ("O", "O"): 2.2, ("Si", "Si"): 2.5}
SIO2_FRAC = {"Si": 1 / 3, "O": 2 / 3}


@pytest.fixture(scope="module")
def ctx(tg):
    import torch
    assert torch.cuda.is_available()
    c = tg.Context(0)
    yield c
    c.close()


def _compute(ctx, system, models, precision, n, nst=1):
    import torch
    e = torch.zeros(n, dtype=torch.float64, device="cuda")
    f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    v = torch.zeros(9 * nst, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    system.compute_device(models, precision, e.data_ptr(), f.data_ptr(), v.data_ptr())
    ctx.synchronize()
    return e.cpu().numpy(), f.cpu().numpy().reshape(n, 3), v.cpu().numpy().reshape(nst, 3, 3)


def _device_descriptors(tg, ctx, hyp, structs, central_species):
    """FP64 descriptors of the given centre species over seeded boxes, computed on the device."""
    import torch
    from turbogap_b200 import native
    out = []
    dummy = tg.Model(ctx, hyp, np.zeros((1, tg.synth.soap_dim(hyp))), np.zeros(1), central_species=central_species)
    for pos, box, sp in structs:
        system = tg.System(ctx, [(pos, box, sp)], max(hyp["rcut_hard"]))
        q = torch.zeros((len(sp), dummy.dim), dtype=torch.float64, device="cuda")
        nr = C.c_int(0)
        torch.cuda.synchronize()
        native.check(native.lib().tgap_descriptors(ctx.h, system.h, dummy.h, 0, C.c_void_p(q.data_ptr()),
                                                   C.byref(nr)), ctx.h, "descriptors")
        ctx.synchronize()
        out.append(q[:nr.value].cpu().numpy())
        system.close()
    dummy.close()
    return np.concatenate(out)


def test_predict_216_atom_diamond_1000_sparse_matches_oracle(ctx, tg, synth):
    hyp, m = helpers.carbon_model(synth, 1000, seed=21, n_pool_structs=10, reps=3)
    assert len(m["alphas"]) == 1000 and m["Qs"].shape == (1000, 324)
    pos, box, sp = synth.diamond_supercell(3, a0=3.567, noise=0.15, seed=20)
    n = len(pos)
    assert n == 216
    e_o, f_o, v_o = helpers.oracle_structure_eval(hyp, [m], pos, box, sp)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7)
    e64, f64, v64 = _compute(ctx, system, [model], tg.TGAP_FP64, n)
    assert np.max(np.abs(e64 - e_o)) < E_TOL
    assert np.max(np.abs(f64 - f_o)) < F_TOL
    assert np.max(np.abs(v64[0] - v_o)) < V_TOL
    # the reference call surface (get_gap_soap on the oracle's own list) agrees as well
    nb = orc.build_neighbors(pos, n, *box, 3.7, sp, False)
    e_g, f_g, v_g = ctx.get_gap_soap(hyp, n, nb, sp, 0, m["alphas"], m["Qs"], 1.0, 4.0)
    assert np.max(np.abs(e_g - e_o)) < E_TOL
    assert np.max(np.abs(f_g - f_o)) < F_TOL
    e32, f32, _ = _compute(ctx, system, [model], tg.TGAP_MIXED, n)
    assert np.sqrt(np.mean((e32 - e64) ** 2)) < E_RMSE
    assert np.sqrt(np.mean((f32 - f64) ** 2)) < F_RMSE
    system.close()
    model.close()


def test_sio2_full_model_size_matches_oracle(ctx, tg, synth):
    hyp = synth.sio2_hypers()
    assert synth.soap_dim(hyp) == 952
    pool_structs = [synth.random_packing(4096, 2.2, SIO2_DMIN, SIO2_FRAC, seed=600 + k)[:3] for k in range(3)]
    mods_np = []
    for cs, seed in ((1, 61), (2, 62)):
        pool = _device_descriptors(tg, ctx, hyp, pool_structs, cs)
        mm = synth.gap_model(pool, 4000, seed=seed)
        mm["central_species"] = cs
        mods_np.append(mm)
    pos, box, sp, _ = synth.random_packing(1536, 2.2, SIO2_DMIN, SIO2_FRAC, seed=65)
    n = len(pos)
    e_o, f_o, v_o = helpers.oracle_structure_eval(hyp, mods_np, pos, box, sp)
    models = [tg.Model(ctx, hyp, mm["Qs"], mm["alphas"], 1.0, 4.0, central_species=mm["central_species"])
              for mm in mods_np]
    system = tg.System(ctx, [(pos, box, sp)], 5.0)
    e64, f64, v64 = _compute(ctx, system, models, tg.TGAP_FP64, n)
    assert np.max(np.abs(e64 - e_o)) < E_TOL
    assert np.max(np.abs(f64 - f_o)) < F_TOL
    assert np.max(np.abs(v64[0] - v_o)) < V_TOL
    e32, f32, _ = _compute(ctx, system, models, tg.TGAP_MIXED, n)
    assert np.sqrt(np.mean((e32 - e64) ** 2)) < E_RMSE
    assert np.sqrt(np.mean((f32 - f64) ** 2)) < F_RMSE
    system.close()
    for m in models:
        m.close()


def test_species_e0_on_the_resident_path(ctx, tg, synth):
    hyp = synth.sio2_hypers()
    pool_q = []
    for k in range(2):
        p, bx, s, _ = synth.random_packing(48, 2.2, SIO2_DMIN, SIO2_FRAC, seed=70 + k)
        pool_q.append((helpers.oracle_descriptors(hyp, p, bx, s, 1), helpers.oracle_descriptors(hyp, p, bx, s, 2)))
    mSi = synth.gap_model(np.concatenate([a for a, _ in pool_q]), 20, seed=3)
    mO = synth.gap_model(np.concatenate([b for _, b in pool_q]), 20, seed=4)
    mSi["central_species"], mO["central_species"] = 1, 2
    pos, box, sp, masses = synth.random_packing(48, 2.2, SIO2_DMIN, SIO2_FRAC, seed=75)
    n = len(pos)
    e0 = np.array([-1.37, -2.71])  # eV, different per species
    e_o, f_o, v_o = helpers.oracle_structure_eval(hyp, [mSi, mO], pos, box, sp)
    e_tot = e_o + orc.calculate_e0(sp, e0)
    models = [tg.Model(ctx, hyp, mm["Qs"], mm["alphas"], 1.0, 4.0, central_species=mm["central_species"])
              for mm in (mSi, mO)]
    system = tg.System(ctx, [(pos, box, sp)], 5.0 + 0.3)
    e_plain, _, _ = _compute(ctx, system, models, tg.TGAP_FP64, n)
    assert np.max(np.abs(e_plain - e_o)) < E_TOL  # nothing added before set_e0
    system.set_e0(e0)
    for prec, tol in ((tg.TGAP_FP64, E_TOL), (tg.TGAP_MIXED, 5e-4)):
        e_g, f_g, v_g = _compute(ctx, system, models, prec, n)
        assert np.max(np.abs(e_g - e_tot)) < tol, prec
        if prec == tg.TGAP_FP64:
            assert np.max(np.abs(f_g - f_o)) < F_TOL  # forces do not see e0
            assert np.max(np.abs(v_g[0] - v_o)) < V_TOL
    # host-buffer calculate_gap_soap entry
    e_h, f_h, _ = system.calculate_gap_soap(models, tg.TGAP_FP64, pos, rebuild=True)
    assert np.max(np.abs(e_h - e_tot)) < E_TOL
    # MD potential energy of the first step = sum of the total site energies at the start
    md = tg.MD(ctx, system, models, masses, 0.5, rebuild_every=5, precision=tg.TGAP_FP64)
    md.set_velocities(np.zeros((n, 3)))
    md.run(1)
    st = md.state()
    assert abs(st["e_pot"] - e_tot.sum()) < E_TOL * n
    md.close()
    # MC state energies include e0; energy differences of the moves do not
    system.set_positions(pos)
    system.update(True)
    mc = tg.MC(ctx, system, models, 300.0, precision=tg.TGAP_FP64)
    s0 = mc.state()
    assert np.max(np.abs(s0["energies"] - e_tot)) < E_TOL
    atoms, disp, u = synth.mc_proposals(n, 40, 0.1, seed=76)
    mc.run(atoms, disp, u)
    s1 = mc.state()
    e_o1, _, _ = helpers.oracle_structure_eval(hyp, [mSi, mO], s1["positions"], box, sp)
    assert np.max(np.abs(s1["energies"] - (e_o1 + orc.calculate_e0(sp, e0)))) < 1e-9
    mc.close()
    system.close()
    for m in models:
        m.close()
