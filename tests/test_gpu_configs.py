"""The other benchmark workloads at full size, through the C ABI, with the checks that hold at
any size (the oracle pins the same code paths at small sizes in test_gpu_parity.py):

* batched: 512 independent periodic carbon cells, atom counts log-uniform in [32, 2048],
  densities uniform in [1.5, 3.5] g/cm^3, 1.1 A minimum distance, triclinic strain up to 5 %,
  one system and one evaluation per precision; per cell the forces sum to zero and the virial is
  symmetric; a handful of cells are checked against the oracle; mixed vs FP64 RMSE;
* two-species scale: 32,768-atom SiO2 at 2.2 g/cm^3, species-resolved n_max 8 + 8, l_max 6,
  rcut 5.0/4.5, one synthetic GAP per centre species with 4,000 sparse points; mixed vs FP64,
  force sum, and a short mixed NVE run at 0.5 fs.
"""
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


def _eval(tg, ctx, system, models, precision, n, nst):
    import torch
    e = torch.zeros(n, dtype=torch.float64, device="cuda")
    f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    v = torch.zeros(9 * nst, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    system.compute_device(models, precision, e.data_ptr(), f.data_ptr(), v.data_ptr())
    ctx.synchronize()
    return e.cpu().numpy(), f.cpu().numpy().reshape(n, 3), v.cpu().numpy().reshape(nst, 3, 3)


def test_batched_512_triclinic_cells(ctx, tg, synth):
    hyp, m = helpers.carbon_model(synth, 2000, seed=9, n_pool_structs=10)
    rng = np.random.default_rng(2024)
    sizes = np.exp(rng.uniform(np.log(32), np.log(2048), 512)).astype(int)
    dens = rng.uniform(1.5, 3.5, 512)
    structs = [synth.random_packing(int(n), float(d), 1.1, seed=3000 + k, strain=0.05)[:3]
               for k, (n, d) in enumerate(zip(sizes, dens))]
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, structs, 3.7)
    ntot = int(sizes.sum())
    e64, f64, v64 = _eval(tg, ctx, system, [model], tg.TGAP_FP64, ntot, 512)
    e32, f32, v32 = _eval(tg, ctx, system, [model], tg.TGAP_MIXED, ntot, 512)
    assert np.all(np.isfinite(e64)) and np.all(np.isfinite(f64)) and np.all(np.isfinite(v64))
    off = np.concatenate([[0], np.cumsum(sizes)])
    fmax = np.abs(f64).max()
    for b in range(512):
        fs = f64[off[b]:off[b + 1]].sum(0)
        assert np.max(np.abs(fs)) < 1e-10 * max(1.0, fmax) * sizes[b], b
        assert np.max(np.abs(v64[b] - v64[b].T)) < 1e-12 * max(1.0, np.abs(v64[b]).max()), b
    # oracle on the smallest, the largest-but-affordable and two random cells
    order = np.argsort(sizes)
    picks = {int(order[0]), int(order[40]), int(order[100])}
    for b in sorted(picks):
        pos, box, sp = structs[b]
        e_o, f_o, v_o = helpers.oracle_structure_eval(hyp, [m], pos, box, sp)
        assert np.max(np.abs(e64[off[b]:off[b + 1]] - e_o)) < 1e-10, b
        assert np.max(np.abs(f64[off[b]:off[b + 1]] - f_o)) < 1e-8, b
        assert np.max(np.abs(v64[b] - v_o)) < 1e-8, b
    e_rmse = np.sqrt(np.mean((e32 - e64) ** 2))
    f_rmse = np.sqrt(np.mean((f32 - f64) ** 2))
    assert e_rmse < 0.5e-3 and f_rmse < 5e-3, (e_rmse, f_rmse)
    system.close()
    model.close()


def test_sio2_32768_two_models(ctx, tg, synth):
    import ctypes as C
    import torch
    from turbogap_b200 import native
    hyp = synth.sio2_hypers()
    dmin = {("Si", "O"): 1.4, ("O", "O"): 2.2, ("Si", "Si"): 2.5}
    pos, box, sp, masses = synth.random_packing(32768, 2.2, dmin, {"Si": 1 / 3, "O": 2 / 3}, seed=3)
    n = len(pos)
    system = tg.System(ctx, [(pos, box, sp)], 5.0)
    # sparse sets: FP64 descriptors of this box's own Si / O centres (device)
    pools = []
    for cs in (1, 2):
        dummy = tg.Model(ctx, hyp, np.zeros((1, synth.soap_dim(hyp))), np.zeros(1), central_species=cs)
        q = torch.zeros((n, dummy.dim), dtype=torch.float64, device="cuda")
        nr = C.c_int(0)
        native.check(native.lib().tgap_descriptors(ctx.h, system.h, dummy.h, 0, C.c_void_p(q.data_ptr()),
                                                   C.byref(nr)), ctx.h, "descriptors")
        ctx.synchronize()
        pools.append(q[:nr.value].cpu().numpy())
        dummy.close()
    mods = []
    for cs, pool, seed in ((1, pools[0], 11), (2, pools[1], 12)):
        mm = synth.gap_model(pool, 4000, seed=seed)
        mods.append(tg.Model(ctx, hyp, mm["Qs"], mm["alphas"], 1.0, 4.0, central_species=cs))
    e64, f64, v64 = _eval(tg, ctx, system, mods, tg.TGAP_FP64, n, 1)
    e32, f32, v32 = _eval(tg, ctx, system, mods, tg.TGAP_MIXED, n, 1)
    assert np.all(np.isfinite(e64)) and np.all(np.isfinite(f64))
    assert np.max(np.abs(f64.sum(0))) < 1e-10 * n * max(1.0, np.abs(f64).max())
    assert np.max(np.abs(v64[0] - v64[0].T)) < 1e-10 * max(1.0, np.abs(v64).max())
    e_rmse = np.sqrt(np.mean((e32 - e64) ** 2))
    f_rmse = np.sqrt(np.mean((f32 - f64) ** 2))
    assert e_rmse < 0.5e-3 and f_rmse < 5e-3, (e_rmse, f_rmse)
    system.close()
    # short mixed NVE at 0.5 fs on a skin-padded list: energy conserved to the integrator's accuracy
    system = tg.System(ctx, [(pos, box, sp)], 5.0 + 0.3)
    md = tg.MD(ctx, system, mods, masses, 0.5, rebuild_every=10, precision=tg.TGAP_MIXED)
    md.set_velocities(synth.maxwell_boltzmann(masses, 300.0, seed=4))
    md.run(1)
    s0 = md.state()
    md.run(40)
    s1 = md.state()
    drift = abs((s1["e_pot"] + s1["e_kin"]) - (s0["e_pot"] + s0["e_kin"])) / n
    assert drift < 1e-4, drift
    md.close()
    system.close()
    for mm in mods:
        mm.close()
