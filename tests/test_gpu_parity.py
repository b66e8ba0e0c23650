"""Parity of the sm_100a path (through the C ABI) with the CPU oracle.

Bars: neighbor pairs bit-exact (list order, rjs and xyz bits); FP64 energies within
1e-10 eV/atom, forces within 1e-8 eV/A, virial within 1e-8 eV; descriptors within 1e-12
(q) and 1e-10 (dq/dr). Mixed precision (FP32 descriptor, bf16x3 tensor-core GEMM) is held to
energy RMSE <= 0.5 meV/atom and force RMSE <= 5 meV/A against FP64.
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


@pytest.fixture(scope="module")
def ctx(tg):
    import torch
    assert torch.cuda.is_available()
    c = tg.Context(0)
    yield c
    c.close()


def _device(n, torch):
    return torch.zeros(n, dtype=torch.float64, device="cuda")


def _compute(tg, ctx, system, models, precision, n, nst=1):
    import torch
    e = _device(n, torch)
    f = _device(3 * n, torch)
    v = _device(9 * nst, torch)
    torch.cuda.synchronize()
    system.compute_device(models, precision, e.data_ptr(), f.data_ptr(), v.data_ptr())
    ctx.synchronize()
    return e.cpu().numpy(), f.cpu().numpy().reshape(n, 3), v.cpu().numpy().reshape(nst, 3, 3)


# ------------------------------------------------------------------------- neighbors

def _nb_compare(nb_g, nb_o):
    assert np.array_equal(nb_g["n_neigh"], nb_o["n_neigh"])
    assert np.array_equal(nb_g["neighbors_list"], nb_o["neighbors_list"])
    assert np.array_equal(nb_g["rjs"], nb_o["rjs"])  # bit-exact distances
    assert np.array_equal(nb_g["xyz"], nb_o["xyz"])
    assert np.array_equal(nb_g["neighbor_species"], nb_o["neighbor_species"])
    assert np.allclose(nb_g["thetas"], nb_o["thetas"], rtol=0, atol=1e-14)
    assert np.allclose(nb_g["phis"], nb_o["phis"], rtol=0, atol=1e-14)


@pytest.mark.parametrize("case", ["diamond_m2", "packing_m4", "packing_large", "packing_dense"])
def test_neighbors_cell_path_bit_exact(ctx, synth, case):
    """The linked-cell list against the oracle's, bit for bit; packing_dense (rcut 7 A: 3 cells a
    side of ~74 atoms, ~180 pairs a site) has cells longer than a warp and rows longer than the
    staging width, so the count pass walks several 32-candidate steps per cell and the fill pass
    walks the cells again."""
    if case == "diamond_m2":
        pos, box, sp = synth.diamond_supercell(3, seed=7)
        rc = 3.7
    elif case == "packing_m4":
        pos, box, sp, _ = synth.random_packing(500, 2.5, 1.2, seed=8)
        rc = 4.0
    elif case == "packing_large":
        pos, box, sp, _ = synth.random_packing(4096, 2.5, 1.2, seed=9)
        rc = 4.0
    else:
        pos, box, sp, _ = synth.random_packing(2000, 2.5, 1.2, seed=13)
        rc = 7.0
    nb_o = orc.build_neighbors(pos, len(pos), *box, rc, sp, False)
    nb_g = ctx.build_neighbors_list(pos, len(pos), *box, rc, sp, box_small=False)
    _nb_compare(nb_g, nb_o)


@pytest.mark.parametrize("strain", [0.0, 0.04])
def test_neighbors_brute_force_and_supercell_bit_exact(ctx, synth, strain):
    pos, box, sp, _ = synth.random_packing(40, 2.0, 1.2, seed=10, strain=strain)
    idx = orc.number_of_unit_cells(*box, 3.7)
    pos_sc, sp_sc, a, b, c = orc.set_supercell(pos, sp, idx, *box)
    small = bool(np.any(idx > 1))
    nb_o = orc.build_neighbors(pos_sc, len(pos), a, b, c, 3.7, sp_sc, small)
    nb_g = ctx.build_neighbors_list(pos_sc, len(pos), a, b, c, 3.7, sp_sc, box_small=small)
    _nb_compare(nb_g, nb_o)


def test_neighbors_triclinic_no_replica(ctx, synth):
    pos, box, sp, _ = synth.random_packing(400, 2.0, 1.2, seed=11, strain=0.05)
    nb_o = orc.build_neighbors(pos, len(pos), *box, 3.7, sp, False)
    nb_g = ctx.build_neighbors_list(pos, len(pos), *box, 3.7, sp, box_small=False)
    _nb_compare(nb_g, nb_o)


def test_neighbors_geometry_refresh(ctx, synth):
    pos, box, sp, _ = synth.random_packing(300, 2.5, 1.2, seed=12)
    nb = orc.build_neighbors(pos, len(pos), *box, 4.0, sp, False)
    moved = pos + np.random.default_rng(0).uniform(-0.1, 0.1, pos.shape)
    geo_o = orc.neighbor_geometry(moved, len(pos), *box, nb["n_neigh"], nb["neighbors_list"], sp)
    geo_g = ctx.build_neighbors_list(moved, len(pos), *box, 4.0, sp, rebuild=False, n_neigh=nb["n_neigh"],
                                     neighbors_list=nb["neighbors_list"])
    assert np.array_equal(geo_g["rjs"], geo_o["rjs"]) and np.array_equal(geo_g["xyz"], geo_o["xyz"])


def test_neighbors_capacity_overflow_reports_required_size(ctx, synth, tg):
    from turbogap_b200 import native
    pos, box, sp = synth.diamond_supercell(3, noise=0.0)
    n = len(pos)
    cap = 10
    buf_i = np.zeros(cap, np.int32)
    buf_d = np.zeros(cap)
    buf_x = np.zeros(3 * cap)
    nn = np.zeros(n, np.int32)
    npairs = C.c_int64(0)
    st = native.lib().tgap_build_neighbors(
        ctx.h, n, n, native.ptr(np.ascontiguousarray(pos)), native.ptr(box[0].copy()), native.ptr(box[1].copy()),
        native.ptr(box[2].copy()), 0, 3.7, native.ptr(sp), 1, native.ptr(nn), native.ptr(buf_i), native.ptr(buf_d),
        native.ptr(buf_x), native.ptr(buf_d), native.ptr(buf_d), native.ptr(buf_i), cap, C.byref(npairs))
    assert st == 3 and npairs.value == 35 * n


# ------------------------------------------------------------------------- descriptor

def _soap_inputs(synth, seed, n_species=1):
    if n_species == 1:
        hyp = synth.carbon_hypers()
        pos, box, sp = synth.diamond_supercell(2, seed=seed)
    else:
        hyp = synth.sio2_hypers()
        pos, box, sp, _ = synth.random_packing(
            48, 2.2, {("Si", "O"): 1.4, ("O", "O"): 2.2, ("Si", "Si"): 2.5}, {"Si": 1 / 3, "O": 2 / 3}, seed=seed)
    rc = max(hyp["rcut_hard"])
    idx = orc.number_of_unit_cells(*box, rc)
    small = bool(np.any(idx > 1))
    pos_sc, sp_sc, a, b, c = orc.set_supercell(pos, sp, idx, *box)
    nb = orc.build_neighbors(pos_sc, len(pos), a, b, c, rc, sp_sc, small)
    ns = len(hyp["alpha_max"])
    mask = np.stack([nb["neighbor_species"] == s + 1 for s in range(ns)], axis=1)
    return hyp, nb, mask


@pytest.mark.parametrize("n_species", [1, 2])
def test_get_soap_matches_oracle(ctx, synth, n_species):
    hyp, nb, mask = _soap_inputs(synth, 21, n_species)
    q_o, d_o = orc.get_soap(orc.Hypers(hyp), nb["n_neigh"], mask, nb["rjs"], nb["thetas"], nb["phis"])
    q_g, d_g = ctx.get_soap(hyp, nb["n_neigh"], mask, nb["rjs"], nb["thetas"], nb["phis"])
    assert np.max(np.abs(q_g - q_o)) < 1e-12
    assert np.max(np.abs(d_g - d_o)) < 1e-10


def test_get_soap_energy_and_forces_matches_oracle(ctx, synth):
    hyp, nb, mask = _soap_inputs(synth, 22)
    H = orc.Hypers(hyp)
    q, der = orc.get_soap(H, nb["n_neigh"], mask, nb["rjs"], nb["thetas"], nb["phis"])
    model = synth.gap_model(q, 30, seed=3)
    n = len(nb["n_neigh"])
    args = (q, der, model["alphas"], 1.0, 4.0, 0.0, model["Qs"], nb["n_neigh"], nb["neighbors_list"], nb["xyz"])
    e_o, f_o, v_o = orc.soap_energy_and_forces(*args, n_sites0=n)
    e_g, f_g, v_g = ctx.get_soap_energy_and_forces(*args, n_sites0=n)
    assert np.max(np.abs(e_g - e_o)) < E_TOL
    assert np.max(np.abs(f_g - f_o)) < F_TOL
    assert np.max(np.abs(v_g - v_o)) < V_TOL


# ------------------------------------------------------------------------- GAP

@pytest.fixture(scope="module")
def carbon(synth):
    hyp, m = helpers.carbon_model(synth, 200, seed=5)
    return hyp, m


def test_get_gap_soap_fp64_matches_oracle(ctx, synth, carbon):
    hyp, m = carbon
    pos, box, sp = synth.diamond_supercell(3, seed=31)
    n = len(pos)
    nb = orc.build_neighbors(pos, n, *box, 3.7, sp, False)
    e_o, f_o, v_o = orc.get_gap_soap(orc.Hypers(hyp), n, nb, sp, 0, m["alphas"], m["Qs"], 1.0, 4.0)
    e_g, f_g, v_g = ctx.get_gap_soap(hyp, n, nb, sp, 0, m["alphas"], m["Qs"], 1.0, 4.0)
    assert np.max(np.abs(e_g - e_o)) < E_TOL
    assert np.max(np.abs(f_g - f_o)) < F_TOL
    assert np.max(np.abs(v_g - v_o)) < V_TOL


def test_resident_compute_fp64_matches_oracle(ctx, tg, synth, carbon):
    hyp, m = carbon
    pos, box, sp, _ = synth.random_packing(256, 2.5, 1.2, seed=32)
    e_o, f_o, v_o = helpers.oracle_structure_eval(hyp, [m], pos, box, sp)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7)
    e_g, f_g, v_g = _compute(tg, ctx, system, [model], tg.TGAP_FP64, len(pos))
    assert np.max(np.abs(e_g - e_o)) < E_TOL
    assert np.max(np.abs(f_g - f_o)) < F_TOL
    assert np.max(np.abs(v_g[0] - v_o)) < V_TOL


def test_dense_sites_with_more_than_32_pairs(ctx, tg, synth, carbon):
    """3.5 g/cm3: most sites have 33-46 in-cutoff neighbors, so the warp kernels compact and
    process each site's pairs in several 32-pair passes."""
    hyp, m = carbon
    pos, box, sp, _ = synth.random_packing(200, 3.5, 1.1, seed=33)
    nb = orc.build_neighbors(pos, len(pos), *box, 3.7, sp, False)
    assert nb["n_neigh"].max() - 1 > 40
    e_o, f_o, v_o = helpers.oracle_structure_eval(hyp, [m], pos, box, sp)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7)
    e_g, f_g, v_g = _compute(tg, ctx, system, [model], tg.TGAP_FP64, len(pos))
    assert np.max(np.abs(e_g - e_o)) < E_TOL
    assert np.max(np.abs(f_g - f_o)) < F_TOL
    assert np.max(np.abs(v_g[0] - v_o)) < V_TOL
    e32, f32, _ = _compute(tg, ctx, system, [model], tg.TGAP_MIXED, len(pos))
    assert np.sqrt(np.mean((e32 - e_g) ** 2)) < 0.5e-3 and np.sqrt(np.mean((f32 - f_g) ** 2)) < 5e-3


def test_batched_uneven_triclinic_structures(ctx, tg, synth, carbon):
    hyp, m = carbon
    structs = []
    for k, n in enumerate([32, 77, 150]):
        pos, box, sp, _ = synth.random_packing(n, 1.5 + k, 1.1, seed=40 + k, strain=0.05)
        structs.append((pos, box, sp))
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, structs, 3.7)
    ntot = sum(len(s[2]) for s in structs)
    e_g, f_g, v_g = _compute(tg, ctx, system, [model], tg.TGAP_FP64, ntot, nst=len(structs))
    off = 0
    for b, (pos, box, sp) in enumerate(structs):
        e_o, f_o, v_o = helpers.oracle_structure_eval(hyp, [m], pos, box, sp)
        n = len(pos)
        assert np.max(np.abs(e_g[off:off + n] - e_o)) < E_TOL
        assert np.max(np.abs(f_g[off:off + n] - f_o)) < F_TOL
        assert np.max(np.abs(v_g[b] - v_o)) < V_TOL
        off += n


def test_two_species_two_models(ctx, tg, synth):
    hyp = synth.sio2_hypers()
    dmin = {("Si", "O"): 1.4, ("O", "O"): 2.2, ("Si", "Si"): 2.5}
    pool_q = []
    for k in range(2):
        p, bx, s, _ = synth.random_packing(48, 2.2, dmin, {"Si": 1 / 3, "O": 2 / 3}, seed=50 + k)
        pool_q.append((helpers.oracle_descriptors(hyp, p, bx, s, 1), helpers.oracle_descriptors(hyp, p, bx, s, 2)))
    mSi = synth.gap_model(np.concatenate([a for a, _ in pool_q]), 20, seed=1)
    mO = synth.gap_model(np.concatenate([b for _, b in pool_q]), 20, seed=2)
    mSi["central_species"] = 1
    mO["central_species"] = 2
    pos, box, sp, _ = synth.random_packing(48, 2.2, dmin, {"Si": 1 / 3, "O": 2 / 3}, seed=55)
    e_o, f_o, v_o = helpers.oracle_structure_eval(hyp, [mSi, mO], pos, box, sp)
    models = [tg.Model(ctx, hyp, mm["Qs"], mm["alphas"], 1.0, 4.0, central_species=mm["central_species"])
              for mm in (mSi, mO)]
    system = tg.System(ctx, [(pos, box, sp)], 5.0)
    e_g, f_g, v_g = _compute(tg, ctx, system, models, tg.TGAP_FP64, len(pos))
    assert np.max(np.abs(e_g - e_o)) < E_TOL
    assert np.max(np.abs(f_g - f_o)) < F_TOL
    assert np.max(np.abs(v_g[0] - v_o)) < V_TOL


def test_isolated_atom_and_dimer(ctx, tg, synth, carbon):
    hyp, m = carbon
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    box = np.diag([30.0, 30.0, 30.0])
    for pos in (np.array([[15.0, 15.0, 15.0]]), np.array([[15.0, 15.0, 15.0], [16.3, 15.2, 14.9]])):
        sp = np.ones(len(pos), np.int32)
        e_o, f_o, _ = helpers.oracle_structure_eval(hyp, [m], pos, box, sp)
        system = tg.System(ctx, [(pos, box, sp)], 3.7)
        e_g, f_g, _ = _compute(tg, ctx, system, [model], tg.TGAP_FP64, len(pos))
        assert np.max(np.abs(e_g - e_o)) < E_TOL
        assert np.max(np.abs(f_g - f_o)) < F_TOL
        if len(pos) == 2:
            assert np.allclose(f_g[0], -f_g[1], atol=1e-14)


def test_bad_hypers_raise(ctx, tg, synth, carbon):
    hyp, m = carbon
    bad = dict(hyp, l_max=20)
    with pytest.raises(tg.TgapError):
        tg.Model(ctx, bad, m["Qs"], m["alphas"])


# ------------------------------------------------------------------------- mixed precision

def test_mixed_precision_rmse_against_fp64(ctx, tg, synth, carbon):
    hyp, m = carbon
    pos, box, sp, _ = synth.random_packing(512, 2.5, 1.2, seed=60)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7)
    e64, f64, v64 = _compute(tg, ctx, system, [model], tg.TGAP_FP64, len(pos))
    e32, f32, v32 = _compute(tg, ctx, system, [model], tg.TGAP_MIXED, len(pos))
    e_rmse = np.sqrt(np.mean((e32 - e64) ** 2))
    f_rmse = np.sqrt(np.mean((f32 - f64) ** 2))
    assert e_rmse < 0.5e-3 and f_rmse < 5e-3, (e_rmse, f_rmse)
    # tighter sanity: the split-bf16 GEMM keeps ~16 mantissa bits
    assert e_rmse < 1e-5 * max(1.0, np.abs(e64).max() * 1e3)


def test_mixed_get_gap_soap_matches_resident_mixed(ctx, tg, synth, carbon):
    hyp, m = carbon
    pos, box, sp = synth.diamond_supercell(3, seed=61)
    n = len(pos)
    nb = orc.build_neighbors(pos, n, *box, 3.7, sp, False)
    e64, f64, _ = ctx.get_gap_soap(hyp, n, nb, sp, 0, m["alphas"], m["Qs"], 1.0, 4.0)
    e32, f32, _ = ctx.get_gap_soap(hyp, n, nb, sp, 0, m["alphas"], m["Qs"], 1.0, 4.0, precision=tg.TGAP_MIXED)
    assert np.sqrt(np.mean((e32 - e64) ** 2)) < 0.5e-3
    assert np.sqrt(np.mean((f32 - f64) ** 2)) < 5e-3


# ------------------------------------------------------------------------- MD

def test_md_fp64_matches_oracle_verlet(ctx, tg, synth, carbon):
    """Every step of the device MD (CUDA-graph steps and the eager rebuild steps in between)
    against the oracle: forces at the device's positions within F_TOL, and the velocity-Verlet
    update (md_utils.f90:486-532) of the oracle from the device's previous state within 1e-12.
    The pair list grows across rebuilds here, which must re-capture the step graph."""
    hyp, m = carbon
    pos, box, sp, masses = synth.random_packing(128, 2.5, 1.2, seed=70)
    vel = synth.maxwell_boltzmann(masses, 3000.0, seed=1)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.3)
    # rebuild often enough that no pair crosses rcut + skin between rebuilds at 3000 K
    md = tg.MD(ctx, system, [model], masses, 1.0, rebuild_every=4, use_graph=True)
    md.set_velocities(vel)
    mm = masses * synth.AMU_TO_EV_FS2_A2
    x, v = pos.copy(), vel.copy()
    xp, fp = np.zeros_like(x), np.zeros_like(x)
    pairs = set()
    for k in range(14):
        md.run(1)
        st = md.state()
        pairs.add(system.n_pairs)
        _, f, _ = helpers.oracle_structure_eval(hyp, [m], x, box, sp)
        assert np.max(np.abs(st["forces"] - f)) < F_TOL, k
        orc.velocity_verlet(x, xp, v, st["forces"], fp, mm, 1.0, 1.0, k == 0)
        assert np.max(np.abs(st["positions"] - x)) < 1e-12, k
        assert np.max(np.abs(st["velocities"] - v)) < 1e-12, k
        x, v = st["positions"].copy(), st["velocities"].copy()
    assert len(pairs) > 1  # the list changed size across rebuilds


def test_md_device_rebuild_count_matches_a_host_rebuild(ctx, tg, synth, carbon):
    """After the first step the MD rebuilds its lists on the device without reading the pair count
    back; tgap_system_n_pairs then reads it, and it equals the count of a host rebuild at the same
    positions (the positions the rebuild step started from)."""
    hyp, m = carbon
    pos, box, sp, masses = synth.random_packing(128, 2.5, 1.2, seed=71)
    vel = synth.maxwell_boltzmann(masses, 3000.0, seed=3)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.3)
    md = tg.MD(ctx, system, [model], masses, 1.0, rebuild_every=3, use_graph=True)
    md.set_velocities(vel)
    md.run(3)
    x3 = md.state()["positions"]
    md.run(1)  # step 3 rebuilds on x3
    n_dev = system.n_pairs
    ref = tg.System(ctx, [(x3, box, sp)], 3.7 + 0.3)
    assert n_dev == ref.n_pairs
    ref.close()
    md.close()
    system.close()
    model.close()


def test_md_graphs_follow_an_e0_set_between_runs(ctx, tg, synth, carbon):
    """e0 set between two md.run calls makes the captured step graphs stale: the next step runs
    eagerly and the graphs are captured again. The trajectory equals that of an MD with e0 set from
    the start (e0 moves no force), and so does the potential energy once both carry it."""
    hyp, m = carbon
    pos, box, sp, masses = synth.random_packing(128, 2.5, 1.2, seed=73)
    vel = synth.maxwell_boltzmann(masses, 1000.0, seed=4)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    out = []
    for late in (False, True):
        system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.3)
        if not late:
            system.set_e0([-2.5])
        md = tg.MD(ctx, system, [model], masses, 1.0, rebuild_every=5, use_graph=True)
        md.set_velocities(vel)
        md.run(12)
        if late:
            system.set_e0([-2.5])
        md.run(13)
        out.append(md.state())
        md.close()
        system.close()
    assert np.max(np.abs(out[0]["positions"] - out[1]["positions"])) < 1e-9
    assert abs(out[0]["e_pot"] - out[1]["e_pot"]) < 1e-8
    model.close()


def test_md_pair_capacity_overflow_is_reported(ctx, tg, synth, carbon):
    """A device-side rebuild that finds more pairs than the arrays reserved (a quarter above the
    first list) clamps the lists inside the arrays and reports TGAP_ERR_CAPACITY at the next check,
    with no fault: the atoms are drawn halfway towards the box centre (128 atoms in a 5 A cube,
    nearly all of them neighbors of each other) before the next rebuild."""
    hyp, m = carbon
    pos, box, sp, masses = synth.random_packing(128, 2.5, 1.2, seed=72)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.3)
    md = tg.MD(ctx, system, [model], masses, 0.5, rebuild_every=2, use_graph=True)
    md.set_velocities(np.zeros_like(pos))
    md.run(2)
    x = md.state()["positions"]
    c = 0.5 * np.asarray(box).sum(axis=0)
    system.set_positions(c + 0.5 * (x - c))
    with pytest.raises(tg.TgapError) as err:
        md.run(2)
        md.state()
    assert err.value.status == 3  # TGAP_ERR_CAPACITY
    ctx.synchronize()
    md.close()
    system.close()
    model.close()


# ------------------------------------------------------------------------- local properties

def test_local_property_predict_matches_oracle(ctx, synth):
    """tgap_local_property_predict (local_properties.f90:46-147, host arrays) against the oracle:
    an integer zeta with nothing clipped, then zeta = 4 + 5e-6 (real power under the 1e-10 rule)
    with V0 set so that about half the sites clip to zero."""
    hyp, nb, mask = _soap_inputs(synth, 23)
    q, der = orc.get_soap(orc.Hypers(hyp), nb["n_neigh"], mask, nb["rjs"], nb["thetas"], nb["phis"])
    model = synth.gap_model(q, 30, seed=5)
    a_pos = np.abs(model["alphas"])
    raw = 1.2 ** 2 * (q @ model["Qs"].T) ** 4 @ model["alphas"]
    for alphas, V0, zeta in ((a_pos, 0.0, 4.0), (model["alphas"], -np.median(raw), 4.0 + 5e-6)):
        V_o, Vd_o = orc.local_property_predict(q, model["Qs"], alphas, V0, 1.2, zeta, der, nb["n_neigh"])
        V_g, Vd_g = ctx.local_property_predict(q, model["Qs"], alphas, V0, 1.2, zeta, der, nb["n_neigh"])
        assert np.max(np.abs(V_g - V_o)) <= 1e-12 * np.max(np.abs(V_o))
        assert np.max(np.abs(Vd_g - Vd_o)) <= 1e-10 * np.max(np.abs(Vd_o))
        assert np.array_equal(V_g == 0.0, V_o == 0.0)
    assert 0 < np.sum(V_o == 0.0) < len(V_o)


@pytest.mark.parametrize("precision_name", ["TGAP_FP64", "TGAP_MIXED"])
def test_local_property_resident_matches_oracle(ctx, tg, synth, carbon, precision_name):
    """tgap_local_property on a resident system (descriptor derivatives never materialised: the
    adjoint writes each pair's dV_i/dr_j) against the oracle on the same neighbor list. FP64: V to
    1e-12 and V_der to 1e-9 of their largest entry. Mixed: V to 1e-4 of the property's scale before
    the offset V0 (the mixed path's energy accuracy) and V_der to 2e-3 of its largest entry, on the
    sites that are not within 1e-3 of that scale from the clipping point (where rounding may decide
    the clip)."""
    precision = getattr(tg, precision_name)
    hyp, m = carbon
    pos, box, sp = synth.diamond_supercell(3, seed=35)
    n = len(pos)
    nb = orc.build_neighbors(pos, n, *box, 3.7, sp, False)
    P = len(nb["rjs"])
    q, der = orc.get_soap(orc.Hypers(hyp), nb["n_neigh"], np.ones((P, 1), bool), nb["rjs"], nb["thetas"],
                          nb["phis"])
    raw = (q @ m["Qs"].T) ** 4 @ m["alphas"]
    V0 = -np.median(raw)
    V_o, Vd_o = orc.local_property_predict(q, m["Qs"], m["alphas"], V0, 1.0, 4.0, der, nb["n_neigh"])
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7)
    assert system.n_pairs == P
    V_g, Vd_g = system.local_property(model, V0, precision)
    start = np.concatenate([[0], np.cumsum(nb["n_neigh"])])
    if precision == tg.TGAP_FP64:
        assert np.max(np.abs(V_g - V_o)) <= 1e-12 * np.max(np.abs(V_o))
        assert np.max(np.abs(Vd_g - Vd_o)) <= 1e-9 * np.max(np.abs(Vd_o))
        assert np.array_equal(V_g == 0.0, V_o == 0.0)
    else:
        far = np.abs(raw + V0) > 1e-3 * np.max(np.abs(raw))
        assert np.max(np.abs(V_g - V_o)[far]) <= 1e-4 * np.max(np.abs(raw))
        pf = np.repeat(far, nb["n_neigh"])
        assert np.max(np.abs(Vd_g - Vd_o)[pf]) <= 2e-3 * np.max(np.abs(Vd_o))
    assert 0 < np.sum(V_o == 0.0) < n
    clipped = np.nonzero(V_g == 0.0)[0]
    for i in clipped:
        assert np.all(Vd_g[start[i]:start[i + 1]] == 0.0)
    system.close()
    model.close()


# ------------------------------------------------------------------------- pairwise terms

def _sio2_pairs(synth):
    pos, box, sp, _ = synth.random_packing(192, 2.2, {("Si", "O"): 1.4, ("O", "O"): 2.2, ("Si", "Si"): 2.5},
                                           {"Si": 1 / 3, "O": 2 / 3}, seed=43)
    nb = orc.build_neighbors(pos, len(pos), *box, 4.0, sp, False)
    return nb, sp


@pytest.mark.parametrize("species_pair", [(1, 2), (2, 2)])
def test_2b_matches_oracle(ctx, synth, species_pair):
    nb, sp = _sio2_pairs(synth)
    rng = np.random.default_rng(7)
    M = 15
    args = dict(alphas=rng.normal(size=M) * 0.1, cutoff=rng.uniform(0.5, 1.0, M), rcut=4.0, buffer=0.6,
                delta=1.1, sigma=0.4, e0=0.05, Qs=np.linspace(1.3, 3.8, M))
    e_o, f_o, v_o = orc.get_2b_energy_and_forces(nb, sp, *species_pair, n_sites0=len(sp) + 5, **args)
    e_g, f_g, v_g = ctx.get_2b_energy_and_forces(nb, sp, *species_pair, n_sites0=len(sp) + 5, **args)
    assert np.max(np.abs(e_g - e_o)) < E_TOL
    assert np.max(np.abs(f_g - f_o)) < F_TOL
    assert np.max(np.abs(v_g - v_o)) < V_TOL
    assert np.all(f_g[len(sp):] == 0.0)


def test_core_pot_matches_oracle(ctx, synth):
    nb, sp = _sio2_pairs(synth)
    x = np.linspace(0.8, 3.5, 40)
    Vk = 5.0 * np.exp(-2.0 * x) * (1.0 - x / 3.5) ** 2
    yp1, ypn = -12.0, 0.0
    y2 = orc.spline_second_derivatives(x, Vk, yp1, ypn)
    for s1, s2 in ((1, 2), (1, 1)):
        e_o, f_o, v_o = orc.get_core_pot_energy_and_forces(nb, sp, s1, s2, x, Vk, yp1, ypn, y2)
        e_g, f_g, v_g = ctx.get_core_pot_energy_and_forces(nb, sp, s1, s2, x, Vk, yp1, ypn, y2)
        assert np.max(np.abs(e_g - e_o)) < E_TOL
        assert np.max(np.abs(f_g - f_o)) < F_TOL
        assert np.max(np.abs(v_g - v_o)) < V_TOL
    with pytest.raises(Exception):
        ctx.get_core_pot_energy_and_forces(nb, sp, 1, 2, x[::-1], Vk, yp1, ypn, y2)


@pytest.mark.parametrize("kernel,centre,pair", [("exp", 2, (2, 1)), ("pol", 2, (1, 1)), ("exp", 1, (2, 2))])
def test_3b_matches_oracle(ctx, synth, kernel, centre, pair):
    nb, sp = _sio2_pairs(synth)
    rng = np.random.default_rng(11)
    M = 12
    Qs = np.stack([rng.uniform(3.0, 7.0, M), rng.uniform(0.0, 2.0, M), rng.uniform(2.0, 6.0, M)], axis=1)
    sigma = np.array([1.0, 1.0, 1.2]) * (3.0 if kernel == "pol" else 1.0)
    args = dict(alphas=rng.normal(size=M) * 0.05, cutoff=rng.uniform(0.5, 1.0, M), rcut=3.8, buffer=0.5,
                delta=0.9, sigma=sigma, e0=0.02, Qs=Qs, kernel=kernel)
    e_o, f_o, v_o = orc.get_3b_energy_and_forces(nb, sp, centre, *pair, **args)
    e_g, f_g, v_g = ctx.get_3b_energy_and_forces(nb, sp, centre, *pair, **args)
    assert np.abs(f_o).max() > 0.0
    assert np.max(np.abs(e_g - e_o)) < E_TOL
    assert np.max(np.abs(f_g - f_o)) < F_TOL
    assert np.max(np.abs(v_g - v_o)) < V_TOL


def test_model_files_drive_the_device_path(ctx, tg, synth, carbon, tmp_path):
    """A carbon soap_turbo model written as TurboGAP files (.gap + alphas + desc), read back by
    gap_file and loaded on the device, gives the oracle's FP64 energies and forces."""
    hyp, m = carbon
    (tmp_path / "c.alphas").write_text("".join(f"{a:.17g}\n" for a in m["alphas"]))
    (tmp_path / "c.desc").write_text("".join(f"{q:.17g}\n" for q in np.asarray(m["Qs"]).ravel()))
    buf = hyp["rcut_hard"][0] - hyp["rcut_soft"][0]
    (tmp_path / "c.gap").write_text(f"""gap_beg soap_turbo
 n_species = 1
 species = C
 rcut = {hyp['rcut_hard'][0]}
 buffer = {buf}
 atom_sigma_r = {hyp['atom_sigma_r'][0]}
 atom_sigma_t = {hyp['atom_sigma_t'][0]}
 n_max = {hyp['alpha_max'][0]}
 l_max = {hyp['l_max']}
 zeta = 4
 delta = 1.0
 alphas_sparse = c.alphas
 desc_sparse = c.desc
gap_end
""")
    g = tg.gap_file.read_gap(str(tmp_path / "c.gap"), base_dir=str(tmp_path))
    (model,) = tg.gap_file.load_soap_models(ctx, g)
    pos, box, sp = synth.diamond_supercell(3, seed=37)
    n = len(pos)
    system = tg.System(ctx, [(pos, box, sp)], g["rcut_max"])
    import torch
    e = torch.zeros(n, dtype=torch.float64, device="cuda")
    f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    v = torch.zeros(9, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    system.compute_device([model], tg.TGAP_FP64, e.data_ptr(), f.data_ptr(), v.data_ptr())
    ctx.synchronize()
    e_o, f_o, _ = helpers.oracle_structure_eval(hyp, [m], pos, box, sp)
    assert np.max(np.abs(e.cpu().numpy() - e_o)) < E_TOL
    assert np.max(np.abs(f.cpu().numpy().reshape(n, 3) - f_o)) < F_TOL
    system.close()
    model.close()


def test_md_multi_step_graph_matches_single_steps(ctx, tg, synth, carbon):
    """md.run(20) sends the rebuild-free stretches (9 steps) as one graph launch; the trajectory
    matches twenty md.run(1) calls (single-step graphs) to 1e-9 A (only the order of FP64 atomic
    additions can differ)."""
    hyp, m = carbon
    pos, box, sp = synth.diamond_supercell(3, seed=39)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    masses = np.full(len(pos), 12.011)
    vel = np.random.default_rng(4).normal(size=(len(pos), 3)) * 0.01
    out = []
    for chunked in (False, True):
        system = tg.System(ctx, [(pos, box, sp)], 3.7 + 0.3)
        md = tg.MD(ctx, system, [model], masses, 1.0, rebuild_every=10, precision=tg.TGAP_MIXED)
        md.set_velocities(vel)
        if chunked:
            md.run(20)
        else:
            for _ in range(20):
                md.run(1)
        out.append(md.state())
        md.close()
        system.close()
    assert np.max(np.abs(out[0]["positions"] - out[1]["positions"])) < 1e-9
    assert abs(out[0]["e_pot"] - out[1]["e_pot"]) < 1e-9
