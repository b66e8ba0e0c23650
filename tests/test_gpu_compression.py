"""SOAP compression on the device (tgap_model_create_compressed: q = P p / |P p|, the
P_transformation of read_gap.f90:489-559) against the oracle's compression: energies, forces and
virial in FP64 within the path's parity bars, the mixed form within its RMSE bars; an identity P
gives the uncompressed model's results."""
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


def _eval(ctx, system, model, precision, n):
    import torch
    e = torch.zeros(n, dtype=torch.float64, device="cuda")
    f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    v = torch.zeros(9, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    system.compute_device([model], precision, e.data_ptr(), f.data_ptr(), v.data_ptr())
    ctx.synchronize()
    return e.cpu().numpy(), f.cpu().numpy().reshape(n, 3), v.cpu().numpy().reshape(3, 3, order="F")


def _compressed_model(synth, hyp, dim_out, nnz, n_sparse, seed):
    """A random sparse P (rows repeated, some rows empty) and sparse points in its space: the
    oracle's compressed descriptors of perturbed diamond cells."""
    rng = np.random.default_rng(seed)
    D = synth.soap_dim(hyp)
    comp = (rng.integers(1, dim_out + 1, nnz), rng.integers(1, D + 1, nnz), rng.normal(size=nnz), dim_out)
    hc = dict(hyp, compress=comp)
    pool = []
    for k in range(2):
        p, box, sp = synth.diamond_supercell(2, seed=2000 + 17 * seed + k)
        pool.append(helpers.oracle_descriptors(hc, p, box, sp))
    m = synth.gap_model(np.concatenate(pool), n_sparse, seed=seed)
    return hc, comp, m


@pytest.mark.parametrize("dim_out, nnz", [(120, 400), (40, 1200)])
def test_compressed_model_matches_oracle(ctx, tg, synth, dim_out, nnz):
    hyp = synth.carbon_hypers()
    hc, comp, m = _compressed_model(synth, hyp, dim_out, nnz, 60, seed=dim_out)
    pos, box, sp, _ = synth.random_packing(160, 2.5, 1.2, seed=31)
    n = len(pos)
    e_o, f_o, v_o = helpers.oracle_structure_eval(hc, [m], pos, box, sp)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], m["delta"], m["zeta"], compress=comp)
    assert model.dim == dim_out
    system = tg.System(ctx, [(pos, box, sp)], 3.7)
    e, f, v = _eval(ctx, system, model, tg.TGAP_FP64, n)
    assert np.max(np.abs(e - e_o)) < 1e-10
    assert np.max(np.abs(f - f_o)) < 1e-8
    assert np.max(np.abs(v - v_o)) < 1e-8
    e32, f32, _ = _eval(ctx, system, model, tg.TGAP_MIXED, n)
    assert np.sqrt(np.mean((e32 - e_o) ** 2)) < 0.5e-3
    assert np.sqrt(np.mean((f32 - f_o) ** 2)) < 5e-3
    system.close()
    model.close()


def test_identity_compression_equals_the_uncompressed_model(ctx, tg, synth):
    hyp, m = helpers.carbon_model(synth, 60, seed=7)
    D = synth.soap_dim(hyp)
    ident = (np.arange(1, D + 1), np.arange(1, D + 1), np.ones(D), D)
    pos, box, sp, _ = synth.random_packing(160, 2.5, 1.2, seed=32)
    n = len(pos)
    system = tg.System(ctx, [(pos, box, sp)], 3.7)
    plain = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    comp = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0, compress=ident)
    for prec, tol in ((tg.TGAP_FP64, 1e-12), (tg.TGAP_MIXED, 1e-6)):
        e0, f0, _ = _eval(ctx, system, plain, prec, n)
        e1, f1, _ = _eval(ctx, system, comp, prec, n)
        assert np.max(np.abs(e1 - e0)) <= tol * max(1.0, np.abs(e0).max())
        assert np.max(np.abs(f1 - f0)) <= tol * max(1.0, np.abs(f0).max())
    system.close()
    plain.close()
    comp.close()


def test_get_soap_with_compression_matches_oracle(ctx, tg, synth):
    """tgap_get_soap (the get_soap surface) with compress_soap: the compressed descriptor and its
    Cartesian derivatives against the oracle's compression at the parity bars of get_soap."""
    import oracle_lib as orc
    hyp = synth.carbon_hypers()
    pos, box, sp = synth.diamond_supercell(2, seed=33)
    rc = max(hyp["rcut_hard"])
    idx = orc.number_of_unit_cells(*box, rc)
    small = bool(np.any(idx > 1))
    pos_sc, sp_sc, a, b, c = orc.set_supercell(pos, sp, idx, *box)
    nb = orc.build_neighbors(pos_sc, len(pos), a, b, c, rc, sp_sc, small)
    mask = (nb["neighbor_species"] == 1)[:, None]
    rng = np.random.default_rng(5)
    D = synth.soap_dim(hyp)
    comp = (rng.integers(1, 81, 300), rng.integers(1, D + 1, 300), rng.normal(size=300))
    comp = (np.concatenate([comp[0], [80]]), np.concatenate([comp[1], [1]]), np.concatenate([comp[2], [1.0]]))
    q_o, d_o = orc.get_soap(orc.Hypers(dict(hyp, compress=comp + (80,))), nb["n_neigh"], mask, nb["rjs"],
                            nb["thetas"], nb["phis"])
    q_g, d_g = ctx.get_soap(hyp, nb["n_neigh"], mask, nb["rjs"], nb["thetas"], nb["phis"], compress=comp)
    assert q_g.shape == q_o.shape == (len(pos), 80)
    assert np.max(np.abs(q_g - q_o)) < 1e-12
    assert np.max(np.abs(d_g - d_o)) < 1e-10
