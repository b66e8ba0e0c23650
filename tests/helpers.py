"""Shared helpers for the parity tests: seeded systems and the oracle's evaluation of them."""
import numpy as np

import oracle_lib as orc


def oracle_structure_eval(hyp, models, pos, box, species, do_forces=True):
    """Energies (n,), forces (n, 3) and virial (3, 3) of one periodic structure from the CPU
    oracle: supercell replication when needed, neighbor list at the model cutoff, then
    get_gap_soap for every model, summed (calculate_gap_soap.f90:343-447)."""
    n = len(pos)
    rc = max(hyp["rcut_hard"])
    idx = orc.number_of_unit_cells(box[0], box[1], box[2], rc)
    small = bool(np.any(idx > 1))
    if small:
        pos_sc, sp_sc, a, b, c = orc.set_supercell(pos, species, idx, *box)
    else:
        pos_sc, sp_sc, a, b, c = pos, np.asarray(species, np.int32), box[0], box[1], box[2]
    nb = orc.build_neighbors(pos_sc, n, a, b, c, rc, sp_sc, small)
    H = orc.Hypers(hyp)
    e = np.zeros(n)
    f = np.zeros((n, 3))
    v = np.zeros((3, 3))
    for m in models:
        em, fm, vm = orc.get_gap_soap(H, n, nb, sp_sc, m.get("central_species", 0), m["alphas"], m["Qs"],
                                      m["delta"], m["zeta"], do_forces)
        e += em
        f += fm
        v += vm
    return e, f, v


def oracle_descriptors(hyp, pos, box, species, central_species=0):
    n = len(pos)
    rc = max(hyp["rcut_hard"])
    idx = orc.number_of_unit_cells(box[0], box[1], box[2], rc)
    small = bool(np.any(idx > 1))
    if small:
        pos_sc, sp_sc, a, b, c = orc.set_supercell(pos, species, idx, *box)
    else:
        pos_sc, sp_sc, a, b, c = pos, np.asarray(species, np.int32), box[0], box[1], box[2]
    nb = orc.build_neighbors(pos_sc, n, a, b, c, rc, sp_sc, small)
    ns = len(hyp["alpha_max"])
    nsp = nb["neighbor_species"]
    mask = np.zeros((len(nsp), ns), bool)
    for s in range(ns):
        mask[:, s] = nsp == s + 1
    q, _ = orc.get_soap(orc.Hypers(hyp), nb["n_neigh"], mask, nb["rjs"], nb["thetas"], nb["phis"],
                        derivatives=False)
    if central_species:
        q = q[np.asarray(species)[:n] == central_species]
    return q


def carbon_model(synth, n_sparse, seed, n_pool_structs=3, reps=2):
    """Synthetic GAP: sparse set drawn from perturbed diamond supercells (oracle descriptors)."""
    hyp = synth.carbon_hypers()
    pool = []
    for k in range(n_pool_structs):
        p, box, sp = synth.diamond_supercell(reps, seed=1000 + seed * 17 + k)
        pool.append(oracle_descriptors(hyp, p, box, sp))
    m = synth.gap_model(np.concatenate(pool), n_sparse, seed=seed)
    return hyp, m
