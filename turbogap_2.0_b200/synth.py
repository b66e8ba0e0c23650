"""Seeded synthetic systems and GAP models for the SOAP/GAP workloads.

No datasets or fitted potentials are available offline, so every input is generated here:
diamond supercells with uniform noise, random periodic packings at a target density with
per-species minimum distances, optional triclinic strain, and synthetic GAP models whose
sparse set is the normalised SOAP vectors of randomly chosen atoms from further seeded
structures of the same kind, with alphas ~ N(0, variance 1e-6).
"""
import numpy as np

AMU_G_CM3 = 1.66053906660  # 1 amu / A^3 in g / cm^3
MASS_AMU = {"C": 12.011, "Si": 28.0855, "O": 15.999}
AMU_TO_EV_FS2_A2 = 103.6426965268  # read_files.f90:333 (amu -> eV fs^2 / A^2)
KB_EV = 8.6173303e-5  # md_interface.f90:114


def carbon_hypers():
    """SOAP poly3 settings shared by the carbon workloads (n_max = l_max = 8, rcut 3.7/3.2)."""
    return dict(alpha_max=[8], l_max=8, rcut_hard=[3.7], rcut_soft=[3.2], nf=[4.0],
                global_scaling=[1.0], atom_sigma_r=[0.5], atom_sigma_r_scaling=[0.0],
                atom_sigma_t=[0.5], atom_sigma_t_scaling=[0.0], amplitude_scaling=[1.0],
                central_weight=[1.0], radial_enhancement=0, species=["C"])


def sio2_hypers():
    """Species-resolved SOAP for SiO2 (n_max 8 per species, l_max 6, rcut 5.0/4.5)."""
    return dict(alpha_max=[8, 8], l_max=6, rcut_hard=[5.0, 5.0], rcut_soft=[4.5, 4.5],
                nf=[4.0, 4.0], global_scaling=[1.0, 1.0], atom_sigma_r=[0.5, 0.5],
                atom_sigma_r_scaling=[0.0, 0.0], atom_sigma_t=[0.5, 0.5],
                atom_sigma_t_scaling=[0.0, 0.0], amplitude_scaling=[1.0, 1.0],
                central_weight=[1.0, 1.0], radial_enhancement=0, species=["Si", "O"])


def soap_dim(hyp):
    n = int(sum(hyp["alpha_max"]))
    return n * (n + 1) // 2 * (int(hyp["l_max"]) + 1)


def diamond_supercell(reps=3, a0=3.567, noise=0.15, seed=0):
    """Cubic diamond, reps^3 conventional cells, uniform +-noise displacement per axis."""
    basis = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                      [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
    cells = np.array([[i, j, k] for i in range(reps) for j in range(reps) for k in range(reps)])
    pos = ((cells[:, None, :] + basis[None, :, :]).reshape(-1, 3)) * a0
    rng = np.random.default_rng(seed)
    pos = pos + rng.uniform(-noise, noise, size=pos.shape)
    L = reps * a0
    box = np.diag([L, L, L]).astype(float)
    species = np.ones(len(pos), np.int32)
    return pos, box, species


def random_packing(n_atoms, density, dmin, fractions=None, seed=0, strain=0.0, max_tries=200000):
    """Random periodic packing.

    n_atoms: total atoms; density in g/cm^3; fractions: {species_name: fraction} (default
    carbon); dmin: scalar or {(a, b): d} with species names. The packing is made in a cubic
    box with the minimum-image convention, then, if strain > 0, a seeded symmetric strain with
    components uniform in [-strain, strain] maps it to a triclinic cell (distances change by at
    most ~strain). Returns positions (n, 3), box rows a, b, c (3, 3), species ids (1-based in
    the order of `fractions`), masses (amu).
    """
    rng = np.random.default_rng(seed)
    if fractions is None:
        fractions = {"C": 1.0}
    names = list(fractions)
    counts = [int(round(fractions[s] * n_atoms)) for s in names]
    counts[-1] = n_atoms - sum(counts[:-1])
    species = np.concatenate([np.full(c, i + 1, np.int32) for i, c in enumerate(counts)])
    rng.shuffle(species)
    mass = np.array([MASS_AMU[names[s - 1]] for s in species])
    vol = mass.sum() * AMU_G_CM3 / density
    L = vol ** (1.0 / 3.0)
    ns = len(names)
    dm = np.zeros((ns + 1, ns + 1))
    if np.isscalar(dmin):
        dm[:] = dmin
    else:
        for (sa, sb), d in dmin.items():
            ia, ib = names.index(sa) + 1, names.index(sb) + 1
            dm[ia, ib] = dm[ib, ia] = d
    dcell = dm.max()
    nc = max(1, int(L / dcell))
    cw = L / nc
    grid = {}
    pos = np.zeros((n_atoms, 3))
    tries = 0
    for i in range(n_atoms):
        si = species[i]
        while True:
            tries += 1
            if tries > max_tries + 50 * n_atoms:
                raise RuntimeError("random_packing: too dense for the minimum distances")
            p = rng.uniform(0.0, L, 3)
            ci = (p // cw).astype(int) % nc
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        key = ((ci[0] + dx) % nc, (ci[1] + dy) % nc, (ci[2] + dz) % nc)
                        for j in grid.get(key, ()):
                            d = pos[j] - p
                            d -= L * np.round(d / L)
                            if d @ d < dm[si, species[j]] ** 2:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                pos[i] = p
                grid.setdefault(tuple(ci), []).append(i)
                break
    box = np.diag([L, L, L]).astype(float)
    if strain > 0.0:
        e = rng.uniform(-strain, strain, (3, 3))
        e = 0.5 * (e + e.T)
        F = np.eye(3) + e
        box = box @ F.T
        pos = pos @ F.T
    return pos, box, species, mass


def maxwell_boltzmann(masses_amu, temperature, seed=0):
    """Velocities (A/fs) at `temperature`, centre-of-mass motion removed."""
    rng = np.random.default_rng(seed)
    m = np.asarray(masses_amu) * AMU_TO_EV_FS2_A2
    v = rng.normal(size=(len(m), 3)) * np.sqrt(KB_EV * temperature / m)[:, None]
    p = (m[:, None] * v).sum(0) / m.sum()
    return v - p


def gap_model(q_pool, n_sparse, seed=0, zeta=4.0, delta=1.0, alpha_var=1e-6):
    """Synthetic GAP model: sparse set = n_sparse rows drawn without replacement from q_pool
    (normalised SOAP vectors), alphas ~ N(0, alpha_var)."""
    rng = np.random.default_rng(seed)
    idx = rng.choice(len(q_pool), size=n_sparse, replace=len(q_pool) < n_sparse)
    Qs = np.ascontiguousarray(q_pool[idx], dtype=np.float64)
    alphas = rng.normal(0.0, np.sqrt(alpha_var), n_sparse)
    return dict(Qs=Qs, alphas=alphas, zeta=zeta, delta=delta)


def mc_proposals(n_atoms, n, radius, seed=0):
    """Single-atom Monte Carlo proposals: atoms uniform over [0, n_atoms), displacements uniform
    in a ball of `radius` (A), and the uniform deviates of the acceptance test."""
    rng = np.random.default_rng(seed)
    atoms = rng.integers(0, n_atoms, size=n).astype(np.int32)
    d = rng.normal(size=(n, 3))
    d *= (radius * rng.random(n) ** (1.0 / 3.0) / np.linalg.norm(d, axis=1))[:, None]
    u = rng.random(n)
    return atoms, d, u
