"""Pins of the CPU oracle (no GPU).

The reference publishes no golden vectors for this path and cannot be built here (Fortran,
no compiler; soap_turbo absent), so the oracle is pinned by known answers computed
independently of it: exact lattice shell counts, brute-force minimum-image searches,
high-precision (mpmath) evaluation of the radial integral that defines the descriptor,
scipy's modified spherical Bessel functions, sphere quadrature of the harmonics, finite
differences and invariances.
"""
import itertools

import numpy as np
import pytest


def _lat(L):
    return np.array([L, 0, 0.0]), np.array([0, L, 0.0]), np.array([0, 0, L * 1.0])


# ------------------------------------------------------------------ neighbors

def test_get_distance_orthorhombic_matches_image_search(orc):
    rng = np.random.default_rng(0)
    a, b, c = np.array([9.1, 0, 0]), np.array([0, 10.3, 0]), np.array([0, 0, 8.7])
    for _ in range(200):
        pi, pj = rng.uniform(-5, 15, 3), rng.uniform(-5, 15, 3)
        dist, d, _ = orc.get_distance(pi, pj, a, b, c)
        best = min((np.linalg.norm(pj - pi + i * a + j * b + k * c), (i, j, k))
                   for i, j, k in itertools.product(range(-3, 4), repeat=3))
        assert abs(d - best[0]) < 1e-12
        assert abs(np.linalg.norm(dist) - d) < 1e-12


def test_get_distance_triclinic_matches_image_search(orc):
    rng = np.random.default_rng(1)
    a, b, c = np.array([7.0, 0.3, -0.2]), np.array([0.4, 6.5, 0.1]), np.array([-0.3, 0.2, 7.4])
    for _ in range(200):
        pi, pj = rng.uniform(0, 7, 3), rng.uniform(0, 7, 3)
        dist, d, _ = orc.get_distance(pi, pj, a, b, c)
        best = min(np.linalg.norm(pj - pi + i * a + j * b + k * c)
                   for i, j, k in itertools.product(range(-3, 4), repeat=3))
        assert abs(d - best) < 1e-12


def test_number_of_unit_cells(orc):
    for L, rc in [(10.7, 3.7), (5.7, 3.7), (7.39, 3.7), (20.0, 4.0)]:
        idx = orc.number_of_unit_cells(*_lat(L), rc)
        assert list(idx) == [int(np.ceil(2 * rc / L))] * 3


def test_diamond_shell_counts(orc, synth):
    """Perfect diamond a=3.567: shells 4 @1.545, 12 @2.522, 12 @2.958, 6 @3.567 (< 3.7)."""
    pos, box, sp = synth.diamond_supercell(3, noise=0.0)
    nb = orc.build_neighbors(pos, len(pos), *box, 3.7, sp, False)
    assert np.all(nb["n_neigh"] == 35)
    start = np.concatenate([[0], np.cumsum(nb["n_neigh"])])
    for i in range(len(pos)):
        assert nb["neighbors_list"][start[i]] == i + 1  # self first
        assert nb["rjs"][start[i]] == 0.0
        r = np.sort(nb["rjs"][start[i] + 1:start[i + 1]])
        assert np.allclose(r[:4], 3.567 * np.sqrt(3) / 4)
        assert np.allclose(r[-6:], 3.567)


def test_cell_list_and_brute_force_agree_as_sets(orc, synth):
    pos, box, sp, _ = synth.random_packing(300, 2.5, 1.2, seed=3)
    cell = orc.build_neighbors(pos, len(pos), *box, 3.7, sp, False)
    brute = orc.build_neighbors(pos, len(pos), *box, 3.7, sp, True)
    assert np.array_equal(cell["n_neigh"], brute["n_neigh"])
    s = np.concatenate([[0], np.cumsum(cell["n_neigh"])])
    for i in range(len(pos)):
        a = cell["neighbors_list"][s[i]:s[i + 1]]
        b = brute["neighbors_list"][s[i]:s[i + 1]]
        assert a[0] == b[0] == i + 1
        assert sorted(a) == sorted(b)
        # brute force visits j in index order
        assert list(b[1:]) == sorted(b[1:])


def test_small_cell_supercell_path(orc, synth):
    """A 5.7 A cell needs 2x2x2 replicas (read_xyz.f90:133-147); neighbors of each site then
    match a direct image sum."""
    pos, box, sp, _ = synth.random_packing(24, 2.0, 1.2, seed=5, strain=0.03)
    idx = orc.number_of_unit_cells(*box, 3.7)
    assert np.all(idx >= 2)
    pos_sc, sp_sc, a, b, c = orc.set_supercell(pos, sp, idx, *box)
    nb = orc.build_neighbors(pos_sc, len(pos), a, b, c, 3.7, sp_sc, True)
    for i in range(len(pos)):
        cnt = 0
        for j in range(len(pos)):
            for n1, n2, n3 in itertools.product(range(-3, 4), repeat=3):
                d = np.linalg.norm(pos[j] - pos[i] + n1 * box[0] + n2 * box[1] + n3 * box[2])
                if 0 < d < 3.7:
                    cnt += 1
        assert nb["n_neigh"][i] == cnt + 1


# ------------------------------------------------------------------ descriptor definition

def _mp_w(am):
    import mpmath as mp
    mp.mp.dps = 60
    S = mp.matrix(am, am)
    for i in range(am):
        for j in range(am):
            a, b = i + 1, j + 1
            S[i, j] = mp.sqrt((2 * a + 5) * (2 * b + 5)) / (a + b + 5)
    E, Q = mp.eighe(S)
    W = Q * mp.diag([1 / mp.sqrt(e) for e in E]) * Q.T
    return W


def test_poly3_orthonormaliser_matches_mpmath(orc):
    W = orc.poly3_w(8)
    Wm = _mp_w(8)
    ref = np.array([[float(Wm[i, j]) for j in range(8)] for i in range(8)])
    assert np.max(np.abs(W - ref) / np.maximum(np.abs(ref), 1.0)) < 1e-14


@pytest.mark.parametrize("r", [0.0, 0.9, 1.5, 2.4, 3.1, 3.3, 3.55, 3.69])
def test_radial_projection_matches_mpmath_integral(orc, synth, r):
    """R_n(r) is defined as an integral over the orthonormal poly3 basis; evaluate it with
    mpmath at 30 digits and compare with the Gauss-Legendre tables."""
    import mpmath as mp
    hyp = synth.carbon_hypers()
    H = orc.Hypers(hyp)
    central = r == 0.0
    R, _ = orc.radial(H, 0, r, central=central)
    mp.mp.dps = 30
    Wm = _mp_w(8)
    mp.mp.dps = 30
    rc, xs = mp.mpf(3.7), mp.mpf(3.2) / mp.mpf(3.7)
    x0 = mp.mpf(r) / rc
    sig = mp.mpf(0.5) / rc
    sf = (1 - xs) / 4
    g = 1 + 2 * x0 ** 3 - 3 * x0 ** 2
    A = g / sig
    for n in range(8):
        def gn(x):
            return sum(Wm[n, a - 1] * mp.sqrt(2 * a + 5) * (1 - x) ** (a + 2) for a in range(1, 9))
        f_in = lambda x: gn(x) * mp.exp(-(x - x0) ** 2 / (2 * sig ** 2))
        f_bf = lambda x: f_in(x) * mp.exp(-(x - xs) ** 2 / (2 * sf ** 2))
        val = A * (mp.quad(f_in, [0, xs / 2, xs]) + mp.quad(f_bf, [xs, 1]))
        assert abs(R[n] - float(val)) < 1e-12 * max(1.0, abs(float(val))), (n, R[n], float(val))


def test_radial_derivative_finite_difference(orc, synth):
    hyp = synth.carbon_hypers()
    hyp["atom_sigma_r_scaling"] = [0.1]
    hyp["amplitude_scaling"] = [1.5]
    hyp["radial_enhancement"] = 2
    H = orc.Hypers(hyp)
    for r in (1.1, 2.0, 3.0, 3.4):
        R, dR = orc.radial(H, 0, r)
        h = 1e-6
        Rp, _ = orc.radial(H, 0, r + h)
        Rm, _ = orc.radial(H, 0, r - h)
        assert np.allclose((Rp - Rm) / (2 * h), dR, rtol=1e-6, atol=1e-8)


def test_angular_bessel_ratio_and_harmonics(orc, synth):
    from scipy.special import spherical_in, sph_harm_y
    hyp = synth.carbon_hypers()
    H = orc.Hypers(hyp)
    rng = np.random.default_rng(2)
    for r in (0.6, 1.3, 2.2, 3.6):
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        A, dA = orc.angular(H, 0, r, u)
        k = r * r / 0.25
        th, ph = np.arccos(u[2]), np.arctan2(u[1], u[0])
        for l in range(9):
            f = spherical_in(l, k) / spherical_in(0, k)
            for m in range(0, l + 1):
                Y = sph_harm_y(l, m, th, ph)
                # real harmonics: m=0 -> Y_l0; m>0 -> sqrt2 (-1)^m Re/Im Y_lm (Condon-Shortley)
                if m == 0:
                    ref = [Y.real]
                    got = [A[l * l]]
                else:
                    ref = [np.sqrt(2) * (-1) ** m * Y.real, np.sqrt(2) * (-1) ** m * Y.imag]
                    got = [A[l * l + 2 * m - 1], A[l * l + 2 * m]]
                assert np.allclose(got, f * np.array(ref), rtol=1e-10, atol=1e-13), (r, l, m)
        # gradient by finite differences on the neighbor vector
        h = 1e-6
        v = r * u
        for x in range(3):
            vp, vm = v.copy(), v.copy()
            vp[x] += h
            vm[x] -= h
            Ap, _ = orc.angular(H, 0, np.linalg.norm(vp), vp / np.linalg.norm(vp))
            Am, _ = orc.angular(H, 0, np.linalg.norm(vm), vm / np.linalg.norm(vm))
            assert np.allclose((Ap - Am) / (2 * h), dA[:, x], atol=1e-7)


# ------------------------------------------------------------------ descriptor properties

def _isolated(orc, synth, coords, hyp=None):
    hyp = hyp or synth.carbon_hypers()
    H = orc.Hypers(hyp)
    coords = np.asarray(coords, float)
    box = np.diag([60.0, 60.0, 60.0])
    sp = np.ones(len(coords), np.int32)
    nb = orc.build_neighbors(coords + 30.0, len(coords), *box, 3.7, sp, False)
    mask = np.ones((len(nb["rjs"]), 1), bool)
    soap, der = orc.get_soap(H, nb["n_neigh"], mask, nb["rjs"], nb["thetas"], nb["phis"])
    return H, nb, soap, der


def test_single_atom_is_central_term_only(orc, synth):
    H, nb, soap, _ = _isolated(orc, synth, [[0, 0, 0]])
    Rc, _ = orc.radial(H, 0, 0.0, central=True)
    c = Rc / np.sqrt(4 * np.pi)
    p = []
    for n in range(8):
        for npr in range(n, 8):
            mult = 1.0 if n == npr else np.sqrt(2.0)
            for l in range(9):
                p.append(mult * c[n] * c[npr] if l == 0 else 0.0)
    p = np.array(p)
    assert np.allclose(soap[0], p / np.linalg.norm(p), atol=1e-14)


def test_soap_unit_norm_and_rotation_invariance(orc, synth):
    rng = np.random.default_rng(4)
    X = rng.normal(size=(7, 3)) * 1.1
    _, _, q1, _ = _isolated(orc, synth, X)
    Qr, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    _, _, q2, _ = _isolated(orc, synth, X @ Qr.T)
    assert np.allclose(np.linalg.norm(q1, axis=1), 1.0, atol=1e-14)
    assert np.allclose(q1, q2, atol=1e-11)


def test_soap_cart_der_finite_difference(orc, synth):
    rng = np.random.default_rng(6)
    X = rng.normal(size=(5, 3)) * 1.2
    H, nb, q, der = _isolated(orc, synth, X)
    start = np.concatenate([[0], np.cumsum(nb["n_neigh"])])
    h = 1e-6
    for i in range(len(X)):
        for k in range(start[i], start[i + 1]):
            j = nb["neighbors_list"][k] - 1
            for x in range(3):
                Xp, Xm = X.copy(), X.copy()
                Xp[j, x] += h
                Xm[j, x] -= h
                qp = _isolated(orc, synth, Xp)[2][i]
                qm = _isolated(orc, synth, Xm)[2][i]
                assert np.allclose((qp - qm) / (2 * h), der[k, :, x], atol=2e-8)


def _compress_np(q, der, pi, pj, pel, dim_out):
    """q_c = P q / |P q| and dq_c = (I - q_c q_c^T) P dq / |P q| from the uncompressed normalised
    descriptor (the normalisation of p cancels: P p / |P p| = P q / |P q|)."""
    P = np.zeros((dim_out, q.shape[1]))
    np.add.at(P, (np.asarray(pi) - 1, np.asarray(pj) - 1), pel)
    pq = q @ P.T
    nr = np.linalg.norm(pq, axis=1)
    qc = pq / nr[:, None]
    return P, qc, nr


def test_soap_compression_matches_the_projection(orc, synth):
    """The oracle's compression (the P_transformation of read_gap.f90:489-559: q = P p / |P p|)
    against the same projection applied to its uncompressed output, for the identity, a selection
    of components (the old index-list format) and a random sparse P with repeated rows; the
    compressed derivatives against finite differences of the compressed descriptor."""
    rng = np.random.default_rng(12)
    X = rng.normal(size=(6, 3)) * 1.2
    hyp = synth.carbon_hypers()
    H, nb, q, der = _isolated(orc, synth, X, hyp)
    D = q.shape[1]
    start = np.concatenate([[0], np.cumsum(nb["n_neigh"])])
    sel = np.sort(rng.choice(D, 120, replace=False)) + 1
    nnz = 400
    cases = [(np.arange(1, D + 1), np.arange(1, D + 1), np.ones(D), D),
             (np.arange(1, 121), sel, np.ones(120), 120),
             (rng.integers(1, 91, nnz), rng.integers(1, D + 1, nnz), rng.normal(size=nnz), 90)]
    for pi, pj, pel, dim_out in cases:
        hc = dict(hyp, compress=(pi, pj, pel, dim_out))
        _, _, qc, derc = _isolated(orc, synth, X, hc)
        P, qref, nr = _compress_np(q, der, pi, pj, pel, dim_out)
        assert qc.shape == (len(X), dim_out)
        assert np.max(np.abs(qc - qref)) < 1e-13
        for i in range(len(X)):
            for k in range(start[i], start[i + 1]):
                pd = P @ der[k]  # (dim_out, 3)
                ref = (pd - np.outer(qref[i], qref[i] @ pd)) / nr[i]
                assert np.max(np.abs(derc[k] - ref)) < 1e-11, (dim_out, i, k)
    # finite differences of the random compression
    pi, pj, pel, dim_out = cases[2]
    hc = dict(hyp, compress=(pi, pj, pel, dim_out))
    _, _, qc, derc = _isolated(orc, synth, X, hc)
    h = 1e-6
    for i, k in ((0, start[0] + 1), (3, start[3] + 2)):
        j = nb["neighbors_list"][k] - 1
        for x in range(3):
            Xp, Xm = X.copy(), X.copy()
            Xp[j, x] += h
            Xm[j, x] -= h
            qp = _isolated(orc, synth, Xp, hc)[2][i]
            qm = _isolated(orc, synth, Xm, hc)[2][i]
            assert np.allclose((qp - qm) / (2 * h), derc[k, :, x], atol=2e-8)


# ------------------------------------------------------------------ GAP and dynamics

def test_gap_forces_virial_fd_and_invariance(orc, synth):
    hyp = synth.carbon_hypers()
    H = orc.Hypers(hyp)
    pos, box, sp = synth.diamond_supercell(2, seed=11)
    N = len(pos)
    nb0 = orc.build_neighbors(pos, N, *box, 3.7, sp, False)
    q0, _ = orc.get_soap(H, nb0["n_neigh"], np.ones((len(nb0["rjs"]), 1), bool), nb0["rjs"],
                         nb0["thetas"], nb0["phis"], derivatives=False)
    model = synth.gap_model(q0, 40, seed=2)

    def ev(p, bx):
        nb = orc.build_neighbors(p, N, *bx, 3.7, sp, False)
        return orc.get_gap_soap(H, N, nb, sp, 0, model["alphas"], model["Qs"], 1.0, 4.0)

    e, f, v = ev(pos, box)
    h = 1e-5
    for i, x in [(0, 0), (7, 2), (33, 1)]:
        pp, pm = pos.copy(), pos.copy()
        pp[i, x] += h
        pm[i, x] -= h
        fd = -(ev(pp, box)[0].sum() - ev(pm, box)[0].sum()) / (2 * h)
        assert abs(fd - f[i, x]) < 1e-9
    for a, b in [(0, 0), (1, 2)]:
        Fm = np.eye(3)
        Fm[a, b] += 1e-6
        Fp = ev(pos @ Fm.T, box @ Fm.T)[0].sum()
        Fm2 = np.eye(3)
        Fm2[a, b] -= 1e-6
        Fn = ev(pos @ Fm2.T, box @ Fm2.T)[0].sum()
        assert abs(-(Fp - Fn) / 2e-6 - 0.5 * (v[a, b] + v[b, a])) < 1e-8
    # translation and permutation invariance
    e2, f2, _ = ev(pos + np.array([0.3, -1.1, 2.0]), box)
    assert np.allclose(e, e2, atol=1e-12) and np.allclose(f, f2, atol=1e-12)
    perm = np.random.default_rng(0).permutation(N)
    e3, f3, _ = ev(pos[perm], box)
    assert np.allclose(e[perm], e3, atol=1e-12) and np.allclose(f[perm], f3, atol=1e-12)
    assert abs(f.sum(axis=0)).max() < 1e-12


def test_velocity_verlet_matches_formula(orc):
    rng = np.random.default_rng(0)
    n = 5
    pos, vel, F, Fp = (rng.normal(size=(n, 3)) for _ in range(4))
    m = rng.uniform(1, 3, n)
    pos0, vel0 = pos.copy(), vel.copy()
    pprev = np.zeros_like(pos)
    Fp0 = Fp.copy()
    dtp = orc.velocity_verlet(pos, pprev, vel, F, Fp, m, 0.7, 0.5, False)
    v_ref = vel0 + 0.5 * (F + Fp0) / m[:, None] * 0.5
    assert np.allclose(vel, v_ref, rtol=0, atol=1e-15)
    assert np.allclose(pos, pos0 + v_ref * 0.7 + 0.5 * F / m[:, None] * 0.49, atol=1e-15)
    assert np.array_equal(pprev, pos0) and np.array_equal(Fp, F) and dtp == 0.7


def test_mc_acceptance_uses_single_precision_kb(orc):
    kb32 = float(np.float32(8.617333262e-5))
    p = orc.mc_move_acceptance(0.1, 0.0, 2000.0)
    assert p == np.exp(-0.1 / (kb32 * 2000.0))
    assert orc.mc_move_acceptance(-1.0, 0.0, 300.0) == 1.0


def test_local_property_predict_pinned_by_gap_forces_and_formula(orc, synth):
    """local_property_predict (local_properties.f90:46-147). With V0 = 0, positive alphas (no
    clipping) and an integer zeta, V equals the GAP energies and minus the sum of V_der over the
    pairs that end on atom j equals the GAP force on j (the force path is pinned by finite
    differences above); each site's pair derivatives sum to zero. With a negative V0 and a zeta
    4 + 5e-6 (an integer for gap.f90's 1e-5 test, not for the 1e-10 test of
    local_properties.f90:76-77), V matches a direct evaluation, clipped sites get 0 and so do
    their derivatives."""
    hyp = synth.carbon_hypers()
    H = orc.Hypers(hyp)
    pos, box, sp = synth.diamond_supercell(3, seed=13)
    N = len(pos)
    nb = orc.build_neighbors(pos, N, *box, 3.7, sp, False)
    P = len(nb["rjs"])
    q, der = orc.get_soap(H, nb["n_neigh"], np.ones((P, 1), bool), nb["rjs"], nb["thetas"], nb["phis"])
    model = synth.gap_model(q, 40, seed=4)
    Qs = model["Qs"]
    a_pos = np.abs(model["alphas"])
    V, Vd = orc.local_property_predict(q, Qs, a_pos, 0.0, 1.0, 4.0, der, nb["n_neigh"])
    e, f, _ = orc.soap_energy_and_forces(q, der, a_pos, 1.0, 4.0, 0.0, Qs, nb["n_neigh"], nb["neighbors_list"],
                                         nb["xyz"], n_sites0=N)
    assert np.max(np.abs(V - e)) <= 1e-14 * np.max(np.abs(e))
    F = np.zeros((N, 3))
    np.add.at(F, (nb["neighbors_list"] - 1) % N, -Vd)
    assert np.max(np.abs(F - f)) <= 1e-12 * np.max(np.abs(f))
    start = np.concatenate([[0], np.cumsum(nb["n_neigh"])])
    sums = np.array([Vd[start[i]:start[i + 1]].sum(0) for i in range(N)])
    assert np.max(np.abs(sums)) <= 1e-12 * np.max(np.abs(Vd))
    # clipping and the local-property integer-zeta rule
    K = q @ Qs.T
    assert K.min() > 0.0
    zeta, d = 4.0 + 5e-6, 1.3
    raw = d * d * (K ** zeta) @ model["alphas"]
    V0 = -np.median(raw)
    V2, Vd2 = orc.local_property_predict(q, Qs, model["alphas"], V0, d, zeta, der, nb["n_neigh"])
    ref = np.maximum(raw + V0, 0.0)
    assert np.max(np.abs(V2 - ref)) <= 1e-13 * np.max(np.abs(raw))
    clipped = V2 == 0.0
    assert 0 < clipped.sum() < N
    for i in np.nonzero(clipped)[0]:
        assert np.all(Vd2[start[i]:start[i + 1]] == 0.0)
    # the integer-power path would differ by more than the rounding
    raw_int = d * d * (K ** 4) @ model["alphas"]
    assert np.max(np.abs(raw_int - raw)) > 1e3 * 1e-13 * np.max(np.abs(raw))


def _sio2_box(synth, n=192, seed=41):
    return synth.random_packing(n, 2.2, {("Si", "O"): 1.4, ("O", "O"): 2.2, ("Si", "Si"): 2.5},
                                {"Si": 1 / 3, "O": 2 / 3}, seed=seed)[:3]


def _pair_term_fd(orc, pos, box, sp, rc, term):
    """Forces and virial of a pair term against central differences of the total energy (the sum
    of the site energies) over atom moves and homogeneous strains."""
    N = len(pos)

    def ev(p, bx):
        nb = orc.build_neighbors(p, N, *bx, rc, sp, False)
        return term(nb)

    e, f, v = ev(pos, box)
    h = 1e-5
    for i, x in [(0, 0), (17, 2), (101, 1)]:
        pp, pm = pos.copy(), pos.copy()
        pp[i, x] += h
        pm[i, x] -= h
        fd = -(ev(pp, box)[0].sum() - ev(pm, box)[0].sum()) / (2 * h)
        assert abs(fd - f[i, x]) < 1e-7 * max(1.0, np.abs(f).max()), (i, x, fd, f[i, x])
    for a, b in [(0, 0), (1, 2)]:
        Fp, Fn = np.eye(3), np.eye(3)
        Fp[a, b] += 1e-6
        Fn[a, b] -= 1e-6
        d = -(ev(pos @ Fp.T, box @ Fp.T)[0].sum() - ev(pos @ Fn.T, box @ Fn.T)[0].sum()) / 2e-6
        assert abs(d - 0.5 * (v[a, b] + v[b, a])) < 1e-6 * max(1.0, np.abs(v).max()), (a, b, d, v)
    assert abs(f.sum(axis=0)).max() < 1e-10 * max(1.0, np.abs(f).max())
    return e, f, v


def test_2b_energy_forces_virial_finite_differences(orc, synth):
    """get_2b_energy_and_forces (gap.f90:329-460) on Si-O pairs of a SiO2 box: the site forces
    are minus the gradient of the summed site energies (each pair counted from both ends) and the
    halved pair virial minus its strain derivative; sites of other species get e0 and no force."""
    pos, box, sp = _sio2_box(synth)
    rng = np.random.default_rng(3)
    M = 12
    alphas, cutoff, Qs = rng.normal(size=M) * 0.1, rng.uniform(0.5, 1.0, M), np.linspace(1.3, 3.8, M)
    args = dict(alphas=alphas, cutoff=cutoff, rcut=4.0, buffer=0.6, delta=1.1, sigma=0.4, e0=0.05, Qs=Qs)
    e, f, _ = _pair_term_fd(orc, pos, box, sp, 4.0,
                            lambda nb: orc.get_2b_energy_and_forces(nb, sp, 1, 2, **args))
    nb = orc.build_neighbors(pos, len(pos), *box, 4.0, sp, False)
    e_oo, f_oo, _ = orc.get_2b_energy_and_forces(nb, sp, 2, 2, **args)  # O-O term: Si sites untouched
    assert np.all(e_oo[sp == 1] == 0.05) and np.all(f_oo[sp == 1] == 0.0)
    assert np.any(e_oo[sp == 2] != 0.05)


def test_core_pot_spline_energy_forces_virial(orc, synth):
    """get_core_pot_energy_and_forces (gap.f90:552-686) with a clamped cubic spline of a smooth
    repulsion: the spline reproduces its knots, and forces and virial are consistent with the
    energy (finite differences)."""
    pos, box, sp = _sio2_box(synth)
    x = np.linspace(0.8, 3.5, 40)
    Vk = 5.0 * np.exp(-2.0 * x) * (1.0 - x / 3.5) ** 2
    dV = lambda r: 5.0 * np.exp(-2.0 * r) * ((1 - r / 3.5) ** 2 * -2.0 - 2.0 / 3.5 * (1 - r / 3.5))
    yp1, ypn = dV(x[0]), dV(x[-1])
    y2 = orc.spline_second_derivatives(x, Vk, yp1, ypn)
    e, f, v = _pair_term_fd(orc, pos, box, sp, 4.0,
                            lambda nb: orc.get_core_pot_energy_and_forces(nb, sp, 1, 2, x, Vk, yp1, ypn, y2))
    # a two-atom box at knot distances returns the tabulated values (1/2 per atom)
    for r in (x[5], x[17]):
        p2 = np.array([[1.0, 1.0, 1.0], [1.0 + r, 1.0, 1.0]])
        b2 = np.eye(3) * 12.0
        nb2 = orc.build_neighbors(p2, 2, *b2, 4.0, np.array([1, 2], np.int32), False)
        e2, _, _ = orc.get_core_pot_energy_and_forces(nb2, np.array([1, 2]), 1, 2, x, Vk, yp1, ypn, y2)
        k = int(np.argmin(np.abs(x - r)))
        assert abs(e2.sum() - Vk[k]) < 1e-12


@pytest.mark.parametrize("kernel", ["exp", "pol"])
def test_3b_energy_forces_virial_finite_differences(orc, synth, kernel):
    """get_3b_energy_and_forces (gap.f90:756-1015) for O-centred Si-O-Si-like triplets (centre O,
    neighbors O and Si in either order) with both kernels: forces on the three atoms of every
    triplet and the virial against finite differences of the summed site energies."""
    pos, box, sp = _sio2_box(synth, seed=45)
    rng = np.random.default_rng(5)
    M = 10
    Qs = np.stack([rng.uniform(3.0, 6.5, M), rng.uniform(0.0, 2.0, M), rng.uniform(2.0, 5.5, M)], axis=1)
    sigma = np.array([1.0, 1.0, 1.2]) * (3.0 if kernel == "pol" else 1.0)
    args = dict(alphas=rng.normal(size=M) * 0.05, cutoff=rng.uniform(0.5, 1.0, M), rcut=3.5, buffer=0.5,
                delta=0.9, sigma=sigma, e0=0.02, Qs=Qs, kernel=kernel)
    e, f, v = _pair_term_fd(orc, pos, box, sp, 3.5, lambda nb: orc.get_3b_energy_and_forces(nb, sp, 2, 2, 1, **args))
    assert np.all(e[sp == 1] == 0.02)  # Si centres untouched
    assert np.abs(f).max() > 0.0
