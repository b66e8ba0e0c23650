"""Host-side checks of libtgap (no GPU): the C ABI loads and exports every symbol declared in
include/*.h, and the host-computed pieces (binary128 orthonormaliser, unit-cell count,
species mapping) agree with independent computations."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            src = open(os.path.join(inc, f)).read()
            names |= set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(tgap_\w+)\s*\(", src, re.M))
    return names


def test_library_exports_every_declared_symbol(tg):
    from turbogap_b200 import native
    L = native.lib()
    names = _declared_symbols()
    assert len(names) >= 30
    for n in sorted(names):
        assert hasattr(L, n), n
    assert L.tgap_version().startswith(b"tgap-b200")


def test_create_without_device_fails_cleanly(tg):
    import torch
    if torch.cuda.is_available():
        return
    from turbogap_b200 import native
    h = C.c_void_p()
    st = native.lib().tgap_create(0, C.byref(h))
    assert st == 2 and not h.value  # TGAP_ERR_CUDA, no context


def test_poly3_orthonormaliser_binary128(tg, orc):
    from turbogap_b200 import native
    for am in (4, 8, 10):
        W = np.zeros(am * am)
        assert native.lib().tgap_debug_poly3_w(am, native.ptr(W)) == 0
        Wo = orc.poly3_w(am)
        assert np.max(np.abs(W.reshape(am, am) - Wo) / np.maximum(np.abs(Wo), 1.0)) < 1e-13


def test_number_of_unit_cells_matches_oracle(tg, orc):
    rng = np.random.default_rng(0)
    for _ in range(50):
        box = np.diag(rng.uniform(4, 30, 3)) + rng.uniform(-0.5, 0.5, (3, 3))
        rc = rng.uniform(2, 6)
        idx = tg.api.Context.number_of_unit_cells(box[0], box[1], box[2], rc)
        assert list(idx) == list(orc.number_of_unit_cells(box[0], box[1], box[2], rc))


@pytest.mark.parametrize("n", [50, 51, 1])
def test_host_velocity_verlet_matches_oracle(tg, orc, n):
    """tgap_velocity_verlet_host (host arrays) against the oracle's velocity_verlet
    (md_utils.f90:486-532) over a first step and two later ones, and its refusal of non-finite
    forces before touching any array; atom counts that fill the pairs of atoms exactly and that
    leave one atom for the scalar tail."""
    from turbogap_b200 import native
    L = native.lib()
    rng = np.random.default_rng(3)
    m = rng.uniform(1.0, 16.0, n) * 103.6426965268
    x = rng.normal(size=(n, 3)) * 5.0
    v = rng.normal(size=(n, 3)) * 0.01
    xo, vo = x.copy(), v.copy()
    fp, fpo, xpo = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))
    xp = np.zeros((n, 3))
    for k in range(3):
        f = rng.normal(size=(n, 3))
        assert L.tgap_velocity_verlet_host(n, native.ptr(x), native.ptr(xp), native.ptr(v), native.ptr(f),
                                           native.ptr(fp), native.ptr(m), 0.5, 0.5, int(k == 0)) == 0
        orc.velocity_verlet(xo, xpo, vo, f, fpo, m, 0.5, 0.5, k == 0)
        assert np.max(np.abs(x - xo)) < 1e-13
        assert np.max(np.abs(v - vo)) < 1e-15
        assert np.array_equal(fp, fpo) and np.array_equal(xp, xpo)
    f[min(7, n - 1), 1] = np.nan
    x0 = x.copy()
    assert L.tgap_velocity_verlet_host(n, native.ptr(x), None, native.ptr(v), native.ptr(f), native.ptr(fp),
                                       native.ptr(m), 0.5, 0.5, 0) == 8  # TGAP_ERR_NUMERIC
    assert np.array_equal(x, x0)


def test_assign_species(tg):
    out = tg.api.assign_species(["Si", "O"], ["O", "Si", "Si", "C", "O"])
    assert list(out) == [2, 1, 1, 0, 2]
    import pytest
    with pytest.raises(tg.TgapError):
        tg.api.assign_species(["C", "C"], ["C"])


def test_package_exports_the_device_api(tg):
    """Every host-side class of the device API resolves from the package (no GPU needed)."""
    for name in ("Context", "Model", "System", "MD", "MC", "assign_species"):
        assert callable(getattr(tg, name)), name


def test_mc_proposals_stay_in_the_ball(tg):
    atoms, d, u = tg.synth.mc_proposals(100, 5000, 0.2, seed=3)
    assert atoms.min() >= 0 and atoms.max() < 100
    r = np.linalg.norm(d, axis=1)
    assert r.max() <= 0.2 + 1e-12
    # uniform in the ball: P(r < R/2) = 1/8
    assert abs(np.mean(r < 0.1) - 0.125) < 0.02
    assert u.min() >= 0.0 and u.max() < 1.0


def test_screen_reference_trainer_learns_a_smooth_target():
    """The numpy reference of the device trainer (minibatch Adam on the screen network) fits a
    smooth function of its inputs; its FP32 gradients agree with the FP64 ones."""
    import screen_ref
    rng = np.random.default_rng(0)
    z = rng.normal(size=(3000, 8)).astype(np.float32)
    t = (np.sin(1.5 * z[:, 0]) + 0.3 * z[:, 1] ** 2).astype(np.float32)
    t = (t - t.mean()) / t.std()
    p0 = {"w1": rng.normal(size=(32, 8)) * 0.5, "b1": np.zeros(32), "w2": rng.normal(size=(32, 32)) * 0.25,
          "b2": np.zeros(32), "w3": rng.normal(size=32) * 0.2, "b3": 0.0}
    l64, g64 = screen_ref.loss_and_grad(p0, z, t)
    l32, g32 = screen_ref.loss_and_grad(p0, z, t, np.float32)
    assert abs(l32 - l64) < 1e-5 * l64
    for k in g64:
        assert np.max(np.abs(np.asarray(g32[k]) - g64[k])) < 1e-4 * np.max(np.abs(g64[k])) + 1e-7, k
    order = np.stack([rng.permutation(len(t)) for _ in range(30)])
    p = screen_ref.adam_train(p0, z, t, order, 30, 256, 3e-3)
    loss, _ = screen_ref.loss_and_grad(p, z, t)
    assert loss < 0.2 and loss < 0.2 * l64, (loss, l64)


def test_bf16_round_is_round_to_nearest_even():
    import screen_ref
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 3.14159], np.float32)
    r = screen_ref.bf16_round(x)
    assert r[0] == 1.0
    assert r[1] == 1.0  # tie to even
    assert r[2] == np.float32(1.0 + 2.0 ** -6)
    assert r[3] == -2.5
    assert abs(r[4] - 3.14159) < 2 ** -7 * 4


def _write_model_files(d, rng):
    """A .gap file with one block of each kind and its sparse-set files (TurboGAP's layout)."""
    D, M = 12, 5
    Qs = rng.random((M, D))
    alphas = rng.normal(size=M)
    (d / "soap.alphas").write_text("".join(f"{a:.17g}\n" for a in alphas))
    (d / "soap.desc").write_text("".join(f"{q:.17g}\n" for q in Qs.ravel()))  # descriptor index fastest
    a2, c2, q2 = rng.normal(size=4), rng.random(4), np.linspace(1.0, 3.0, 4)
    (d / "b2.alphas").write_text("".join(f"{a:.17g} {c:.17g}\n" for a, c in zip(a2, c2)))
    (d / "b2.desc").write_text("".join(f"{q:.17g}\n" for q in q2))
    a3, c3, q3 = rng.normal(size=3), rng.random(3), rng.random((3, 3)) * 4
    (d / "b3.alphas").write_text("".join(f"{a:.17g}, {c:.17g}\n" for a, c in zip(a3, c3)))
    (d / "b3.desc").write_text("".join(f"{q:.17g}\n" for q in q3.ravel()))
    x = np.linspace(0.5, 3.0, 11)
    V = 4.0 * np.exp(-2.0 * x)
    (d / "core.dat").write_text(f"11 1.0e31 0.0\n" + "".join(f"{a:.17g} {b:.17g}\n" for a, b in zip(x, V)))
    (d / "model.gap").write_text(f"""# a model of every kind
gap_beg soap_turbo
  n_species = 2
  species = C H
  rcut = 3.7 3.0
  buffer = 0.5 0.0
  atom_sigma_r = 0.5 0.4
  atom_sigma_t = 0.5 0.4
  n_max = 4 2
  l_max = 3
  zeta = 4.0
  delta = 0.2
  central_species = 1
  alphas_sparse = "soap.alphas"
  desc_sparse = 'soap.desc'
gap_end
! a comment line
gap_beg distance_2b
  delta = 0.5
  sigma = 0.3
  rcut = 4.5
  species1 = C
  species2 = H
  desc_sparse = b2.desc
  alphas_sparse = b2.alphas
gap_end
gap_beg angle_3b
  sigma = 1.0, 2.0, 3.0
  rcut = 3.0
  Z_center = C
  Z1 = C
  Z2 = H
  kernel_type = pol
  desc_sparse = b3.desc
  alphas_sparse = b3.alphas
gap_end
gap_beg core_pot
  species1 = C
  species2 = C
  core_pot_file = core.dat
gap_end
""")
    return dict(Qs=Qs, alphas=alphas, a2=a2, c2=c2, q2=q2, a3=a3, c3=c3, q3=q3, x=x, V=V)


def test_gap_file_reader(tg, tmp_path):
    """read_gap on a file of every model kind: defaults, buffer -> rcut_soft, the sparse-set file
    layouts and the core_pot table (natural start slope replaced by the spline's derivative)."""
    import oracle_lib as orc
    ref = _write_model_files(tmp_path, np.random.default_rng(0))
    g = tg.gap_file.read_gap(str(tmp_path / "model.gap"), base_dir=str(tmp_path))
    assert [len(g[k]) for k in ("soap_turbo", "distance_2b", "angle_3b", "core_pot")] == [1, 1, 1, 1]
    s = g["soap_turbo"][0]
    h = s["hypers"]
    assert h["species"] == ["C", "H"] and h["alpha_max"] == [4, 2] and h["l_max"] == 3
    assert h["rcut_hard"] == [3.7, 3.0] and h["rcut_soft"] == [3.2, 3.0]  # buffer 0 keeps rcut
    assert h["nf"] == [4.0, 4.0] and h["amplitude_scaling"] == [1.0, 1.0] and h["atom_sigma_t_scaling"] == [0.0, 0.0]
    assert s["zeta"] == 4.0 and s["delta"] == 0.2 and s["central_species"] == 1 and s["basis"] == "poly3"
    assert np.array_equal(s["Qs"], ref["Qs"]) and np.array_equal(s["alphas"], ref["alphas"])
    b2 = g["distance_2b"][0]
    assert b2["buffer"] == 0.5 and b2["sigma"] == 0.3 and b2["species2"] == "H"
    assert np.array_equal(b2["alphas"], ref["a2"]) and np.array_equal(b2["cutoff"], ref["c2"])
    assert np.array_equal(b2["Qs"], ref["q2"])
    b3 = g["angle_3b"][0]
    assert b3["kernel_type"] == "pol" and list(b3["sigma"]) == [1.0, 2.0, 3.0] and b3["species_center"] == "C"
    assert np.array_equal(b3["Qs"], ref["q3"]) and b3["delta"] == 1.0
    cp = g["core_pot"][0]
    y2 = orc.spline_second_derivatives(ref["x"], ref["V"], 1.0e31, 0.0)
    assert np.allclose(cp["dVdx2"], y2, rtol=0, atol=1e-12)
    assert cp["ypn"] == 0.0 and abs(cp["yp1"]) < 1e30  # natural start: slope taken from the spline
    assert g["rcut_max"] == 4.5


def test_gap_file_compression(tg, tmp_path):
    """SOAP compression in a model file (read_gap.f90:489-559): a P_transformation block and the
    older index-list format give (P_i, P_j, P_el, dim_out); compress_mode without a file is refused
    when the model is loaded (its recipe is not in the reference sources)."""
    gf = tg.gap_file
    (tmp_path / "p.dat").write_text("4 2 3 5\nP_transformation\n1 3 0.5\n2 7 1.0\n1 9 -2.0\n5 1 1.0\n"
                                    "end_transformation\n")
    pi, pj, pel, d = gf.read_compress_file(str(tmp_path / "p.dat"), 2)
    assert d == 5 and list(pi) == [1, 2, 1, 5] and list(pj) == [3, 7, 9, 1] and list(pel) == [0.5, 1.0, -2.0, 1.0]
    (tmp_path / "old.dat").write_text("8 3 3\n4\n9\n12\n")
    pi, pj, pel, d = gf.read_compress_file(str(tmp_path / "old.dat"), 1)
    assert d == 3 and list(pi) == [1, 2, 3] and list(pj) == [4, 9, 12] and list(pel) == [1.0, 1.0, 1.0]
    (tmp_path / "p1.dat").write_text("8 8 5\nP_transformation\n1 3 0.5\n2 7 1.0\n1 9 -2.0\n5 1 1.0\n"
                                     "end_transformation\n")
    gap = tmp_path / "c.gap"
    gap.write_text("gap_beg soap_turbo\nn_species = 1\nspecies = C\nrcut = 3.7\nn_max = 8\nl_max = 8\n"
                   "atom_sigma_r = 0.5\natom_sigma_t = 0.5\ncompress_soap = .true.\n"
                   "file_compress_soap = p1.dat\ngap_end\n")
    g = gf.read_gap(str(gap), base_dir=str(tmp_path))
    s = g["soap_turbo"][0]
    assert s["compress_soap"] and s["compress"][3] == 5 and list(s["compress"][1]) == [3, 7, 9, 1]
    gap.write_text(gap.read_text().replace("file_compress_soap = p1.dat", "compress_mode = trivial"))
    g = gf.read_gap(str(gap), base_dir=str(tmp_path))
    assert g["soap_turbo"][0]["compress"] is None and g["soap_turbo"][0]["compress_mode"] == "trivial"


def test_extended_xyz_read_and_round_trip(tg, tmp_path):
    """An extended-XYZ frame as TurboGAP files hold them (case-insensitive keys, quoted Lattice,
    Properties with a column to skip, fix flags and masses), then a write/read round trip of two
    frames with velocities, forces, local energies, energy and virial."""
    (tmp_path / "in.xyz").write_text(
        '3\nlattice="10.0 0 0 0 11.0 0 0.5 0 12.0" PROPERTIES=species:S:1:pos:R:3:charge:R:1:fix_atoms:L:3:masses:R:1'
        ' pbc="T T T"\n'
        "C 0.1 0.2 0.3 -0.5 T F F 12.011\n"
        "H 1.0 2.0 3.0 0.25 F F F 1.008\n"
        "C -1.5 0.0 7.25 0.25 F T T 12.011\n")
    (fr,) = tg.xyz.read_xyz(str(tmp_path / "in.xyz"))
    assert fr["n"] == 3 and fr["species"] == ["C", "H", "C"]
    assert np.array_equal(fr["lattice"], [[10, 0, 0], [0, 11, 0], [0.5, 0, 12]])
    assert np.array_equal(fr["positions"][2], [-1.5, 0.0, 7.25])
    assert fr["fix_atom"].tolist() == [[True, False, False], [False, False, False], [False, True, True]]
    assert np.allclose(fr["masses"], [12.011, 1.008, 12.011]) and fr["info"]["pbc"] == "T T T"
    assert list(tg.xyz.species_channels(fr, ["H", "C"])) == [2, 1, 2]
    rng = np.random.default_rng(1)
    frames = []
    for k in range(2):
        frames.append(dict(species=["Si", "O", "O"], positions=rng.random((3, 3)) * 5, lattice=np.eye(3) * 5.1,
                           velocities=rng.normal(size=(3, 3)), forces=rng.normal(size=(3, 3)),
                           local_energy=rng.normal(size=3), energy=float(rng.normal()),
                           virial=rng.normal(size=(3, 3))))
    tg.xyz.write_xyz(str(tmp_path / "out.xyz"), frames)
    back = tg.xyz.read_xyz(str(tmp_path / "out.xyz"))
    assert len(back) == 2
    for a, b in zip(frames, back):
        assert np.array_equal(a["positions"], b["positions"]) and np.array_equal(a["velocities"], b["velocities"])
        assert np.array_equal(a["lattice"], b["lattice"]) and b["species"] == ["Si", "O", "O"]
        assert float(b["info"]["energy"]) == a["energy"]
        v = np.array([float(x) for x in b["info"]["virial"].split()]).reshape(3, 3)
        assert np.array_equal(v, a["virial"])
