"""Host-side mirror of TurboGAP's SOAP/GAP operator interface, backed by libtgap (sm_100a).

Reference routines and their counterparts here (arrays in numpy row-major form, which is the
Fortran column-major layout of the reference read with the first index fastest: positions
(N, 3) == positions(3, N), soap (n_sites, D) == soap(D, n_sites), soap_cart_der (P, D, 3) ==
soap_cart_der(3, D, P), Qs (n_sparse, D) == Qs(D, n_sparse)):

    build_neighbors_list        src/neighbors/neighbors_interface.f90:144   Context.build_neighbors_list
    get_soap (soap_turbo)       src/gap/gap_interface.f90:301-306          Context.get_soap
    get_soap_energy_and_forces  src/gap/gap.f90:39                         Context.get_soap_energy_and_forces
    get_gap_soap                src/gap/gap_interface.f90:41               Context.get_gap_soap
    calculate_gap_soap          src/gap/calculate_gap_soap.f90:171         System.compute (all models)
    velocity_verlet MD step     src/md/md_utils.f90:486                    MD

Errors raise TgapError with the library status (see include/tgap.h), mirroring the points
where the reference would stop.
"""
import ctypes as C

import numpy as np

from . import native as N
from .native import TGAP_FP64, TGAP_MIXED, TgapError, check, ptr  # noqa: F401


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Context:
    """One device, one stream, reusable device buffers (tgap_context)."""

    def __init__(self, device=0):
        self._L = N.lib()
        h = C.c_void_p()
        st = self._L.tgap_create(int(device), C.byref(h))
        if st != 0:
            raise TgapError(st, f"tgap_create(device={device}) failed")
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self._L.tgap_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        check(self._L.tgap_synchronize(self.h), self.h, "synchronize")

    def autotune_set(self, key, value):
        """Fixes one launch choice (tgap_autotune_set): a key of the autotune report, or '*' and a
        suffix for every key ending with it ('*/persist': 0 = one site per warp, 1 = persistent
        work-queue descriptor kernels)."""
        check(self._L.tgap_autotune_set(self.h, key.encode(), int(value)), self.h, "autotune_set")

    def host_register(self, array):
        """Page-locks a numpy array for this context (tgap_host_register): host-buffer calls then
        copy to and from it directly. Keep the array alive until host_unregister."""
        check(self._L.tgap_host_register(self.h, ptr(array), array.nbytes), self.h, "tgap_host_register")

    def host_unregister(self, array):
        check(self._L.tgap_host_unregister(self.h, ptr(array)), self.h, "tgap_host_unregister")

    def autotune_clear(self):
        check(self._L.tgap_autotune_clear(self.h), self.h, "autotune_clear")

    def set_stream(self, stream_handle):
        check(self._L.tgap_set_stream(self.h, C.c_void_p(stream_handle) if stream_handle else None),
              self.h, "set_stream")

    @property
    def kernel_launches(self):
        return int(self._L.tgap_kernel_launches(self.h))

    # ------------------------------------------------------------ reference call surface

    @staticmethod
    def number_of_unit_cells(a, b, c, rcut):
        idx = np.zeros(3, np.int32)
        check(N.lib().tgap_number_of_unit_cells(ptr(_f64(a)), ptr(_f64(b)), ptr(_f64(c)), float(rcut), ptr(idx)))
        return idx

    def build_neighbors_list(self, positions, n_sites, a, b, c, rcut_max, species_supercell,
                             box_small=False, rebuild=True, n_neigh=None, neighbors_list=None,
                             capacity=None):
        """build_neighbors_list: positions (N_sc, 3) of the (replicated) supercell."""
        pos = _f64(positions)
        nsc = pos.shape[0]
        sp = _i32(species_supercell)
        a, b, c = _f64(a), _f64(b), _f64(c)
        if rebuild:
            cap = int(capacity) if capacity else 100 * n_sites  # neighbors_interface.f90:283
            while True:
                nn = np.zeros(n_sites, np.int32)
                nl = np.zeros(cap, np.int32)
                rjs = np.zeros(cap)
                xyz = np.zeros((cap, 3))
                th = np.zeros(cap)
                ph = np.zeros(cap)
                nsp = np.zeros(cap, np.int32)
                npairs = C.c_int64(0)
                st = self._L.tgap_build_neighbors(self.h, n_sites, nsc, ptr(pos), ptr(a), ptr(b), ptr(c),
                                                  int(box_small), float(rcut_max), ptr(sp), 1, ptr(nn), ptr(nl),
                                                  ptr(rjs), ptr(xyz), ptr(th), ptr(ph), ptr(nsp), cap,
                                                  C.byref(npairs))
                if st == 3:  # TGAP_ERR_CAPACITY: grow and retry (check_extend_neighbor_list)
                    cap = int(npairs.value)
                    continue
                check(st, self.h, "tgap_build_neighbors")
                P = int(npairs.value)
                return dict(n_neigh=nn, neighbors_list=nl[:P].copy(), rjs=rjs[:P].copy(), xyz=xyz[:P].copy(),
                            thetas=th[:P].copy(), phis=ph[:P].copy(), neighbor_species=nsp[:P].copy())
        nn = _i32(n_neigh)
        nl = _i32(neighbors_list)
        P = nl.shape[0]
        rjs = np.zeros(P); xyz = np.zeros((P, 3)); th = np.zeros(P); ph = np.zeros(P)
        nsp = np.zeros(P, np.int32)
        npairs = C.c_int64(P)
        check(self._L.tgap_build_neighbors(self.h, n_sites, nsc, ptr(pos), ptr(a), ptr(b), ptr(c), int(box_small),
                                           float(rcut_max), ptr(sp), 0, ptr(nn), ptr(nl), ptr(rjs), ptr(xyz),
                                           ptr(th), ptr(ph), ptr(nsp), P, C.byref(npairs)),
              self.h, "tgap_build_neighbors")
        return dict(n_neigh=nn, neighbors_list=nl, rjs=rjs, xyz=xyz, thetas=th, phis=ph, neighbor_species=nsp)

    def get_soap(self, hypers, n_neigh, mask, rjs, thetas, phis, do_derivatives=True, basis="poly3",
                 scaling_mode="polynomial", compress=None):
        """soap_turbo get_soap. mask: (P, n_species) bool. Returns soap (n_sites, D) and,
        when do_derivatives, soap_cart_der (P, D, 3). compress: (P_i, P_j, P_el[, dim_out]) 1-based
        entries of the compression (D is then the largest P_i)."""
        nn = _i32(n_neigh)
        n_sites = nn.shape[0]
        rjs = _f64(rjs)
        P = rjs.shape[0]
        ns = len(hypers["alpha_max"])
        m = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8).reshape(P, ns).T)
        nmax = int(np.sum(hypers["alpha_max"]))
        D = nmax * (nmax + 1) // 2 * (int(hypers["l_max"]) + 1)
        cp = None
        if compress is not None:
            cp = (np.ascontiguousarray(compress[0], np.int32), np.ascontiguousarray(compress[1], np.int32),
                  _f64(compress[2]))
            D = int(cp[0].max())
        soap = np.zeros((n_sites, D))
        der = np.zeros((P, D, 3)) if do_derivatives else None
        hv = {k: _f64(np.broadcast_to(np.asarray(hypers[k], float), (ns,))) for k in N.HYPER_KEYS}
        am = _i32(hypers["alpha_max"])
        check(self._L.tgap_get_soap(
            self.h, n_sites, ptr(nn), ns, None, None, P, ptr(m), ptr(rjs), ptr(_f64(thetas)), ptr(_f64(phis)),
            ptr(am), int(hypers["l_max"]), ptr(hv["rcut_hard"]), ptr(hv["rcut_soft"]), ptr(hv["nf"]),
            ptr(hv["global_scaling"]), ptr(hv["atom_sigma_r"]), ptr(hv["atom_sigma_r_scaling"]),
            ptr(hv["atom_sigma_t"]), ptr(hv["atom_sigma_t_scaling"]), ptr(hv["amplitude_scaling"]),
            int(hypers.get("radial_enhancement", 0)), ptr(hv["central_weight"]), basis.encode(),
            scaling_mode.encode(), int(do_derivatives), int(cp is not None), 0 if cp is None else len(cp[0]),
            None if cp is None else ptr(cp[0]), None if cp is None else ptr(cp[1]),
            None if cp is None else ptr(cp[2]), ptr(soap), ptr(der)),
            self.h, "tgap_get_soap")
        return soap, der

    def get_soap_energy_and_forces(self, soap, soap_der, alphas, delta, zeta, e0, Qs, n_neigh,
                                   neighbors_list, xyz, do_forces=True, n_sites0=None):
        soap = _f64(soap)
        n_sites, D = soap.shape
        Qs = _f64(Qs)
        M = Qs.shape[0]
        nn = _i32(n_neigh)
        nl = _i32(neighbors_list)
        P = nl.shape[0]
        if n_sites0 is None:
            n_sites0 = n_sites
        en = np.zeros(n_sites)
        fo = np.zeros((n_sites0, 3))
        vir = np.zeros(9)
        check(self._L.tgap_get_soap_energy_and_forces(
            self.h, D, n_sites, M, ptr(soap), ptr(_f64(soap_der)) if do_forces else None, ptr(_f64(alphas)),
            float(delta), float(zeta), float(e0), ptr(Qs), ptr(nn), ptr(nl), ptr(_f64(xyz)), P, int(do_forces),
            int(n_sites0), ptr(en), ptr(fo), ptr(vir)), self.h, "tgap_get_soap_energy_and_forces")
        return en, fo, vir.reshape(3, 3, order="F")

    def get_2b_energy_and_forces(self, nb, species, species1, species2, alphas, cutoff, rcut, buffer, delta, sigma,
                                 e0, Qs, n_sites0=None, do_forces=True):
        """get_2b_energy_and_forces on a neighbor-list dict (n_neigh, rjs, xyz, neighbor_species);
        species per site and species1/2 as channel indices."""
        nn = _i32(nb["n_neigh"])
        n, P = len(nn), int(nn.sum())
        n0 = n if n_sites0 is None else n_sites0
        en, fo, vir = np.zeros(n), np.zeros((n0, 3)), np.zeros(9)
        check(self._L.tgap_get_2b_energy_and_forces(
            self.h, n, P, ptr(_f64(nb["rjs"])), ptr(_f64(nb["xyz"])), len(alphas), ptr(_f64(alphas)),
            ptr(_f64(cutoff)), float(rcut), float(buffer), float(delta), float(sigma), float(e0), ptr(_f64(Qs)),
            ptr(nn), int(do_forces), ptr(_i32(species)), ptr(_i32(nb["neighbor_species"])), int(species1),
            int(species2), n0, ptr(en), ptr(fo), ptr(vir)), self.h, "tgap_get_2b_energy_and_forces")
        return en, fo, vir.reshape(3, 3, order="F")

    def get_3b_energy_and_forces(self, nb, species, species_center, species1, species2, alphas, cutoff, rcut,
                                 buffer, delta, sigma, e0, Qs, kernel="exp", n_sites0=None, do_forces=True):
        """get_3b_energy_and_forces on a neighbor-list dict (with neighbors_list); Qs (n_sparse, 3)."""
        nn = _i32(nb["n_neigh"])
        n, P = len(nn), int(nn.sum())
        n0 = n if n_sites0 is None else n_sites0
        en, fo, vir = np.zeros(n), np.zeros((n0, 3)), np.zeros(9)
        Qf = np.asfortranarray(Qs, dtype=np.float64).ravel(order="F")
        check(self._L.tgap_get_3b_energy_and_forces(
            self.h, n0, n, P, ptr(_f64(nb["rjs"])), ptr(_f64(nb["xyz"])), len(alphas), ptr(_f64(alphas)),
            ptr(_f64(cutoff)), float(rcut), float(buffer), float(delta), ptr(_f64(sigma)), float(e0), ptr(Qf),
            ptr(nn), ptr(_i32(nb["neighbors_list"])), int(do_forces), 1 if kernel == "pol" else 0,
            ptr(_i32(species)), ptr(_i32(nb["neighbor_species"])), int(species_center), int(species1),
            int(species2), ptr(en), ptr(fo), ptr(vir)), self.h, "tgap_get_3b_energy_and_forces")
        return en, fo, vir.reshape(3, 3, order="F")

    def get_core_pot_energy_and_forces(self, nb, species, species1, species2, x, V, yp1, ypn, dVdx2, n_sites0=None,
                                       do_forces=True):
        nn = _i32(nb["n_neigh"])
        n, P = len(nn), int(nn.sum())
        n0 = n if n_sites0 is None else n_sites0
        en, fo, vir = np.zeros(n), np.zeros((n0, 3)), np.zeros(9)
        check(self._L.tgap_get_core_pot_energy_and_forces(
            self.h, len(x), n, P, n0, ptr(_f64(nb["rjs"])), ptr(_f64(nb["xyz"])), ptr(_f64(x)), ptr(_f64(V)),
            float(yp1), float(ypn), ptr(_f64(dVdx2)), ptr(nn), int(do_forces), ptr(_i32(species)),
            ptr(_i32(nb["neighbor_species"])), int(species1), int(species2), ptr(en), ptr(fo), ptr(vir)),
            self.h, "tgap_get_core_pot_energy_and_forces")
        return en, fo, vir.reshape(3, 3, order="F")

    def local_property_predict(self, soap, Qs, alphas, V0, delta, zeta, soap_cart_der=None, n_neigh=None):
        """local_property_predict: soap (n_sites, D), Qs (M, D), soap_cart_der (P, D, 3) or None.
        Returns V (n_sites) and V_der (P, 3) or None."""
        soap = _f64(soap)
        n_sites, D = soap.shape
        Qs = _f64(Qs)
        do_der = soap_cart_der is not None
        nn = _i32(n_neigh) if do_der else None
        P = int(nn.sum()) if do_der else 0
        V = np.zeros(n_sites)
        Vd = np.zeros((max(P, 1), 3))
        check(self._L.tgap_local_property_predict(
            self.h, D, n_sites, Qs.shape[0], ptr(soap), ptr(Qs), ptr(_f64(alphas)), float(V0), float(delta),
            float(zeta), int(do_der), ptr(_f64(soap_cart_der)) if do_der else None, ptr(nn) if do_der else None, P,
            ptr(V), ptr(Vd)), self.h, "tgap_local_property_predict")
        return V, (Vd[:P] if do_der else None)

    def get_gap_soap(self, hypers, n_total_sites, nb, species_supercell, central_species, alphas, Qs, delta,
                     zeta, do_forces=True, precision=TGAP_FP64, energies0=None, forces0=None, want_soap=False):
        """get_gap_soap for one model on a global neighbor list `nb` (dict as returned by
        build_neighbors_list). energies0/forces0 are overwritten for touched sites."""
        hs, keep = N.make_hypers(hypers)
        nn = _i32(nb["n_neigh"])
        n_sites0 = nn.shape[0]
        en = np.zeros(n_total_sites) if energies0 is None else energies0
        fo = np.zeros((n_total_sites, 3)) if forces0 is None else forces0
        vir = np.zeros(9)
        Qs = _f64(Qs)
        D = int(sum(hypers["alpha_max"]))
        D = D * (D + 1) // 2 * (int(hypers["l_max"]) + 1)
        soap = np.zeros((n_sites0, D)) if want_soap else None
        check(self._L.tgap_get_gap_soap(
            self.h, C.byref(hs), int(n_total_sites), n_sites0, ptr(nn), ptr(_i32(nb["neighbors_list"])),
            ptr(_f64(nb["rjs"])), ptr(_f64(nb["xyz"])), ptr(_i32(species_supercell)), int(central_species),
            Qs.shape[0], ptr(_f64(alphas)), ptr(Qs), float(delta), float(zeta), int(do_forces), int(precision),
            ptr(en), ptr(fo), ptr(vir), ptr(soap)), self.h, "tgap_get_gap_soap")
        del keep
        out = (en, fo, vir.reshape(3, 3, order="F"))
        return out + (soap,) if want_soap else out


def assign_species(species_types, names):
    """assign_species_multiplicity: character*8 names -> channel ids (1-based, 0 = absent)."""
    st = b"".join(s.encode().ljust(8)[:8] for s in species_types)
    nm = b"".join(s.encode().ljust(8)[:8] for s in names)
    out = np.zeros(len(names), np.int32)
    check(N.lib().tgap_assign_species(len(species_types), st, len(names), nm, ptr(out)))
    return out


class Model:
    """One soap_turbo GAP model resident on the device (tgap_model)."""

    def __init__(self, ctx, hypers, Qs, alphas, delta=1.0, zeta=4.0, central_species=0, compress=None):
        """compress: SOAP compression (P_i, P_j, P_el, dim_out), 1-based entries of P
        (tgap_model_create_compressed); Qs then has dim_out columns."""
        self.ctx = ctx
        self.hypers = dict(hypers)
        hs, keep = N.make_hypers(hypers)
        Qs = _f64(Qs)
        h = C.c_void_p()
        if compress is None:
            check(ctx._L.tgap_model_create(ctx.h, C.byref(hs), int(central_species), Qs.shape[0],
                                           ptr(_f64(alphas)), ptr(Qs), float(delta), float(zeta), C.byref(h)),
                  ctx.h, "tgap_model_create")
        else:
            pi = np.ascontiguousarray(compress[0], np.int32)
            pj = np.ascontiguousarray(compress[1], np.int32)
            pel = _f64(compress[2])
            check(ctx._L.tgap_model_create_compressed(ctx.h, C.byref(hs), int(central_species), Qs.shape[0],
                                                      ptr(_f64(alphas)), ptr(Qs), float(delta), float(zeta),
                                                      int(compress[3]), len(pi), ptr(pi), ptr(pj), ptr(pel),
                                                      C.byref(h)), ctx.h, "tgap_model_create_compressed")
        del keep
        self.h = h
        self.dim = int(ctx._L.tgap_model_dim(h))
        self.n_sparse = Qs.shape[0]
        self.central_species = central_species

    def close(self):
        if getattr(self, "h", None):
            # a handle whose context was closed first cannot be destroyed (its destroy would use
            # the freed context); its device memory goes with the process
            if getattr(self.ctx, "h", None):
                self.ctx._L.tgap_model_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class System:
    """A batch of periodic structures resident on the device (tgap_system).

    structures: list of (positions (n, 3), box rows (3, 3), species ids (n,))."""

    def __init__(self, ctx, structures, rcut_max):
        self.ctx = ctx
        pos = np.concatenate([_f64(s[0]).reshape(-1, 3) for s in structures])
        boxes = np.concatenate([_f64(s[1]).reshape(9) for s in structures])
        sp = np.concatenate([_i32(s[2]) for s in structures])
        offs = np.zeros(len(structures) + 1, np.int32)
        offs[1:] = np.cumsum([len(s[2]) for s in structures])
        self.offsets = offs
        self.n_atoms = int(offs[-1])
        self.n_structures = len(structures)
        h = C.c_void_p()
        check(ctx._L.tgap_system_create(ctx.h, len(structures), ptr(offs), ptr(pos), ptr(boxes), ptr(sp),
                                        float(rcut_max), C.byref(h)), ctx.h, "tgap_system_create")
        self.h = h

    @property
    def n_pairs(self):
        return int(self.ctx._L.tgap_system_n_pairs(self.h))

    def device_positions(self):
        p = C.c_void_p()
        check(self.ctx._L.tgap_system_positions(self.h, C.byref(p)))
        return p.value

    def set_positions(self, positions):
        check(self.ctx._L.tgap_system_set_positions(self.h, ptr(_f64(positions))), self.ctx.h, "set_positions")

    def update(self, rebuild=True):
        check(self.ctx._L.tgap_system_update(self.h, int(rebuild)), self.ctx.h, "tgap_system_update")

    def set_e0(self, e0):
        """Isolated-atom energy per species channel (e0[c - 1] for channel c), added to every
        energy output of the system (calculate_e0, calculate_gap_soap.f90:135-169)."""
        e = _f64(e0).reshape(-1)
        check(self.ctx._L.tgap_system_set_e0(self.h, len(e), ptr(e)), self.ctx.h, "tgap_system_set_e0")

    def get_positions(self):
        """Host copy of the resident positions (n_atoms, 3)."""
        x = np.zeros((self.n_atoms, 3))
        check(self.ctx._L.tgap_system_get_positions(self.h, ptr(x)), self.ctx.h, "tgap_system_get_positions")
        return x

    def set_site_range(self, beg, end=None):
        """Only atoms [beg, end) are descriptor centres of later evaluations (one rank's share of
        an atom decomposition, split_tasks misc.f90:88-111); None restores all sites."""
        check(self.ctx._L.tgap_system_set_site_range(self.h, int(beg), -1 if end is None else int(end)),
              self.ctx.h, "tgap_system_set_site_range")

    def calculate_gap_soap(self, models, precision, positions=None, rebuild=True):
        """Host-buffer evaluation (tgap_calculate_gap_soap): positions (n, 3) in (None keeps the
        resident ones), energies (n,), forces (n, 3) and per-structure virials (n_structures, 3, 3)
        out."""
        arr = (C.c_void_p * len(models))(*[m.h.value for m in models])
        e = np.zeros(self.n_atoms)
        f = np.zeros((self.n_atoms, 3))
        v = np.zeros((self.n_structures, 9))
        x = None if positions is None else _f64(positions).reshape(self.n_atoms, 3)
        check(self.ctx._L.tgap_calculate_gap_soap(self.ctx.h, self.h, len(models), arr, int(precision),
                                                  ptr(x) if x is not None else None, int(rebuild), ptr(e), ptr(f),
                                                  ptr(v)), self.ctx.h, "tgap_calculate_gap_soap")
        return e, f, v.reshape(self.n_structures, 3, 3)

    def compute_device(self, models, precision, d_energies, d_forces, d_virial, do_forces=True):
        """Device-pointer form: outputs are raw device addresses (ints)."""
        arr = (C.c_void_p * len(models))(*[m.h.value for m in models])
        check(self.ctx._L.tgap_compute(self.ctx.h, self.h, len(models), arr, int(precision), int(do_forces),
                                       C.c_void_p(d_energies), C.c_void_p(d_forces) if d_forces else None,
                                       C.c_void_p(d_virial) if d_virial else None), self.ctx.h, "tgap_compute")

    def local_property(self, model, V0, precision, do_derivatives=True):
        """Per-site property of a property model (tgap_local_property): V (n_atoms) and, with
        do_derivatives, dV_i/dr_j per list pair (n_pairs, 3), as host arrays."""
        import torch
        n, P = self.n_atoms, self.n_pairs
        V = torch.zeros(n, dtype=torch.float64, device="cuda")
        Vd = torch.zeros(3 * max(P, 1), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        check(self.ctx._L.tgap_local_property(self.ctx.h, self.h, model.h, float(V0), int(precision),
                                              int(do_derivatives), C.c_void_p(V.data_ptr()),
                                              C.c_void_p(Vd.data_ptr()) if do_derivatives else None),
              self.ctx.h, "tgap_local_property")
        self.ctx.synchronize()
        return V.cpu().numpy(), (Vd.cpu().numpy()[:3 * P].reshape(P, 3) if do_derivatives else None)

    def autotune(self, models, precision, reps=5):
        """Times the tunable launch shapes of this system's evaluation and keeps the fastest in the
        context (tgap_autotune); returns the report lines."""
        arr = (C.c_void_p * len(models))(*[m.h.value for m in models])
        check(self.ctx._L.tgap_autotune(self.ctx.h, self.h, len(models), arr, int(precision), int(reps)),
              self.ctx.h, "tgap_autotune")
        need = C.c_int64(0)
        check(self.ctx._L.tgap_autotune_report(self.ctx.h, None, 0, C.byref(need)), self.ctx.h, "autotune report")
        buf = C.create_string_buffer(max(1, need.value))
        check(self.ctx._L.tgap_autotune_report(self.ctx.h, buf, need.value, C.byref(need)), self.ctx.h,
              "autotune report")
        return [line for line in buf.value.decode().splitlines() if line]

    def close(self):
        if getattr(self, "h", None):
            # a handle whose context was closed first cannot be destroyed (its destroy would use
            # the freed context); its device memory goes with the process
            if getattr(self.ctx, "h", None):
                self.ctx._L.tgap_system_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Terms:
    """Pair and triplet GAP terms resident on the device (tgap_terms): distance_2b, core_pot and
    angle_3b, added after the SOAP models. Species are channel indices (1-based)."""

    def __init__(self, ctx):
        self.ctx = ctx
        h = C.c_void_p()
        check(ctx._L.tgap_terms_create(ctx.h, C.byref(h)), ctx.h, "tgap_terms_create")
        self.h = h
        self._keep = []

    def add_2b(self, species1, species2, alphas, cutoff, Qs, rcut, buffer=0.5, delta=1.0, sigma=1.0, e0=0.0):
        a = [_f64(alphas), _f64(cutoff), _f64(Qs)]
        check(self.ctx._L.tgap_terms_add_2b(self.h, int(species1), int(species2), len(a[0]), *[ptr(x) for x in a],
                                            float(rcut), float(buffer), float(delta), float(sigma), float(e0)),
              self.ctx.h, "tgap_terms_add_2b")

    def add_core_pot(self, species1, species2, x, V, yp1, ypn, dVdx2):
        a = [_f64(x), _f64(V)]
        check(self.ctx._L.tgap_terms_add_core_pot(self.h, int(species1), int(species2), len(a[0]), ptr(a[0]),
                                                  ptr(a[1]), float(yp1), float(ypn), ptr(_f64(dVdx2))),
              self.ctx.h, "tgap_terms_add_core_pot")

    def add_3b(self, species_center, species1, species2, alphas, cutoff, Qs, rcut, sigma, buffer=0.5, delta=1.0,
               e0=0.0, kernel="exp"):
        Qf = np.asfortranarray(Qs, dtype=np.float64).ravel(order="F")
        a = [_f64(alphas), _f64(cutoff)]
        check(self.ctx._L.tgap_terms_add_3b(self.h, int(species_center), int(species1), int(species2), len(a[0]),
                                            ptr(a[0]), ptr(a[1]), ptr(Qf), float(rcut), float(buffer), float(delta),
                                            ptr(_f64(sigma)), float(e0), 1 if kernel == "pol" else 0),
              self.ctx.h, "tgap_terms_add_3b")

    def compute_device(self, system, d_energies, d_forces, d_virial, do_forces=True):
        """Adds the terms' energies, forces and virial into device arrays."""
        check(self.ctx._L.tgap_terms_compute(self.ctx.h, system.h, self.h, int(do_forces), C.c_void_p(d_energies),
                                             C.c_void_p(d_forces) if d_forces else None,
                                             C.c_void_p(d_virial) if d_virial else None),
              self.ctx.h, "tgap_terms_compute")

    def close(self):
        if getattr(self, "h", None):
            if getattr(self.ctx, "h", None):
                self.ctx._L.tgap_terms_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MD:
    """NVE velocity-Verlet driver on the device (tgap_md)."""

    def __init__(self, ctx, system, models, masses_amu, dt, rebuild_every=10, precision=TGAP_FP64,
                 use_graph=True):
        self.ctx = ctx
        self.system = system
        self.models = list(models)
        arr = (C.c_void_p * len(models))(*[m.h.value for m in models])
        h = C.c_void_p()
        check(ctx._L.tgap_md_create(ctx.h, system.h, len(models), arr, ptr(_f64(masses_amu)), float(dt),
                                    int(rebuild_every), int(precision), int(use_graph), C.byref(h)),
              ctx.h, "tgap_md_create")
        self.h = h

    def set_velocities(self, v):
        check(self.ctx._L.tgap_md_set_velocities(self.h, ptr(_f64(v))), self.ctx.h, "set_velocities")

    def run(self, n_steps):
        check(self.ctx._L.tgap_md_run(self.h, int(n_steps)), self.ctx.h, "tgap_md_run")

    def state(self):
        n = self.system.n_atoms
        pos = np.zeros((n, 3)); vel = np.zeros((n, 3)); f = np.zeros((n, 3))
        ep = C.c_double(); ek = C.c_double()
        check(self.ctx._L.tgap_md_get_state(self.h, ptr(pos), ptr(vel), ptr(f), C.byref(ep), C.byref(ek)),
              self.ctx.h, "md_get_state")
        return dict(positions=pos, velocities=vel, forces=f, e_pot=ep.value, e_kin=ek.value)

    def set_terms(self, terms):
        """Adds pair and triplet terms (Terms) to every force evaluation; None removes them."""
        check(self.ctx._L.tgap_md_set_terms(self.h, terms.h if terms is not None else None), self.ctx.h,
              "tgap_md_set_terms")
        self._terms = terms

    def close(self):
        if getattr(self, "h", None):
            # a handle whose context was closed first cannot be destroyed (its destroy would use
            # the freed context); its device memory goes with the process
            if getattr(self.ctx, "h", None):
                self.ctx._L.tgap_md_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MC:
    """Metropolis single-atom moves with local updates on the device (tgap_mc).

    The system must have been built with rcut_max = model cutoff + skin. Proposals come from the
    caller: atoms (0-based), displacements (n, 3) and uniform deviates in [0, 1)."""

    def __init__(self, ctx, system, models, temperature, precision=TGAP_FP64, use_graph=True):
        self.ctx = ctx
        self.system = system
        self.models = list(models)
        arr = (C.c_void_p * len(models))(*[m.h.value for m in models])
        h = C.c_void_p()
        check(ctx._L.tgap_mc_create(ctx.h, system.h, len(models), arr, float(temperature), int(precision),
                                    int(use_graph), C.byref(h)), ctx.h, "tgap_mc_create")
        self.h = h

    def set_screen(self, w):
        """Installs a learned screen (weights as returned by turbogap_b200.screen.fit); proposals then
        take two uniform deviates each (uniforms of shape (n, 2))."""
        f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)
        pca = f32(w["pca"])
        n_pca, dim = pca.shape
        hidden = len(w["b1"])
        keep = [f32(w[k]) for k in ("mean", "pca", "w1", "b1", "w2", "b2", "w3")]
        check(self.ctx._L.tgap_mc_set_screen(self.h, dim, n_pca, hidden, *[ptr(a) for a in keep], float(w["b3"])),
              self.ctx.h, "tgap_mc_set_screen")
        self.screened = True

    def screen_log(self, n):
        des = np.zeros(n)
        st = np.zeros(n, np.uint8)
        check(self.ctx._L.tgap_mc_screen_log(self.h, n, ptr(des), ptr(st)), self.ctx.h, "tgap_mc_screen_log")
        return des, st

    def screen_fallback(self, window=256, min_confirm=0.1, min_pass=0.002, max_pass=0.99):
        """Sets when the driver gives up on the screen and continues as plain GAP MC: over each
        window of screen-judged proposals, a pass rate below min_pass or above max_pass (the screen
        settles too few proposals to pay for itself) or an exact-stage confirmation rate below
        min_confirm switches it off."""
        check(self.ctx._L.tgap_mc_screen_fallback(self.h, int(window), float(min_confirm), float(min_pass),
                                                  float(max_pass)),
              self.ctx.h, "tgap_mc_screen_fallback")

    def set_batch(self, slots):
        """Proposals evaluated side by side by the speculative batch of plain GAP MC (1..16)."""
        check(self.ctx._L.tgap_mc_set_batch(self.h, int(slots)), self.ctx.h, "tgap_mc_set_batch")

    def batch_stats(self):
        b, n = C.c_int64(), C.c_int64()
        check(self.ctx._L.tgap_mc_batch_stats(self.h, C.byref(b), C.byref(n)), self.ctx.h, "tgap_mc_batch_stats")
        return dict(batches=b.value, settled=n.value)

    def screen_stats(self):
        active = C.c_int()
        v = [C.c_int64() for _ in range(4)]
        check(self.ctx._L.tgap_mc_screen_stats(self.h, C.byref(active), *[C.byref(x) for x in v]),
              self.ctx.h, "tgap_mc_screen_stats")
        return dict(active=bool(active.value), judged=v[0].value, passed=v[1].value, confirmed=v[2].value,
                    fallbacks=v[3].value)

    def run(self, atoms, displacements, uniforms, logs=True):
        atoms = np.ascontiguousarray(atoms, dtype=np.int32)
        disp = _f64(displacements)
        u = _f64(uniforms)
        n = len(atoms)
        per = 2 if getattr(self, "screened", False) else 1
        if disp.size != 3 * n or u.size != per * n:
            raise ValueError("proposal arrays disagree in length")
        acc = C.c_int64(0)
        de = np.zeros(n) if logs else None
        ok = np.zeros(n, np.uint8) if logs else None
        check(self.ctx._L.tgap_mc_run(self.h, n, ptr(atoms), ptr(disp), ptr(u), C.byref(acc),
                                      ptr(de) if logs else None, ptr(ok) if logs else None),
              self.ctx.h, "tgap_mc_run")
        return dict(accepted=acc.value, de=de, accept=ok.astype(bool) if logs else None)

    def state(self):
        n = self.system.n_atoms
        pos = np.zeros((n, 3)); e = np.zeros(n)
        et = C.c_double(); acc = C.c_int64(); reb = C.c_int64()
        check(self.ctx._L.tgap_mc_get_state(self.h, ptr(pos), ptr(e), C.byref(et), C.byref(acc), C.byref(reb)),
              self.ctx.h, "mc_get_state")
        return dict(positions=pos, energies=e, e_total=et.value, accepted=acc.value, rebuilds=reb.value)

    def close(self):
        if getattr(self, "h", None):
            # a handle whose context was closed first cannot be destroyed (its destroy would use
            # the freed context); its device memory goes with the process
            if getattr(self.ctx, "h", None):
                self.ctx._L.tgap_mc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

