"""ctypes bindings of the CPU oracle (oracle/_build/liboracle.so).

The oracle is test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline use it, always as the checker. Arrays follow the Fortran call surface of TurboGAP
(column-major, first index fastest; neighbor ids 1-based).
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "_build", "liboracle.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


class _Hypers(C.Structure):
    _fields_ = [
        ("n_species", C.c_int),
        ("alpha_max", C.POINTER(C.c_int)),
        ("l_max", C.c_int),
        ("rcut_hard", C.POINTER(C.c_double)),
        ("rcut_soft", C.POINTER(C.c_double)),
        ("nf", C.POINTER(C.c_double)),
        ("global_scaling", C.POINTER(C.c_double)),
        ("atom_sigma_r", C.POINTER(C.c_double)),
        ("atom_sigma_r_scaling", C.POINTER(C.c_double)),
        ("atom_sigma_t", C.POINTER(C.c_double)),
        ("atom_sigma_t_scaling", C.POINTER(C.c_double)),
        ("amplitude_scaling", C.POINTER(C.c_double)),
        ("central_weight", C.POINTER(C.c_double)),
        ("radial_enhancement", C.c_int),
        ("n_compress", C.c_int),
        ("dim_out", C.c_int),
        ("compress_P_i", C.POINTER(C.c_int)),
        ("compress_P_j", C.POINTER(C.c_int)),
        ("compress_P_el", C.POINTER(C.c_double)),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_get_distance.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, C.POINTER(C.c_double), _ip]
        L.orc_number_of_unit_cells.argtypes = [_dp, _dp, _dp, C.c_double, _ip]
        L.orc_set_supercell.argtypes = [C.c_int, _dp, _ip, _ip, _dp, _dp, _dp, _dp, _ip]
        L.orc_build_neighbors.restype = C.c_int64
        L.orc_build_neighbors.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.c_int, C.c_double,
                                          _ip, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_neighbor_geometry.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _ip, _ip, _ip, _dp, _dp,
                                            _dp, _dp, _ip]
        L.orc_soap_dim.argtypes = [C.POINTER(_Hypers)]
        L.orc_radial_nodes.argtypes = [C.POINTER(_Hypers), C.c_int, _dp, _dp, C.c_int]
        L.orc_poly3_w.argtypes = [C.c_int, _dp]
        L.orc_radial.argtypes = [C.POINTER(_Hypers), C.c_int, C.c_double, C.c_int, _dp, _dp]
        L.orc_angular.argtypes = [C.POINTER(_Hypers), C.c_int, C.c_double, _dp, _dp, _dp]
        L.orc_get_soap.argtypes = [C.POINTER(_Hypers), C.c_int, _ip, C.c_int, _up, _dp, _dp, _dp,
                                   _dp, C.c_void_p]
        L.orc_get_soap_energy_and_forces.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp,
                                                     C.c_double, C.c_double, C.c_double, _dp, _ip,
                                                     _ip, _dp, C.c_int, C.c_int, _dp, _dp, _dp]
        L.orc_get_gap_soap.argtypes = [C.POINTER(_Hypers), C.c_int, C.c_int, _ip, _ip, _dp, _dp,
                                       _dp, _dp, _ip, C.c_int, C.c_int, _dp, _dp, C.c_double,
                                       C.c_double, C.c_int, _dp, _dp, _dp]
        L.orc_calculate_e0.argtypes = [C.c_int, _ip, C.c_int, _dp, _dp]
        L.orc_local_property_predict.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.c_double,
                                                 C.c_double, C.c_double, C.c_int, _dp, _ip, _dp, _dp]
        L.orc_get_2b_energy_and_forces.argtypes = [C.c_int, _dp, _dp, C.c_int, _dp, _dp, C.c_double, C.c_double,
                                                   C.c_double, C.c_double, C.c_double, _dp, _ip, C.c_int, _ip,
                                                   _ip, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]
        L.orc_get_core_pot_energy_and_forces.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.c_double,
                                                         C.c_double, _dp, _ip, C.c_int, _ip, _ip, C.c_int, C.c_int,
                                                         _dp, _dp, _dp]
        L.orc_get_3b_energy_and_forces.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_int, _dp, _dp, C.c_double,
                                                   C.c_double, C.c_double, _dp, C.c_double, _dp, _ip, _ip, C.c_int,
                                                   C.c_int, _ip, _ip, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]
        L.orc_velocity_verlet.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double,
                                          C.POINTER(C.c_double), C.c_int]
        L.orc_mc_move_acceptance.restype = C.c_double
        L.orc_mc_move_acceptance.argtypes = [C.c_double, C.c_double, C.c_double]
        L.orc_num_threads.restype = C.c_int
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class Hypers:
    """SOAP hypers of one model (per-species arrays), kept alive for the ctypes struct."""

    def __init__(self, sp):
        ns = len(sp["alpha_max"])
        self.arrays = {}
        self.s = _Hypers()
        self.s.n_species = ns
        self.s.l_max = int(sp["l_max"])
        self.s.radial_enhancement = int(sp.get("radial_enhancement", 0))
        a = np.ascontiguousarray(sp["alpha_max"], dtype=np.int32)
        self.arrays["alpha_max"] = a
        self.s.alpha_max = a.ctypes.data_as(C.POINTER(C.c_int))
        for k in ("rcut_hard", "rcut_soft", "nf", "global_scaling", "atom_sigma_r",
                  "atom_sigma_r_scaling", "atom_sigma_t", "atom_sigma_t_scaling",
                  "amplitude_scaling", "central_weight"):
            v = np.ascontiguousarray(np.broadcast_to(np.asarray(sp[k], dtype=np.float64), (ns,)))
            self.arrays[k] = v
            setattr(self.s, k, v.ctypes.data_as(C.POINTER(C.c_double)))
        # SOAP compression: sp["compress"] = (P_i, P_j, P_el, dim_out), 1-based indices
        if sp.get("compress") is not None:
            pi, pj, pel, dim_out = sp["compress"]
            for k, v, t in (("compress_P_i", pi, np.int32), ("compress_P_j", pj, np.int32),
                            ("compress_P_el", pel, np.float64)):
                a = np.ascontiguousarray(v, dtype=t)
                self.arrays[k] = a
                setattr(self.s, k, a.ctypes.data_as(C.POINTER(C.c_int if t is np.int32 else C.c_double)))
            self.s.n_compress = len(self.arrays["compress_P_i"])
            self.s.dim_out = int(dim_out)

    @property
    def ref(self):
        return C.byref(self.s)

    def dim(self):
        return lib().orc_soap_dim(self.ref)


def get_distance(posi, posj, a, b, c):
    dist = np.zeros(3)
    d = C.c_double()
    sh = np.zeros(3, np.int32)
    lib().orc_get_distance(np.asarray(posi, float), np.asarray(posj, float), np.asarray(a, float),
                           np.asarray(b, float), np.asarray(c, float), dist, C.byref(d), sh)
    return dist, d.value, sh


def number_of_unit_cells(a, b, c, rcut):
    idx = np.zeros(3, np.int32)
    lib().orc_number_of_unit_cells(np.asarray(a, float), np.asarray(b, float),
                                   np.asarray(c, float), rcut, idx)
    return idx


def set_supercell(pos, species, indices, a, b, c):
    n = pos.shape[0]
    nsc = n * int(np.prod(indices))
    a = np.array(a, float); b = np.array(b, float); c = np.array(c, float)
    pos_sc = np.zeros((nsc, 3))
    sp_sc = np.zeros(nsc, np.int32)
    lib().orc_set_supercell(n, np.ascontiguousarray(pos, float), np.ascontiguousarray(species, np.int32),
                            np.asarray(indices, np.int32), a, b, c, pos_sc, sp_sc)
    return pos_sc, sp_sc, a, b, c


def build_neighbors(pos_sc, n_sites, a, b, c, rcut_max, species_sc, box_small):
    """Returns dict(n_neigh, neighbors_list (1-based), rjs, xyz (P,3), thetas, phis, species)."""
    L = lib()
    pos_sc = np.ascontiguousarray(pos_sc, float)
    a = np.array(a, float); b = np.array(b, float); c = np.array(c, float)
    sp = np.ascontiguousarray(species_sc, np.int32)
    nsc = pos_sc.shape[0]
    P = L.orc_build_neighbors(n_sites, nsc, pos_sc, a, b, c, int(box_small), rcut_max, sp,
                              None, None, None, None, None, None, None)
    if P < 0:
        raise RuntimeError("unsupported lattice")
    nn = np.zeros(n_sites, np.int32)
    nl = np.zeros(P, np.int32)
    rjs = np.zeros(P); xyz = np.zeros((P, 3)); th = np.zeros(P); ph = np.zeros(P)
    nsp = np.zeros(P, np.int32)
    P2 = L.orc_build_neighbors(n_sites, nsc, pos_sc, a, b, c, int(box_small), rcut_max, sp,
                               _ptr(nn), _ptr(nl), _ptr(rjs), _ptr(xyz), _ptr(th), _ptr(ph), _ptr(nsp))
    assert P2 == P
    return dict(n_neigh=nn, neighbors_list=nl, rjs=rjs, xyz=xyz, thetas=th, phis=ph,
                neighbor_species=nsp, a=a, b=b, c=c)


def neighbor_geometry(pos_sc, n_sites, a, b, c, n_neigh, nl, species_sc):
    P = nl.shape[0]
    rjs = np.zeros(P); xyz = np.zeros((P, 3)); th = np.zeros(P); ph = np.zeros(P)
    nsp = np.zeros(P, np.int32)
    lib().orc_neighbor_geometry(n_sites, np.ascontiguousarray(pos_sc, float), np.asarray(a, float),
                                np.asarray(b, float), np.asarray(c, float),
                                np.ascontiguousarray(n_neigh, np.int32),
                                np.ascontiguousarray(nl, np.int32),
                                np.ascontiguousarray(species_sc, np.int32), rjs, xyz, th, ph, nsp)
    return dict(rjs=rjs, xyz=xyz, thetas=th, phis=ph, neighbor_species=nsp)


def get_soap(h, n_neigh, mask, rjs, thetas, phis, derivatives=True):
    """mask: (P, n_species) bool. Returns soap (n_sites, D) and soap_cart_der (P, D, 3)."""
    n_sites = len(n_neigh)
    P = len(rjs)
    D = h.dim()
    soap = np.zeros((n_sites, D))
    der = np.zeros((P, D, 3)) if derivatives else None
    m = np.ascontiguousarray(np.asarray(mask, np.uint8).T)  # column-major P x ns
    rc = lib().orc_get_soap(h.ref, n_sites, np.ascontiguousarray(n_neigh, np.int32), P, m,
                            np.ascontiguousarray(rjs, float), np.ascontiguousarray(thetas, float),
                            np.ascontiguousarray(phis, float), soap,
                            _ptr(der) if derivatives else None)
    if rc != 0:
        raise RuntimeError("orc_get_soap failed")
    return soap, der


def radial(h, s, r, central=False):
    am = int(h.arrays["alpha_max"][s])
    R = np.zeros(am); dR = np.zeros(am)
    lib().orc_radial(h.ref, s, r, int(central), R, dR)
    return R, dR


def angular(h, s, r, u):
    L = int(h.s.l_max)
    A = np.zeros((L + 1) ** 2); dA = np.zeros(3 * (L + 1) ** 2)
    lib().orc_angular(h.ref, s, r, np.asarray(u, float), A, dA)
    return A, dA.reshape(-1, 3)


def radial_nodes(h, s, cap=256):
    am = int(h.arrays["alpha_max"][s])
    xq = np.zeros(cap); tq = np.zeros(cap * am)
    n = lib().orc_radial_nodes(h.ref, s, xq, tq, cap)
    return xq[:n], tq[: n * am].reshape(n, am)


def poly3_w(am):
    W = np.zeros(am * am)
    lib().orc_poly3_w(am, W)
    return W.reshape(am, am)


def soap_energy_and_forces(soap, soap_der, alphas, delta, zeta, e0, Qs, n_neigh, nl, xyz,
                           do_forces=True, n_sites0=None):
    n_sites, D = soap.shape
    M = len(alphas)
    if n_sites0 is None:
        n_sites0 = n_sites
    en = np.zeros(n_sites)
    fo = np.zeros((n_sites0, 3))
    vir = np.zeros(9)
    lib().orc_get_soap_energy_and_forces(
        D, n_sites, M, np.ascontiguousarray(soap), np.ascontiguousarray(soap_der),
        np.ascontiguousarray(alphas, float), delta, zeta, e0, np.ascontiguousarray(Qs, float),
        np.ascontiguousarray(n_neigh, np.int32), np.ascontiguousarray(nl, np.int32),
        np.ascontiguousarray(xyz, float), int(do_forces), n_sites0, en, fo, vir)
    return en, fo, vir.reshape(3, 3, order="F")


def local_property_predict(soap, Qs, alphas, V0, delta, zeta, soap_cart_der=None, n_neigh=None):
    """local_property_predict: soap (n_sites, D), Qs (M, D), soap_cart_der (P, D, 3) or None."""
    soap = np.ascontiguousarray(soap, float)
    n_sites, D = soap.shape
    do_der = soap_cart_der is not None
    P = int(np.sum(n_neigh)) if do_der else 0
    V = np.zeros(n_sites)
    V_der = np.zeros((max(P, 1), 3))
    der = np.ascontiguousarray(soap_cart_der, float) if do_der else np.zeros(3)
    nn = np.ascontiguousarray(n_neigh if do_der else np.zeros(max(n_sites, 1)), np.int32)
    lib().orc_local_property_predict(D, n_sites, len(alphas), soap, np.ascontiguousarray(Qs, float),
                                     np.ascontiguousarray(alphas, float), V0, delta, zeta, int(do_der), der, nn,
                                     V, V_der)
    return V, (V_der[:P] if do_der else None)


def get_2b_energy_and_forces(nb, species, sp1, sp2, alphas, cutoff, rcut, buffer, delta, sigma, e0, Qs,
                             n_sites0=None, do_forces=True):
    """get_2b_energy_and_forces on a neighbor-list dict; species per site (channel indices)."""
    n = len(nb["n_neigh"])
    n0 = n if n_sites0 is None else n_sites0
    en, fo, vir = np.zeros(n), np.zeros((n0, 3)), np.zeros(9)
    lib().orc_get_2b_energy_and_forces(
        n, np.ascontiguousarray(nb["rjs"], float), np.ascontiguousarray(nb["xyz"], float), len(alphas),
        np.ascontiguousarray(alphas, float), np.ascontiguousarray(cutoff, float), rcut, buffer, delta, sigma, e0,
        np.ascontiguousarray(Qs, float), np.ascontiguousarray(nb["n_neigh"], np.int32), int(do_forces),
        np.ascontiguousarray(species, np.int32), np.ascontiguousarray(nb["neighbor_species"], np.int32), sp1, sp2,
        n0, en, fo, vir)
    return en, fo, vir.reshape(3, 3, order="F")


def get_core_pot_energy_and_forces(nb, species, sp1, sp2, x, V, yp1, ypn, dVdx2, n_sites0=None, do_forces=True):
    n = len(nb["n_neigh"])
    n0 = n if n_sites0 is None else n_sites0
    en, fo, vir = np.zeros(n), np.zeros((n0, 3)), np.zeros(9)
    lib().orc_get_core_pot_energy_and_forces(
        len(x), n, n0, np.ascontiguousarray(nb["rjs"], float), np.ascontiguousarray(nb["xyz"], float),
        np.ascontiguousarray(x, float), np.ascontiguousarray(V, float), yp1, ypn, np.ascontiguousarray(dVdx2, float),
        np.ascontiguousarray(nb["n_neigh"], np.int32), int(do_forces), np.ascontiguousarray(species, np.int32),
        np.ascontiguousarray(nb["neighbor_species"], np.int32), sp1, sp2, en, fo, vir)
    return en, fo, vir.reshape(3, 3, order="F")


def get_3b_energy_and_forces(nb, species, sp0, sp1, sp2, alphas, cutoff, rcut, buffer, delta, sigma, e0, Qs,
                             kernel="exp", n_sites0=None, do_forces=True):
    """get_3b_energy_and_forces on a neighbor-list dict; Qs (n_sparse, 3), sigma (3,)."""
    n = len(nb["n_neigh"])
    n0 = n if n_sites0 is None else n_sites0
    en, fo, vir = np.zeros(n), np.zeros((n0, 3)), np.zeros(9)
    lib().orc_get_3b_energy_and_forces(
        n0, n, np.ascontiguousarray(nb["rjs"], float), np.ascontiguousarray(nb["xyz"], float), len(alphas),
        np.ascontiguousarray(alphas, float), np.ascontiguousarray(cutoff, float), rcut, buffer, delta,
        np.ascontiguousarray(sigma, float), e0, np.asfortranarray(Qs, float).ravel(order="F"),
        np.ascontiguousarray(nb["n_neigh"], np.int32), np.ascontiguousarray(nb["neighbors_list"], np.int32),
        int(do_forces), 1 if kernel == "pol" else 0, np.ascontiguousarray(species, np.int32),
        np.ascontiguousarray(nb["neighbor_species"], np.int32), sp0, sp1, sp2, en, fo, vir)
    return en, fo, vir.reshape(3, 3, order="F")


def spline_second_derivatives(x, y, yp1, ypn):
    """Second derivatives of the interpolating cubic spline (the tridiagonal solve of the standard
    cubic spline, clamped end slopes yp1/ypn, natural ends when a slope is > 0.99e30), as TurboGAP's
    model reader prepares dVdx2 for get_core_pot_energy_and_forces."""
    x = np.asarray(x, float)
    y = np.asarray(y, float)
    n = len(x)
    y2, u = np.zeros(n), np.zeros(n)
    if yp1 > 0.99e30:
        y2[0], u[0] = 0.0, 0.0
    else:
        y2[0] = -0.5
        u[0] = (3.0 / (x[1] - x[0])) * ((y[1] - y[0]) / (x[1] - x[0]) - yp1)
    for i in range(1, n - 1):
        sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1])
        p = sig * y2[i - 1] + 2.0
        y2[i] = (sig - 1.0) / p
        u[i] = (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1])
        u[i] = (6.0 * u[i] / (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / p
    if ypn > 0.99e30:
        qn, un = 0.0, 0.0
    else:
        qn = 0.5
        un = (3.0 / (x[-1] - x[-2])) * (ypn - (y[-1] - y[-2]) / (x[-1] - x[-2]))
    y2[-1] = (un - qn * u[-2]) / (qn * y2[-2] + 1.0)
    for k in range(n - 2, -1, -1):
        y2[k] = y2[k] * y2[k + 1] + u[k]
    return y2


def get_gap_soap(h, n_total_sites, nb, species_sc, central_species, alphas, Qs, delta, zeta,
                 do_forces=True):
    n_sites0 = len(nb["n_neigh"])
    en = np.zeros(n_total_sites)
    fo = np.zeros((n_total_sites, 3))
    vir = np.zeros(9)
    rc = lib().orc_get_gap_soap(
        h.ref, n_total_sites, n_sites0, np.ascontiguousarray(nb["n_neigh"], np.int32),
        np.ascontiguousarray(nb["neighbors_list"], np.int32), np.ascontiguousarray(nb["rjs"]),
        np.ascontiguousarray(nb["thetas"]), np.ascontiguousarray(nb["phis"]),
        np.ascontiguousarray(nb["xyz"]), np.ascontiguousarray(species_sc, np.int32),
        int(central_species), len(alphas), np.ascontiguousarray(alphas, float),
        np.ascontiguousarray(Qs, float), delta, zeta, int(do_forces), en, fo, vir)
    if rc != 0:
        raise RuntimeError("orc_get_gap_soap failed")
    return en, fo, vir.reshape(3, 3, order="F")


def velocity_verlet(pos, pos_prev, vel, forces, forces_prev, masses, dt, dt_prev, first_step):
    dtp = C.c_double(dt_prev)
    lib().orc_velocity_verlet(len(masses), pos, pos_prev, vel, np.ascontiguousarray(forces),
                              forces_prev, np.ascontiguousarray(masses, float), dt, C.byref(dtp),
                              int(first_step))
    return dtp.value


def mc_move_acceptance(e_new, e_prev, temp):
    return lib().orc_mc_move_acceptance(e_new, e_prev, temp)


def calculate_e0(species, e0):
    """Per-site e0 by species channel (calculate_gap_soap.f90:135-169), zero for other sites."""
    sp = np.ascontiguousarray(species, np.int32)
    e = np.ascontiguousarray(e0, float)
    out = np.zeros(len(sp))
    lib().orc_calculate_e0(len(sp), sp, len(e), e, out)
    return out


def num_threads():
    return lib().orc_num_threads()
