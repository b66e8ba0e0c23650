"""ctypes bindings of libtgap.so (the C ABI declared in include/tgap.h).

The library is required: importing the GPU entry points without it raises immediately, there
is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libtgap.so")

TGAP_FP64 = 0
TGAP_MIXED = 1

STATUS = {
    0: "OK", 1: "ERR_ARGUMENT", 2: "ERR_CUDA", 3: "ERR_CAPACITY", 4: "ERR_HYPERS",
    5: "ERR_TIMEOUT", 6: "ERR_UNSUPPORTED", 7: "ERR_NOMEM", 8: "ERR_NUMERIC",
}


class TgapError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class SoapHypers(C.Structure):
    """tgap_soap_hypers (per-species arrays, read_gap.f90:156-432)."""
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
    ]


HYPER_KEYS = ("rcut_hard", "rcut_soft", "nf", "global_scaling", "atom_sigma_r", "atom_sigma_r_scaling",
              "atom_sigma_t", "atom_sigma_t_scaling", "amplitude_scaling", "central_weight")


def make_hypers(h):
    """Build a SoapHypers struct from a dict; returns (struct, keep-alive arrays)."""
    ns = len(h["alpha_max"])
    keep = {}
    s = SoapHypers()
    s.n_species = ns
    s.l_max = int(h["l_max"])
    s.radial_enhancement = int(h.get("radial_enhancement", 0))
    a = np.ascontiguousarray(h["alpha_max"], dtype=np.int32)
    keep["alpha_max"] = a
    s.alpha_max = a.ctypes.data_as(C.POINTER(C.c_int))
    for k in HYPER_KEYS:
        v = np.ascontiguousarray(np.broadcast_to(np.asarray(h[k], dtype=np.float64), (ns,)))
        keep[k] = v
        setattr(s, k, v.ctypes.data_as(C.POINTER(C.c_double)))
    return s, keep


_lib = None


def lib():
    """Load libtgap.so (fails loudly when the extension is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libtgap.so not built ({LIB_PATH}); run turbogap_2.0_b200/build.py")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, dbl = C.c_void_p, C.c_int, C.c_int64, C.c_double
    P = C.POINTER
    sig = {
        "tgap_create": (i32, [i32, P(vp)]),
        "tgap_destroy": (i32, [vp]),
        "tgap_set_stream": (i32, [vp, vp]),
        "tgap_synchronize": (i32, [vp]),
        "tgap_last_error": (C.c_char_p, [vp]),
        "tgap_version": (C.c_char_p, []),
        "tgap_kernel_launches": (i64, [vp]),
        "tgap_number_of_unit_cells": (i32, [vp, vp, vp, dbl, vp]),
        "tgap_build_neighbors": (i32, [vp, i32, i32, vp, vp, vp, vp, i32, dbl, vp, i32, vp, vp, vp, vp, vp, vp,
                                       vp, i64, P(i64)]),
        "tgap_get_soap": (i32, [vp, i32, vp, i32, vp, vp, i32, vp, vp, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp,
                                vp, vp, vp, i32, vp, C.c_char_p, C.c_char_p, i32, i32, i32, vp, vp, vp, vp, vp]),
        "tgap_get_soap_energy_and_forces": (i32, [vp, i32, i32, i32, vp, vp, vp, dbl, dbl, dbl, vp, vp, vp, vp,
                                                  i32, i32, i32, vp, vp, vp]),
        "tgap_get_gap_soap": (i32, [vp, P(SoapHypers), i32, i32, vp, vp, vp, vp, vp, i32, i32, vp, vp, dbl, dbl,
                                    i32, i32, vp, vp, vp, vp]),
        "tgap_assign_species": (i32, [i32, C.c_char_p, i32, C.c_char_p, vp]),
        "tgap_model_create": (i32, [vp, P(SoapHypers), i32, i32, vp, vp, dbl, dbl, P(vp)]),
        "tgap_model_create_compressed": (i32, [vp, P(SoapHypers), i32, i32, vp, vp, dbl, dbl, i32, i32, vp, vp, vp,
                                               P(vp)]),
        "tgap_model_destroy": (i32, [vp]),
        "tgap_model_dim": (i32, [vp]),
        "tgap_system_create": (i32, [vp, i32, vp, vp, vp, vp, dbl, P(vp)]),
        "tgap_system_destroy": (i32, [vp]),
        "tgap_system_n_atoms": (i32, [vp]),
        "tgap_system_n_pairs": (i64, [vp]),
        "tgap_system_positions": (i32, [vp, P(vp)]),
        "tgap_system_set_positions": (i32, [vp, vp]),
        "tgap_system_update": (i32, [vp, i32]),
        "tgap_system_set_e0": (i32, [vp, i32, vp]),
        "tgap_system_set_site_range": (i32, [vp, i32, i32]),
        "tgap_system_get_positions": (i32, [vp, vp]),
        "tgap_velocity_verlet": (i32, [vp, i32, vp, vp, vp, vp, vp, vp, dbl, dbl, i32]),
        "tgap_velocity_verlet_host": (i32, [i32, vp, vp, vp, vp, vp, vp, dbl, dbl, i32]),
        "tgap_host_register": (i32, [vp, vp, C.c_size_t]),
        "tgap_host_unregister": (i32, [vp, vp]),
        "tgap_compute": (i32, [vp, vp, i32, vp, i32, i32, vp, vp, vp]),
        "tgap_descriptors": (i32, [vp, vp, vp, i32, vp, P(i32)]),
        "tgap_md_create": (i32, [vp, vp, i32, vp, vp, dbl, i32, i32, i32, P(vp)]),
        "tgap_md_destroy": (i32, [vp]),
        "tgap_md_set_velocities": (i32, [vp, vp]),
        "tgap_md_run": (i32, [vp, i32]),
        "tgap_md_get_state": (i32, [vp, vp, vp, vp, P(dbl), P(dbl)]),
        "tgap_mc_create": (i32, [vp, vp, i32, vp, dbl, i32, i32, P(vp)]),
        "tgap_mc_destroy": (i32, [vp]),
        "tgap_mc_run": (i32, [vp, i64, vp, vp, vp, P(i64), vp, vp]),
        "tgap_mc_get_state": (i32, [vp, vp, vp, P(dbl), P(i64), P(i64)]),
        "tgap_mc_set_screen": (i32, [vp, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, C.c_float]),
        "tgap_mc_screen_log": (i32, [vp, i64, vp, vp]),
        "tgap_mc_screen_fallback": (i32, [vp, i64, C.c_double, C.c_double, C.c_double]),
        "tgap_mc_screen_stats": (i32, [vp, vp, vp, vp, vp, vp]),
        "tgap_mc_set_batch": (i32, [vp, i32]),
        "tgap_mc_batch_stats": (i32, [vp, vp, vp]),
        "tgap_screen_grad": (i32, [vp, i64, i32, i32, vp, vp, vp, vp, vp, vp, vp, C.c_float,
                                   vp, vp, vp, vp, vp, vp, vp]),
        "tgap_screen_train": (i32, [vp, i64, i32, i32, vp, vp, i32, i32, C.c_float, vp,
                                    vp, vp, vp, vp, vp, vp, vp]),
        "tgap_local_property_predict": (i32, [vp, i32, i32, i32, vp, vp, vp, C.c_double, C.c_double, C.c_double,
                                              i32, vp, vp, i32, vp, vp]),
        "tgap_local_property": (i32, [vp, vp, vp, C.c_double, i32, i32, vp, vp]),
        "tgap_get_2b_energy_and_forces": (i32, [vp, i32, i32, vp, vp, i32, vp, vp, C.c_double, C.c_double,
                                                C.c_double, C.c_double, C.c_double, vp, vp, i32, vp, vp, i32, i32,
                                                i32, vp, vp, vp]),
        "tgap_get_3b_energy_and_forces": (i32, [vp, i32, i32, i32, vp, vp, i32, vp, vp, C.c_double, C.c_double,
                                                C.c_double, vp, C.c_double, vp, vp, vp, i32, i32, vp, vp, i32, i32,
                                                i32, vp, vp, vp]),
        "tgap_get_core_pot_energy_and_forces": (i32, [vp, i32, i32, i32, i32, vp, vp, vp, vp, C.c_double,
                                                      C.c_double, vp, vp, i32, vp, vp, i32, i32, vp, vp, vp]),
        "tgap_terms_create": (i32, [vp, vp]),
        "tgap_terms_destroy": (i32, [vp]),
        "tgap_terms_add_2b": (i32, [vp, i32, i32, i32, vp, vp, vp, C.c_double, C.c_double, C.c_double, C.c_double,
                                    C.c_double]),
        "tgap_terms_add_core_pot": (i32, [vp, i32, i32, i32, vp, vp, C.c_double, C.c_double, vp]),
        "tgap_terms_add_3b": (i32, [vp, i32, i32, i32, i32, vp, vp, vp, C.c_double, C.c_double, C.c_double, vp,
                                    C.c_double, i32]),
        "tgap_terms_compute": (i32, [vp, vp, vp, i32, vp, vp, vp]),
        "tgap_md_set_terms": (i32, [vp, vp]),
        "tgap_autotune": (i32, [vp, vp, i32, vp, i32, i32]),
        "tgap_autotune_report": (i32, [vp, vp, i64, vp]),
        "tgap_autotune_clear": (i32, [vp]),
        "tgap_autotune_set": (i32, [vp, C.c_char_p, i32]),
        "tgap_screen_eval": (i32, [vp, i64, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, C.c_float, vp, vp]),
        "tgap_debug_poly3_w": (i32, [i32, vp]),
        "tgap_calculate_gap_soap": (i32, [vp, vp, i32, vp, i32, vp, i32, vp, vp, vp]),
        "tgap_timing_enable": (i32, [vp, i32]),
        "tgap_timing_reset": (i32, [vp]),
        "tgap_timing_report": (i32, [vp, i32, vp, vp, vp, P(i32)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def ptr(a):
    """Data pointer of a numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.c_void_p)


def check(status, ctx=None, what=""):
    if status != 0:
        msg = lib().tgap_last_error(ctx).decode() if ctx else ""
        raise TgapError(status, f"{what} {msg}".strip())
