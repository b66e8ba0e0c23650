"""Reader of TurboGAP model files: the `.gap` hypers file, the sparse-set `alphas`/`desc` files it
names and the core_pot tables (read_gap_hypers / read_alphas_and_descriptors,
src/gap/read_gap.f90:45-875), so real TurboGAP models can drive the device path.

Format (read_gap.f90:89-771). Records are read the way Fortran list-directed input reads them:
tokens separated by blanks or commas, quotes around strings optional, a line starting with '#' or
'!' ignored. Each model is a block `gap_beg <type>` ... `gap_end` of `keyword = value(s)` records,
<type> one of soap_turbo, distance_2b, angle_3b, core_pot. Defaults, derived settings and file
layouts follow the reference:
  * soap_turbo: per-species arrays sized by n_species; nf 4, buffer 0.5, sigma scalings 0,
    amplitude_scaling 1, central_weight 1, global_scaling 1, zeta 2, delta 1, l_max 8,
    central_species 0; `buffer` is the soft-cutoff width, so rcut_soft = rcut - buffer (rcut when
    the buffer is 0) (:424-432). alphas file: one value per sparse point; desc file: n_sparse x dim
    values, one per record, descriptor index fastest (:810-827). With compress_soap the
    descriptor is P p / |P p|: file_compress_soap holds P (a P_transformation block or the older
    index list, :489-529) and dim is its length; a compress_mode recipe without a file is soap_turbo
    code that the reference sources do not hold, so such a model is refused when loaded.
  * distance_2b / angle_3b: delta 1, sigma 1, buffer 0.5 (not read from the file), kernel_type
    "exp"; alphas file: `alpha cutoff` per sparse point; desc file: 1 (2b) or 3 (3b) values per
    sparse point, one per record (:828-872).
  * core_pot: table file `n yp1 ypn`, then n records `x V`; entries beyond core_pot_cutoff are
    dropped and those within core_pot_buffer of it tapered by (cos + 1)/2 (:672-690); spline second
    derivatives of the clamped (or, for an end slope > 0.99e30, natural) cubic spline, and a natural
    end's slope replaced by the spline's derivative there (:701-760).
Relative file names resolve against `base_dir` (the reference opens them relative to the working
directory, which is the default here too).
"""
import os
import re

import numpy as np

_SPLIT = re.compile(r"[\s,]+")


def _tokens(line):
    t = [x.strip("'\"") for x in _SPLIT.split(line.strip()) if x]
    return t


def _values(tok):
    """Values of a `keyword = v1 v2 ...` record."""
    return tok[2:] if len(tok) > 1 and tok[1] == "=" else tok[1:]


def _bool(s):
    return s.strip(".").lower() in ("t", "true", "1", "y", "yes")


def _lines(path):
    with open(path) as f:
        return [ln.rstrip("\n") for ln in f]


def _records(path):
    """Non-empty records of a one-value-per-record file (list-directed: one value per line)."""
    out = []
    for ln in _lines(path):
        tok = _tokens(ln)
        if tok:
            out.append(tok)
    return out


def read_compress_file(path, n_species):
    """SOAP compression file (read_gap.f90:489-529): a first record of n_species + 2 integers, the
    last the compressed length; then either a `P_transformation` block of `P_i P_j P_el` records up
    to `end_transformation`, or (the older format) one record per compressed component holding the
    1-based index of the power-spectrum component it keeps (P_i = i, P_el = 1). Returns
    (P_i, P_j, P_el, dim_out)."""
    lines = [ln for ln in _lines(path)]
    head = _tokens(lines[0])
    if len(head) < n_species + 2:
        raise ValueError(f"{path}: the first record needs {n_species + 2} integers")
    dim_out = int(float(head[n_species + 1]))
    rest = [_tokens(ln) for ln in lines[1:]]
    rest = [t for t in rest if t]
    if rest and rest[0][0] == "P_transformation":
        pi, pj, pel = [], [], []
        for t in rest[1:]:
            if t[0] == "end_transformation":
                break
            pi.append(int(float(t[0])))
            pj.append(int(float(t[1])))
            pel.append(float(t[2]))
        return np.array(pi, np.int32), np.array(pj, np.int32), np.array(pel), dim_out
    pj = np.array([int(float(t[0])) for t in rest[:dim_out]], np.int32)
    return np.arange(1, dim_out + 1, dtype=np.int32), pj, np.ones(dim_out), dim_out


def read_alphas_and_descriptors(file_desc, file_alphas, descriptor_type):
    """read_alphas_and_descriptors (read_gap.f90:773-875). soap_turbo: alphas (M,), Qs (M, dim);
    distance_2b: alphas, cutoff, Qs (M,); angle_3b: alphas, cutoff, Qs (M, 3)."""
    ra = _records(file_alphas)
    rd = _records(file_desc)
    M = len(ra)
    if M == 0 or len(rd) % M:
        raise ValueError(f"{file_desc}: {len(rd)} records is not a multiple of the {M} sparse points")
    dim = len(rd) // M
    d = np.array([float(r[0]) for r in rd])
    if descriptor_type == "soap_turbo":
        return dict(alphas=np.array([float(r[0]) for r in ra]), Qs=d.reshape(M, dim))
    want = {"distance_2b": 1, "angle_3b": 3}[descriptor_type]
    if dim != want:
        raise ValueError(f"bad {descriptor_type} files: {dim} values per sparse point, expected {want}")
    out = dict(alphas=np.array([float(r[0]) for r in ra]), cutoff=np.array([float(r[1]) for r in ra]))
    out["Qs"] = d if want == 1 else d.reshape(M, 3)
    return out


def spline_second_derivatives(x, y, yp1, ypn):
    """Second derivatives of the interpolating cubic spline through (x, y): the tridiagonal system
    of the standard cubic spline with end slopes yp1 / ypn, or a natural end for a slope > 0.99e30."""
    x = np.asarray(x, float)
    y = np.asarray(y, float)
    n = len(x)
    y2, u = np.zeros(n), np.zeros(n)
    if yp1 <= 0.99e30:
        y2[0] = -0.5
        u[0] = (3.0 / (x[1] - x[0])) * ((y[1] - y[0]) / (x[1] - x[0]) - yp1)
    for i in range(1, n - 1):
        sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1])
        p = sig * y2[i - 1] + 2.0
        y2[i] = (sig - 1.0) / p
        u[i] = (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1])
        u[i] = (6.0 * u[i] / (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / p
    qn = un = 0.0
    if ypn <= 0.99e30:
        qn = 0.5
        un = (3.0 / (x[-1] - x[-2])) * (ypn - (y[-1] - y[-2]) / (x[-1] - x[-2]))
    y2[-1] = (un - qn * u[-2]) / (qn * y2[-2] + 1.0)
    for k in range(n - 2, -1, -1):
        y2[k] = y2[k] * y2[k + 1] + u[k]
    return y2


def _spline_der_at(x, y, y2, r):
    """Derivative of the spline of splines.f90:107-156 at a tabulated abscissa."""
    n = len(x)
    j = 0
    while j < n - 2 and not (r < x[j + 1]):
        j += 1
    h = x[j + 1] - x[j]
    A = (x[j + 1] - r) / h
    B = 1.0 - A
    return -y[j] / h + y[j + 1] / h + (1 - 3 * A * A) * h / 6 * y2[j] + (3 * B * B - 1) * h / 6 * y2[j + 1]


def read_core_pot_table(path, core_pot_cutoff=1.0e10, core_pot_buffer=0.0):
    """A core_pot table (read_gap.f90:672-760): x, V (tapered), yp1, ypn and dVdx2."""
    rec = _records(path)
    n, yp1, ypn = int(float(rec[0][0])), float(rec[0][1]), float(rec[0][2])
    xs, Vs = [], []
    for r in rec[1:1 + n]:
        x, v = float(r[0]), float(r[1])
        if x <= core_pot_cutoff:
            if x > core_pot_cutoff - core_pot_buffer:
                v = v * 0.5 * (np.cos(np.pi / core_pot_buffer * (x - core_pot_cutoff + core_pot_buffer)) + 1.0)
            xs.append(x)
            Vs.append(v)
    x, V = np.array(xs), np.array(Vs)
    y2 = spline_second_derivatives(x, V, yp1, ypn)
    if yp1 > 0.99e30:
        yp1 = _spline_der_at(x, V, y2, x[0])
    if ypn > 0.99e30:
        ypn = _spline_der_at(x, V, y2, x[-1])
    return dict(x=x, V=V, yp1=yp1, ypn=ypn, dVdx2=y2)


_SOAP_ARRAYS = {"nf": "nf", "rcut": "rcut_hard", "buffer": "rcut_soft", "atom_sigma_r": "atom_sigma_r",
                "atom_sigma_t": "atom_sigma_t", "atom_sigma_r_scaling": "atom_sigma_r_scaling",
                "atom_sigma_t_scaling": "atom_sigma_t_scaling", "amplitude_scaling": "amplitude_scaling",
                "central_weight": "central_weight", "global_scaling": "global_scaling"}


def _soap_block(recs, path_of):
    n_species = 1
    for tok in recs:
        if tok[0] == "n_species":
            n_species = int(_values(tok)[0])
    ns = n_species
    hyp = dict(nf=[4.0] * ns, rcut_hard=[None] * ns, rcut_soft=[0.5] * ns, atom_sigma_r=[None] * ns,
               atom_sigma_t=[None] * ns, atom_sigma_r_scaling=[0.0] * ns, atom_sigma_t_scaling=[0.0] * ns,
               amplitude_scaling=[1.0] * ns, central_weight=[1.0] * ns, global_scaling=[1.0] * ns,
               alpha_max=[8] * ns, l_max=8, radial_enhancement=0, species=[""] * ns)
    out = dict(zeta=2.0, delta=1.0, central_species=0, basis="poly3", scaling_mode="polynomial",
               compress_soap=False, file_compress=None, compress_mode=None, compress=None, file_alphas=None,
               file_desc=None, local_properties=[])
    lp = dict(n=0, labels=[], desc=[], alphas=[], zetas=[], deltas=[], v0s=[])
    for tok in recs:
        k, v = tok[0], _values(tok)
        if k in _SOAP_ARRAYS:
            hyp[_SOAP_ARRAYS[k]] = [float(x) for x in v[:ns]]
        elif k == "n_max":
            hyp["alpha_max"] = [int(float(x)) for x in v[:ns]]
        elif k == "species":
            hyp["species"] = v[:ns]
        elif k == "l_max":
            hyp["l_max"] = int(float(v[0]))
        elif k == "radial_enhancement":
            re_ = int(float(v[0]))
            hyp["radial_enhancement"] = re_ if 0 <= re_ <= 2 else 0  # :85-96 defaults out-of-range to 0
        elif k in ("zeta", "delta"):
            out[k] = float(v[0])
        elif k == "central_species":
            out["central_species"] = int(float(v[0]))
        elif k in ("basis", "scaling_mode"):
            out[k] = v[0]
        elif k == "compress_soap":
            out["compress_soap"] = _bool(v[0])
        elif k == "file_compress_soap":
            out["file_compress"] = None if v[0] == "none" else v[0]
        elif k == "compress_mode":
            out["compress_mode"] = None if v[0] == "none" else v[0]
        elif k == "alphas_sparse":
            out["file_alphas"] = v[0]
        elif k == "desc_sparse":
            out["file_desc"] = v[0]
        elif k in ("has_local_properties", "has_vdw"):
            if _bool(v[0]) and lp["n"] == 0:
                lp["n"] = 1
        elif k == "n_local_properties":
            lp["n"] = int(float(v[0]))
        elif k == "local_property_labels":
            lp["labels"] = v
        elif k in ("local_property_qs", "vdw_qs"):
            lp["desc"] = v
        elif k in ("local_property_alphas", "vdw_alphas"):
            lp["alphas"] = v
        elif k in ("local_property_zetas", "vdw_zeta"):
            lp["zetas"] = [float(x) for x in v]
        elif k in ("local_property_deltas", "vdw_delta"):
            lp["deltas"] = [float(x) for x in v]
        elif k in ("local_property_v0s", "vdw_v0"):
            lp["v0s"] = [float(x) for x in v]
    # the "buffer" is the width of the soft-cutoff region (:424-432)
    hyp["rcut_soft"] = [h if b == 0.0 else h - b for h, b in zip(hyp["rcut_hard"], hyp["rcut_soft"])]
    out["hypers"] = hyp
    if out["compress_soap"]:
        # a compression file takes priority over compress_mode (:489-491)
        if out["file_compress"]:
            out["compress"] = read_compress_file(path_of(out["file_compress"]), ns)
        elif out["compress_mode"]:
            out["compress"] = None  # a soap_turbo recipe (get_compress_indices), resolved on loading
        else:
            raise ValueError("compress_soap without file_compress_soap or compress_mode (read_gap.f90:545-548)")
    if out["file_alphas"] and out["file_desc"]:
        out.update(read_alphas_and_descriptors(path_of(out["file_desc"]), path_of(out["file_alphas"]), "soap_turbo"))
    for j in range(lp["n"]):
        m = dict(label=lp["labels"][j] if j < len(lp["labels"]) else "", zeta=lp["zetas"][j],
                 delta=lp["deltas"][j], V0=lp["v0s"][j])
        m.update(read_alphas_and_descriptors(path_of(lp["desc"][j]), path_of(lp["alphas"][j]), "soap_turbo"))
        out["local_properties"].append(m)
    return out


def _pair_block(kind, recs, path_of):
    out = dict(delta=1.0, sigma=1.0 if kind == "distance_2b" else np.ones(3), buffer=0.5, rcut=None,
               species1=None, species2=None)
    if kind == "angle_3b":
        out.update(species_center=None, kernel_type="exp")
    files = {}
    for tok in recs:
        k, v = tok[0], _values(tok)
        if k == "delta":
            out["delta"] = float(v[0])
        elif k == "sigma":
            out["sigma"] = float(v[0]) if kind == "distance_2b" else np.array([float(x) for x in v[:3]])
        elif k == "rcut":
            out["rcut"] = float(v[0])
        elif k in ("Z1", "z1", "species1"):
            out["species1"] = v[0]
        elif k in ("Z2", "z2", "species2"):
            out["species2"] = v[0]
        elif k in ("Z_center", "z_center", "species_center") and kind == "angle_3b":
            out["species_center"] = v[0]
        elif k == "kernel_type" and kind == "angle_3b":
            out["kernel_type"] = v[0]
        elif k in ("desc_sparse", "alphas_sparse"):
            files[k] = v[0]
    out.update(read_alphas_and_descriptors(path_of(files["desc_sparse"]), path_of(files["alphas_sparse"]), kind))
    return out


def read_gap(path, base_dir=None, core_pot_cutoff=1.0e10, core_pot_buffer=0.0):
    """Every model of a `.gap` file: dict with lists soap_turbo, distance_2b, angle_3b, core_pot
    and rcut_max (the largest cutoff of them, read_gap.f90:89-771)."""
    root = os.getcwd() if base_dir is None else base_dir
    path_of = lambda f: f if os.path.isabs(f) else os.path.join(root, f)
    out = dict(soap_turbo=[], distance_2b=[], angle_3b=[], core_pot=[], rcut_max=0.0)
    kind, recs = None, []
    for ln in _lines(path):
        tok = _tokens(ln)
        if not tok or tok[0][0] in "#!":
            continue
        if tok[0] == "gap_beg":
            kind, recs = (tok[1] if len(tok) > 1 else None), []
            continue
        if tok[0] == "gap_end":
            if kind == "soap_turbo":
                m = _soap_block(recs, path_of)
                out["rcut_max"] = max(out["rcut_max"], max(m["hypers"]["rcut_hard"]))
                out["soap_turbo"].append(m)
            elif kind in ("distance_2b", "angle_3b"):
                m = _pair_block(kind, recs, path_of)
                out["rcut_max"] = max(out["rcut_max"], m["rcut"])
                out[kind].append(m)
            elif kind == "core_pot":
                m = {"species1": None, "species2": None}
                for t in recs:
                    v = _values(t)
                    if t[0] in ("Z1", "z1", "species1"):
                        m["species1"] = v[0]
                    elif t[0] in ("Z2", "z2", "species2"):
                        m["species2"] = v[0]
                    elif t[0] == "core_pot_file":
                        m["file"] = v[0]
                m.update(read_core_pot_table(path_of(m["file"]), core_pot_cutoff, core_pot_buffer))
                out["rcut_max"] = max(out["rcut_max"], float(np.max(m["x"])))
                out["core_pot"].append(m)
            kind, recs = None, []
            continue
        if kind is not None:
            recs.append(tok)
    return out


def load_soap_models(ctx, gap, precision_ready=True):
    """Device models (api.Model) of the soap_turbo blocks of a read_gap result."""
    from .api import Model
    models = []
    for m in gap["soap_turbo"]:
        if m["compress_soap"] and m["compress"] is None:
            raise NotImplementedError(f"compress_mode {m['compress_mode']}: its recipe (soap_turbo's "
                                      "get_compress_indices) is not in the reference sources; give a file_compress_soap")
        if m["basis"] != "poly3":
            raise NotImplementedError(f"basis {m['basis']} is not supported on this path")
        models.append(Model(ctx, m["hypers"], m["Qs"], m["alphas"], m["delta"], m["zeta"],
                            central_species=m["central_species"], compress=m["compress"] if m["compress_soap"] else None))
    return models


def load_terms(ctx, gap, species):
    """Device pair/triplet terms (api.Terms) of the distance_2b, angle_3b and core_pot blocks of a
    read_gap result; `species` lists the species names in channel order (index 1 first), as the
    system's species channels are numbered."""
    from .api import Terms
    idx = {name: i + 1 for i, name in enumerate(species)}
    t = Terms(ctx)
    for b in gap["distance_2b"]:
        t.add_2b(idx[b["species1"]], idx[b["species2"]], b["alphas"], b["cutoff"], b["Qs"], b["rcut"],
                 b["buffer"], b["delta"], b["sigma"], 0.0)
    for c in gap["core_pot"]:
        t.add_core_pot(idx[c["species1"]], idx[c["species2"]], c["x"], c["V"], c["yp1"], c["ypn"], c["dVdx2"])
    for b in gap["angle_3b"]:
        t.add_3b(idx[b["species_center"]], idx[b["species1"]], idx[b["species2"]], b["alphas"], b["cutoff"], b["Qs"],
                 b["rcut"], b["sigma"], b["buffer"], b["delta"], 0.0, b["kernel_type"])
    return t
