"""Extended-XYZ structures, as TurboGAP reads and writes them (src/xyz/read_xyz.f90,
src/xyz/write_xyz.f90), so structure files drive the device path and trajectories come back out.

Reading (read_n_sites_properties :376-425, read_xyz_line :431-486). Each frame is a line with the
number of atoms, a comment line and one line per atom. The comment line holds
`Lattice="ax ay az bx by bz cx cy cz"` (the three cell vectors) and `Properties=name:type:count:...`
(keys case-insensitive); the atom columns follow Properties: `species` (S:1), `pos`/`positions`
(R:3), `vel`/`velocities` (R:3), `fix_atoms`/`fix_atom` (3 flags), `mass`/`masses` (R:1, amu;
the reference multiplies by 103.6426965268 for eV fs^2/A^2, read_xyz.f90:255); other properties
are skipped by their column count. A file may hold several frames, read in order.

Writing (write_xyz.f90:177-360): the same layout with Lattice, Properties
(species:S:1:pos:R:3[:vel:R:3][:forces:R:3][:local_energy:R:1]), and optional energy= and
virial="..." keys, numbers printed to full double precision.
"""
import re

import numpy as np

_KV = re.compile(r'(\w+)\s*=\s*("([^"]*)"|\S+)')


def _header(line):
    """Key=value pairs of a comment line (quoted values may hold blanks)."""
    out = {}
    for m in _KV.finditer(line):
        out[m.group(1).lower()] = m.group(3) if m.group(3) is not None else m.group(2)
    return out


def _columns(properties):
    """(name, type, count) triples of a Properties string."""
    t = properties.split(":")
    if len(t) % 3:
        raise ValueError(f"malformed Properties={properties}")
    return [(t[i].lower(), t[i + 1].upper(), int(t[i + 2])) for i in range(0, len(t), 3)]


def _flag(s):
    return s.strip(".").upper() in ("T", "TRUE", "1")


def read_xyz(path):
    """Every frame of an extended-XYZ file: dicts with n, lattice (3, 3; rows a, b, c), species
    (list of str), positions (n, 3) and, when present, velocities (n, 3), masses (n, amu),
    fix_atom (n, 3 bool) and the remaining header keys (info)."""
    with open(path) as f:
        lines = f.read().splitlines()
    frames, i = [], 0
    while i < len(lines):
        if not lines[i].strip():
            i += 1
            continue
        n = int(lines[i].split()[0])
        head = _header(lines[i + 1])
        cols = _columns(head.get("properties", "species:S:1:pos:R:3"))
        fr = dict(n=n, species=[], positions=np.zeros((n, 3)))
        if "lattice" in head:
            fr["lattice"] = np.array([float(x) for x in head["lattice"].split()]).reshape(3, 3)
        names = [c[0] for c in cols]
        if "vel" in names or "velocities" in names:
            fr["velocities"] = np.zeros((n, 3))
        if "mass" in names or "masses" in names:
            fr["masses"] = np.zeros(n)
        if "fix_atoms" in names or "fix_atom" in names:
            fr["fix_atom"] = np.zeros((n, 3), bool)
        for a in range(n):
            tok = lines[i + 2 + a].split()
            j = 0
            for name, _, cnt in cols:
                v = tok[j:j + cnt]
                if name == "species":
                    fr["species"].append(v[0])
                elif name in ("pos", "positions"):
                    fr["positions"][a] = [float(x) for x in v]
                elif name in ("vel", "velocities"):
                    fr["velocities"][a] = [float(x) for x in v]
                elif name in ("mass", "masses"):
                    fr["masses"][a] = float(v[0])
                elif name in ("fix_atoms", "fix_atom"):
                    fr["fix_atom"][a] = [_flag(x) for x in v]
                j += cnt
        fr["info"] = {k: v for k, v in head.items() if k not in ("lattice", "properties")}
        frames.append(fr)
        i += 2 + n
    return frames


def write_xyz(path, frames, append=False):
    """Writes frames (dicts as read_xyz returns, plus optional forces (n, 3), local_energy (n,),
    energy and virial (3, 3)) in the layout TurboGAP writes."""
    if isinstance(frames, dict):
        frames = [frames]
    with open(path, "a" if append else "w") as f:
        for fr in frames:
            n = len(fr["species"])
            cols = ["species:S:1", "pos:R:3"]
            extra = [k for k in ("velocities", "forces") if fr.get(k) is not None]
            cols += [{"velocities": "vel:R:3", "forces": "forces:R:3"}[k] for k in extra]
            if fr.get("local_energy") is not None:
                cols.append("local_energy:R:1")
            head = [f"Properties={':'.join(cols)}"]
            if fr.get("lattice") is not None:
                head.append('Lattice="' + " ".join(f"{x:.17g}" for x in np.asarray(fr["lattice"]).ravel()) + '"')
            if fr.get("energy") is not None:
                head.append(f"energy={fr['energy']:.17g}")
            if fr.get("virial") is not None:
                v = np.asarray(fr["virial"])
                head.append('virial="' + " ".join(f"{v[r, c]:.17g}" for r in range(3) for c in range(3)) + '"')
            f.write(f"{n}\n {' '.join(head)}\n")
            for a in range(n):
                row = [fr["species"][a]] + [f"{x:.17g}" for x in fr["positions"][a]]
                for k in extra:
                    row += [f"{x:.17g}" for x in fr[k][a]]
                if fr.get("local_energy") is not None:
                    row.append(f"{fr['local_energy'][a]:.17g}")
                f.write(" ".join(row) + "\n")


def species_channels(frame, species_types):
    """Species channel (1-based index into species_types) of every atom; an unknown species is an
    error, as in read_xyz_lines (:277-283)."""
    idx = {s: k + 1 for k, s in enumerate(species_types)}
    try:
        return np.array([idx[s] for s in frame["species"]], np.int32)
    except KeyError as e:
        raise ValueError(f"atom species {e} is not among {species_types}") from None
