"""Force Field X input formats: Tinker/FFX XYZ coordinates, keyword (.key) files and
AMOEBA parameter (.prm) files, resolved into an AmoebaSystem + AmoebaParams.

  read_xyz      XYZFilter.readFile (P/parsers/XYZFilter.java): atom count, then one line
                per atom (index, name, x, y, z, atom type, bonded atoms)
  write_xyz     XYZFilter.writeFile: the same layout
  read_key      KeyFilter (P/parsers/KeyFilter.java): keyword, values; '#' comments
  read_prm      ForceFieldFilter: atom, vdw, vdwpr, polarize and multipole records
  load_system   the atom typing Force Field X applies to build the hot path's inputs:
    multipoles   parameters/MultipoleType.java:545-680 (multipoleTypeFactory order: own
                 type, 1 neighbour, 2 neighbours, 3 neighbours, 1-2 + 1-3 sites) and
                 :787-860 (frame from the signs of the frame types)
    polar groups parameters/PolarizeType.java:395-416 (growGroup from the seed's polarize
                 group types), called by ParticleMeshEwald.java:2616-2650
    polarize     parameters/PolarizeType.java:138-148 (pdamp = alpha^(1/6), 0 if thole 0)
    vdW          nonbonded/VanDerWaals.java:1421-1433 (reduction toward the single bonded
                 atom), VanDerWaalsForm.java:355-470 (class tables, vdwpr)
    keys         box (a-axis, b-axis, c-axis), vdw-cutoff, ewald-cutoff, ewald-alpha,
                 pme-order, pme-grid or pme-mesh-density / pme-spacing, polar-eps,
                 polarization, spacegroup
(paths under modules/potential/src/main/java/ffx/potential/).  Space groups with an
orthorhombic cell are expanded to the P1 cell of their symmetry mates (unit_cell): the
reference sums the asymmetric unit's interactions with its mates
(C/SpaceGroup, ParticleMeshEwald symmetry loops); the cell of mates has the same energy
per asymmetric unit.
"""
from __future__ import annotations

import math
import os
import re
from typing import Dict, List, Optional, Tuple

import numpy as np

from .system import (FRAME_BISECTOR, FRAME_NONE, FRAME_THREEFOLD, FRAME_ZONLY, FRAME_ZTHENBISECTOR, FRAME_ZTHENX,
                     POLAR_DIRECT, POLAR_MUTUAL, POLAR_NONE, AmoebaParams, AmoebaSystem, combine_vdw,
                     connectivity_lists, pack_multipole_bohr, pme_grid_dim, tile_system)


def read_prm(path):
    lines = open(path).read().split("\n")
    atoms, vdw, vdwpr, polar, mpoles = {}, {}, {}, {}, {}
    i = 0
    while i < len(lines):
        line = lines[i].split("#")[0].replace("\\", " ")
        tok = line.split()
        i += 1
        if not tok:
            continue
        kw = tok[0].lower()
        if kw == "atom":
            m = re.match(r'\s*atom\s+(\d+)\s+(\d+)\s+(\S+)\s+"[^"]*"\s+(\d+)\s+(\S+)\s+(\d+)', line)
            atoms[int(m.group(1))] = dict(cls=int(m.group(2)), z=int(m.group(4)))
        elif kw == "vdw":
            red = float(tok[4]) if len(tok) > 4 else 0.0
            vdw[int(tok[1])] = (float(tok[2]), float(tok[3]), red)
        elif kw == "vdwpr":
            vdwpr[(int(tok[1]), int(tok[2]))] = (float(tok[3]), float(tok[4]))
        elif kw == "polarize":
            t = int(tok[1])
            a, th = float(tok[2]), float(tok[3])
            nxt = 4
            if len(tok) > 4:
                try:
                    int(tok[4])
                except ValueError:
                    nxt = 5  # direct damping value
            group = [int(x) for x in tok[nxt:]] or None
            polar[t] = dict(alpha=a, thole=th, group=group)
        elif kw == "multipole":
            ints = [int(x) for x in tok[1:-1]]
            charge = float(tok[-1])
            frame_types = [x for x in ints if x != 0]
            nt = len(frame_types)
            if nt == 1:
                frame = FRAME_NONE
            elif nt == 2:
                frame = FRAME_ZONLY
            elif nt == 3:
                frame = FRAME_BISECTOR if (frame_types[1] < 0 or frame_types[2] < 0) else FRAME_ZTHENX
            elif nt == 4:
                frame = None
                if frame_types[2] < 0 and frame_types[3] < 0:
                    frame = FRAME_ZTHENBISECTOR
                    if frame_types[1] < 0:
                        frame = FRAME_THREEFOLD
                if frame is None:
                    frame = FRAME_ZTHENX
            else:
                raise ValueError(line)
            d = [float(x) for x in lines[i].split("#")[0].replace("\\", " ").split()]
            q1 = [float(x) for x in lines[i + 1].split("#")[0].replace("\\", " ").split()]
            q2 = [float(x) for x in lines[i + 2].split("#")[0].replace("\\", " ").split()]
            q3 = [float(x) for x in lines[i + 3].split("#")[0].replace("\\", " ").split()]
            i += 4
            quad = [[q1[0], q2[0], q3[0]], [q2[0], q2[1], q3[1]], [q3[0], q3[1], q3[2]]]
            key = " ".join(str(abs(x)) for x in frame_types)
            # ForceField.addForceFieldType: a later entry with the same key replaces the earlier one.
            mpoles[key] = dict(frame=frame, mp=pack_multipole_bohr(charge, d, quad))
    return atoms, vdw, vdwpr, polar, mpoles


def read_xyz(path):
    lines = open(path).read().split("\n")
    n = int(lines[0].split()[0])
    xyz = np.zeros((n, 3))
    types = np.zeros(n, dtype=np.int64)
    bonds = []
    for a in range(n):
        tok = lines[1 + a].split()
        idx = int(tok[0]) - 1
        assert idx == a
        xyz[a] = [float(tok[2]), float(tok[3]), float(tok[4])]
        types[a] = int(tok[5])
        for b in tok[6:]:
            b = int(b) - 1
            if b > a:
                bonds.append((a, b))
    return xyz, types, np.array(bonds, dtype=np.int64)


def read_key(path):
    kv = {}
    for line in open(path):
        tok = line.split("#")[0].split()
        if len(tok) >= 2:
            kv[tok[0].lower()] = tok[1:]
    return kv


def assign_multipoles(types, n12, n13, mpoles):
    """MultipoleType.multipoleTypeFactory (MultipoleType.java:545-680)."""
    n = len(types)
    mp = np.zeros((n, 10))
    frame = np.zeros(n, dtype=np.int32)
    axis = -np.ones((n, 3), dtype=np.int32)

    def found(i, key, ax):
        if key in mpoles:
            mp[i] = mpoles[key]["mp"]
            frame[i] = mpoles[key]["frame"]
            for s, a in enumerate(ax):
                axis[i, s] = a
            return True
        return False

    for i in range(n):
        k1 = str(types[i])
        if found(i, k1, []):
            continue
        nb = n12[i]
        done = False
        for a2 in nb:
            if found(i, f"{k1} {types[a2]}", [a2]):
                done = True
                break
        if done:
            continue
        for a2 in nb:
            for a3 in nb:
                if a2 == a3:
                    continue
                if found(i, f"{k1} {types[a2]} {types[a3]}", [a2, a3]):
                    done = True
                    break
            if done:
                break
        if done:
            continue
        for a2 in nb:
            for a3 in nb:
                if a2 == a3:
                    continue
                for a4 in nb:
                    if a4 in (a2, a3):
                        continue
                    if found(i, f"{k1} {types[a2]} {types[a3]} {types[a4]}", [a2, a3, a4]):
                        done = True
                        break
                if done:
                    break
            if done:
                break
        if done:
            continue
        for a2 in nb:
            for a3 in n13[i]:
                if found(i, f"{k1} {types[a2]} {types[a3]}", [a2, a3]):
                    done = True
                    break
                for a4 in n13[i]:
                    if a4 != a3 and found(i, f"{k1} {types[a2]} {types[a3]} {types[a4]}", [a2, a3, a4]):
                        done = True
                        break
                if done:
                    break
            if done:
                break
        if not done:
            raise RuntimeError(f"no multipole for atom {i + 1} type {types[i]}")
    return mp, frame, axis


def polarization_groups(types, n12, polar):
    """PolarizeType.growGroup(List, Atom) (PolarizeType.java:395-416)."""
    n = len(types)
    groups = []
    for i in range(n):
        group = [i]
        pt = polar[types[i]]
        if pt["group"] is not None:
            stack = [i]

            def grow(seed):
                for a in n12[seed]:
                    g = polar[types[seed]]["group"] or []
                    if types[a] in g and a not in group:
                        group.append(a)
                        grow(a)

            grow(i)
        groups.append(sorted(group))
    return groups


def write_xyz(path, xyz, types, bonds, names=None, title="") -> None:
    """XYZFilter.writeFile layout: count and title, then index, name, x, y, z, type, bonds."""
    xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    n = xyz.shape[0]
    nb: List[List[int]] = [[] for _ in range(n)]
    for a, b in np.asarray(bonds, dtype=np.int64).reshape(-1, 2):
        nb[a].append(int(b))
        nb[b].append(int(a))
    with open(path, "w") as f:
        f.write(f"{n:6d}  {title}\n")
        for a in range(n):
            name = names[a] if names is not None else "X"
            links = "".join(f"{b + 1:6d}" for b in sorted(nb[a]))
            f.write(f"{a + 1:6d}  {name:<3s}{xyz[a, 0]:12.6f}{xyz[a, 1]:12.6f}{xyz[a, 2]:12.6f}{int(types[a]):6d}{links}\n")


# Symmetry operators (fractional: x' = R x + t), standard settings of the International
# Tables, in the order Force Field X's SpaceGroupDefinitions lists them
# (crystal/SpaceGroupDefinitions.java: P-1 :116-126, P21 :146-156, P21/c :312-328,
# C2/c :329-349, Pbca :1270-1287; the P212121 order follows the reference's
# 1n7s.P212121 / 1n7s.P1 test pair).
def _op(r, t):
    return (np.array(r, dtype=np.float64), np.array(t, dtype=np.float64))


_I, _INV = np.eye(3), -np.eye(3)
_M2Y, _MY = np.diag([-1.0, 1.0, -1.0]), np.diag([1.0, -1.0, 1.0])   # 2-fold along b; mirror normal to b

SPACE_GROUPS = {
    "P1": [_op(np.eye(3), (0, 0, 0))],
    "P-1": [_op(_I, (0, 0, 0)), _op(_INV, (0, 0, 0))],
    "P21": [_op(_I, (0, 0, 0)), _op(_M2Y, (0, 0.5, 0))],
    "P21/C": [_op(_I, (0, 0, 0)), _op(_INV, (0, 0, 0)), _op(_M2Y, (0, 0.5, 0.5)), _op(_MY, (0, 0.5, 0.5))],
    "C2/C": [_op(_I, (0, 0, 0)), _op(_M2Y, (0, 0, 0.5)), _op(_INV, (0, 0, 0)), _op(_MY, (0, 0, 0.5)),
             _op(_I, (0.5, 0.5, 0)), _op(_M2Y, (0.5, 0.5, 0.5)), _op(_INV, (0.5, 0.5, 0)), _op(_MY, (0.5, 0.5, 0.5))],
    "PBCA": [_op(_I, (0, 0, 0)), _op(np.diag([-1.0, -1.0, 1.0]), (0.5, 0, 0.5)),
             _op(np.diag([-1.0, 1.0, -1.0]), (0, 0.5, 0.5)), _op(np.diag([1.0, -1.0, -1.0]), (0.5, 0.5, 0)),
             _op(_INV, (0, 0, 0)), _op(np.diag([1.0, 1.0, -1.0]), (0.5, 0, 0.5)),
             _op(np.diag([1.0, -1.0, 1.0]), (0, 0.5, 0.5)), _op(np.diag([-1.0, 1.0, 1.0]), (0.5, 0.5, 0))],
    "P222": [_op(np.eye(3), (0, 0, 0)), _op(np.diag([-1, -1, 1]), (0, 0, 0)),
             _op(np.diag([-1, 1, -1]), (0, 0, 0)), _op(np.diag([1, -1, -1]), (0, 0, 0))],
    "P2221": [_op(np.eye(3), (0, 0, 0)), _op(np.diag([-1, -1, 1]), (0, 0, 0.5)),
              _op(np.diag([-1, 1, -1]), (0, 0, 0.5)), _op(np.diag([1, -1, -1]), (0, 0, 0))],
    "P21212": [_op(np.eye(3), (0, 0, 0)), _op(np.diag([-1, -1, 1]), (0, 0, 0)),
               _op(np.diag([-1, 1, -1]), (0.5, 0.5, 0)), _op(np.diag([1, -1, -1]), (0.5, 0.5, 0))],
    "P212121": [_op(np.eye(3), (0, 0, 0)), _op(np.diag([-1, -1, 1]), (0.5, 0, 0.5)),
                _op(np.diag([1, -1, -1]), (0.5, 0.5, 0)), _op(np.diag([-1, 1, -1]), (0, 0.5, 0.5))],
}


def space_group(key: Dict[str, List[str]]) -> str:
    sg = key.get("spacegroup", ["P1"])[0].upper().replace(" ", "")
    if sg not in SPACE_GROUPS:
        raise ValueError(f"space group {sg}: supported are {sorted(SPACE_GROUPS)}")
    return sg


def cell_matrices(box, angles=(90.0, 90.0, 90.0)):
    """(A^-1, A) of Crystal.updateCrystal (C/Crystal.java:1428-1548): the rows of A^-1 are
    the lattice vectors, x_frac = x A, x = x_frac A^-1; orthorhombic, monoclinic and
    general branches as the library and the oracle build them."""
    a, b, c = (float(v) for v in box)
    al, be, ga = (float(v) if float(v) > 0 else 90.0 for v in angles)
    if al == 90.0 and be == 90.0 and ga == 90.0:
        return np.diag([a, b, c]), np.diag([1.0 / a, 1.0 / b, 1.0 / c])
    deg = 0.017453292519943295
    if al == 90.0 and ga == 90.0:
        cos_a, sin_b, cos_b, sin_g, cos_g = 0.0, math.sin(be * deg), math.cos(be * deg), 1.0, 0.0
        beta_term, gamma_term = 0.0, sin_b
    else:
        cos_a, sin_b, cos_b = math.cos(al * deg), math.sin(be * deg), math.cos(be * deg)
        sin_g, cos_g = math.sin(ga * deg), math.cos(ga * deg)
        beta_term = (cos_a - cos_b * cos_g) / sin_g
        gamma_term = math.sqrt(sin_b * sin_b - beta_term * beta_term)
    ai = np.array([[a, 0.0, 0.0], [b * cos_g, b * sin_g, 0.0], [c * cos_b, c * beta_term, c * gamma_term]])
    return ai, np.linalg.inv(ai)


def expand_coordinates(xyz, box, sg: str, angles=(90.0, 90.0, 90.0)) -> np.ndarray:
    """Coordinates of the unit cell's symmetry mates of an asymmetric unit, mate after mate
    (x_frac' = R x_frac + t; no wrapping, the energy is periodic)."""
    xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    box = np.asarray(box, dtype=np.float64)
    ai, a = cell_matrices(box, angles)
    if np.count_nonzero(ai - np.diag(np.diag(ai))) == 0:
        frac = xyz / box
        return np.concatenate([((frac @ R.T) + t) * box for R, t in SPACE_GROUPS[sg]])
    frac = xyz @ a
    return np.concatenate([((frac @ R.T) + t) @ ai for R, t in SPACE_GROUPS[sg]])


def expand_system(system: AmoebaSystem, box, sg: str, angles=(90.0, 90.0, 90.0)) -> AmoebaSystem:
    """A resolved asymmetric-unit system expanded to the P1 cell of its symmetry mates
    (attributes n_symm, n_asu set)."""
    cell = tile_system(system, expand_coordinates(system.xyz, box, sg, angles), len(SPACE_GROUPS[sg]))
    cell.n_symm = len(SPACE_GROUPS[sg])
    cell.n_asu = system.n_atoms
    return cell


def params_from_key(key: Dict[str, List[str]], **overrides) -> AmoebaParams:
    """AmoebaParams from a key file's keywords (ForceFieldEnergy / PME defaults otherwise)."""
    space_group(key)
    a = float(key["a-axis"][0])
    box = [a, float(key.get("b-axis", [a])[0]), float(key.get("c-axis", [a])[0])]
    angles = tuple(float(key.get(ang, ["90.0"])[0]) for ang in ("alpha", "beta", "gamma"))
    kw = dict(box=box, angles=angles)
    for name, field, conv in (("vdw-cutoff", "vdw_cutoff", float), ("ewald-cutoff", "ewald_cutoff", float),
                              ("ewald-alpha", "ewald_alpha", float), ("pme-order", "pme_order", int),
                              ("polar-eps", "polar_eps", float), ("pme-mesh-density", "pme_mesh_density", float)):
        if name in key:
            kw[field] = conv(key[name][0])
    if "pme-grid" in key:
        g = [int(v) for v in key["pme-grid"]]
        kw["pme_grid"] = (g + [g[-1]] * 3)[:3]
    else:
        dens = kw.get("pme_mesh_density", 1.2)
        kw["pme_grid"] = [pme_grid_dim(b, dens) for b in box]
    if "polarization" in key:
        kw["polarization"] = {"MUTUAL": POLAR_MUTUAL, "DIRECT": POLAR_DIRECT,
                              "NONE": POLAR_NONE}[key["polarization"][0].upper()]
    kw.update(overrides)
    return AmoebaParams(**kw)


def system_from_types(xyz, types, bonds, prm) -> AmoebaSystem:
    """Resolve per-atom AMOEBA parameters for atoms of the given types and bonds."""
    atoms, vdw, vdwpr, polar, mpoles = prm
    n = len(types)
    n12, n13, n14, n15 = connectivity_lists(n, bonds)
    mp, frame, axis = assign_multipoles(types, n12, n13, mpoles)
    ip11 = polarization_groups(types, n12, polar)
    alpha = np.array([polar[t]["alpha"] for t in types])
    thole = np.array([polar[t]["thole"] for t in types])
    pdamp = np.where(thole == 0.0, 0.0, alpha ** (1.0 / 6.0))
    classes = sorted({atoms[t]["cls"] for t in types})
    cidx = {c: j for j, c in enumerate(classes)}
    vtype = np.array([cidx[atoms[t]["cls"]] for t in types], dtype=np.int32)
    radius = [vdw[c][0] for c in classes]
    eps = [vdw[c][1] for c in classes]
    pairs = {}
    for (c1, c2), val in vdwpr.items():
        if c1 in cidx and c2 in cidx:
            pairs[(cidx[c1], cidx[c2])] = val
    inv, ee = combine_vdw(radius, eps, pairs)
    red_parent = np.arange(n, dtype=np.int32)
    red_factor = np.zeros(n)
    for a in range(n):
        red = vdw[atoms[types[a]]["cls"]][2]
        if red > 0.0 and len(n12[a]) == 1:
            red_parent[a] = n12[a][0]
            red_factor[a] = red
    return AmoebaSystem(xyz=np.asarray(xyz, dtype=np.float64), multipole=mp, frame=frame, axis=axis,
                        polarizability=alpha, thole=thole, pdamp=pdamp, vdw_type=vtype, red_parent=red_parent,
                        red_factor=red_factor, vdw_inv_rmin=inv, vdw_eps=ee, n12=n12, n13=n13, n14=n14, n15=n15,
                        ip11=ip11)


def load_system(xyz_path: str, key_path: str, prm_path: Optional[str] = None, expand_symmetry: bool = True,
                **overrides) -> Tuple[AmoebaSystem, AmoebaParams]:
    """An FFX structure: coordinates and topology from the XYZ file, keys from the key
    file, parameters from ``prm_path`` (else the key file's ``parameters`` keyword,
    relative to the key file).  A space group other than P1 is expanded to the P1 unit
    cell of the symmetry mates (see unit_cell); the returned system then carries the
    attributes n_symm and n_asu."""
    key = read_key(key_path)
    if prm_path is None:
        if "parameters" not in key:
            raise ValueError("no parameter file: pass prm_path or set the parameters keyword")
        prm_path = key["parameters"][0]
        if not os.path.isabs(prm_path):
            prm_path = os.path.join(os.path.dirname(os.path.abspath(key_path)), prm_path)
    xyz, types, bonds = read_xyz(xyz_path)
    params = params_from_key(key, **overrides)
    sg = space_group(key)
    n_asu = len(types)
    if expand_symmetry and sg != "P1":
        xyz, types, bonds = unit_cell(xyz, types, bonds, params.box, sg, params.angles)
    system = system_from_types(xyz, types, bonds, read_prm(prm_path))
    system.n_symm = len(types) // n_asu
    system.n_asu = n_asu
    return system, params


def unit_cell(xyz, types, bonds, box, sg: str, angles=(90.0, 90.0, 90.0)):
    """The P1 unit cell of an asymmetric unit: every symmetry mate's atoms (types and bonds
    repeated with the atom offset of the mate).  The crystal energy per asymmetric unit is
    the cell's energy over the number of mates, and the asymmetric unit's gradient is the
    first mate's rows of the cell's gradient (the mates are images of one another)."""
    n = len(types)
    ops = SPACE_GROUPS[sg]
    cell_xyz = expand_coordinates(xyz, box, sg, angles)
    cell_types = np.concatenate([np.asarray(types)] * len(ops))
    b = np.asarray(bonds, dtype=np.int64).reshape(-1, 2)
    cell_bonds = np.concatenate([b + m * n for m in range(len(ops))])
    return cell_xyz, cell_types, cell_bonds
