"""Generate the reference-pinned golden fixtures from the Force Field X source tree.

Run in a container that has the reference checked out (it is read here as data):

    python tests/golden/make_fixtures.py /path/to/forcefieldx

It parses the reference's own test inputs (modules/potential/src/test/resources/
dhfr.{xyz,key}, ubiquitin.{xyz,key}) and its AMOEBA_BIO_2009 parameter file,
resolves the per-atom AMOEBA parameters with a restatement of Force Field X's
assignment rules, and writes:

  tests/golden/<name>_system.npz   resolved per-atom system (AmoebaSystem.save_npz)
  tests/golden/fixtures.json       keys (box, cutoffs, PME grid) and the golden
                                   per-term energies and interaction counts that
                                   EnergyTest.java asserts for the same inputs.

Assignment rules restated (paths under modules/potential/src/main/java/ffx/potential/):
  multipoles      parameters/MultipoleType.java:545-680 (multipoleTypeFactory order:
                  own type, 1 neighbour, 2 neighbours, 3 neighbours, 1-2 + 1-3 sites)
                  and :787-860 (frame from the signs of the frame types)
  polar groups    parameters/PolarizeType.java:395-416 (growGroup from the seed's
                  polarize group types), called by ParticleMeshEwald.java:2616-2650
  polarize        parameters/PolarizeType.java:138-148 (pdamp = alpha^(1/6), 0 if thole 0)
  vdW             nonbonded/VanDerWaals.java:1421-1433 (reduction toward the single
                  bonded atom), VanDerWaalsForm.java:355-470 (class tables, vdwpr)
"""
from __future__ import annotations

import json
import math
import os
import re
import sys
from collections import defaultdict

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from forcefieldx_b200.system import (AmoebaSystem, FRAME_BISECTOR, FRAME_NONE, FRAME_THREEFOLD,  # noqa: E402
                                     FRAME_ZONLY, FRAME_ZTHENBISECTOR, FRAME_ZTHENX, combine_vdw,
                                     connectivity_lists, pack_multipole_bohr, pme_grid_dim)

PRM = "modules/potential/src/main/java/ffx/potential/parameters/ff/AMOEBA_BIO_2009"
RES = "modules/potential/src/test/resources"
ENERGY_TEST = "modules/potential/src/test/java/ffx/potential/commands/EnergyTest.java"


def parse_prm(path):
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


def parse_xyz(path):
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


def parse_key(path):
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


def golden_from_energy_test(path, xyz_name):
    txt = open(path).read()
    i = txt.index(f'"{xyz_name}"')
    block = txt[i:txt.index("}", i)]
    block = "\n".join(l.split("//")[0] for l in block.split("\n"))
    nums = re.findall(r"-?\d+\.?\d*(?:[eE][-+]?\d+)?|true|false", block.split(",", 1)[1])
    vals = [x for x in nums]
    # Order (EnergyTest constructor): nAtoms, bond E, n, angle E, n, stretch-bend E, n, Urey-Bradley E, n,
    # out-of-plane E, n, torsion E, n, improper E, n, pi-orbital E, n, torsion-torsion E, n,
    # stretch-torsion E, n, angle-torsion E, n, vdW E, n, permanent E, n, polarization E, n, GK E, n, openmm.
    v = vals
    return dict(n_atoms=int(v[0]), vdw=float(v[23]), n_vdw=int(v[24]), permanent=float(v[25]),
                n_permanent=int(v[26]), polarization=float(v[27]), n_polar=int(v[28]),
                source=f"{ENERGY_TEST} ({xyz_name})", tolerance=1.0e-2)


def build(ref_root, name, xyz_file, key_file, prm):
    atoms, vdw, vdwpr, polar, mpoles = prm
    xyz, types, bonds = parse_xyz(os.path.join(ref_root, RES, xyz_file))
    key = parse_key(os.path.join(ref_root, RES, key_file))
    n = len(types)
    n12, n13, n14, n15 = connectivity_lists(n, bonds)
    mp, frame, axis = assign_multipoles(types, n12, n13, mpoles)
    ip11 = polarization_groups(types, n12, polar)
    sym = all(i in ip11[k] for i in range(n) for k in ip11[i])
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
    system = AmoebaSystem(xyz=xyz, multipole=mp, frame=frame, axis=axis, polarizability=alpha, thole=thole,
                          pdamp=pdamp, vdw_type=vtype, red_parent=red_parent, red_factor=red_factor,
                          vdw_inv_rmin=inv, vdw_eps=ee, n12=n12, n13=n13, n14=n14, n15=n15, ip11=ip11)
    system.save_npz(os.path.join(HERE, f"{name}_system.npz"))
    box = [float(key["a-axis"][0]), float(key.get("b-axis", key["a-axis"])[0]),
           float(key.get("c-axis", key["a-axis"])[0])]
    density = float(key.get("pme-mesh-density", ["1.2"])[0])
    grid = [pme_grid_dim(b, density) for b in box]
    keys = dict(box=box, vdw_cutoff=float(key["vdw-cutoff"][0]), ewald_cutoff=float(key["ewald-cutoff"][0]),
                ewald_alpha=float(key["ewald-alpha"][0]), pme_order=int(key.get("pme-order", ["5"])[0]),
                pme_grid=grid, polar_eps=float(key.get("polar-eps", ["1e-6"])[0]))
    return dict(keys=keys, golden=golden_from_energy_test(os.path.join(ref_root, ENERGY_TEST), xyz_file),
                n_atoms=n, ip11_symmetric=bool(sym),
                frames={str(f): int((frame == f).sum()) for f in range(6)})


ERF_TEST = "modules/numerics/src/test/java/ffx/numerics/special/ErfTest.java"
BSPLINE_TEST = "modules/numerics/src/test/java/ffx/numerics/spline/UniformBSplineTest.java"


def numerics_known_answers(ref_root):
    """Known-answer vectors of ErfTest (tolerance 1e-15) and UniformBSplineTest (1e-6)."""
    erf = []
    txt = open(os.path.join(ref_root, ERF_TEST)).read()
    for m in re.finditer(r'\{"Test[^"]*",\s*([^,]+),\s*([^}]+)\}', txt):
        x = eval(m.group(1).replace("e0", "e0"))
        expected = eval(m.group(2))
        erf.append([float(x), float(expected)])
    txt = open(os.path.join(ref_root, BSPLINE_TEST)).read()
    arrays = {m.group(1): [float(v) for v in m.group(2).split(",")]
              for m in re.finditer(r"double\[\] (\w+) = \{([^}]*)\}", txt)}
    cases = []
    for m in re.finditer(r'\{"Order (\d), x = ([0-9.]+)", \d, [^,]+, (\w+), (\w+)\}', txt):
        cases.append(dict(order=int(m.group(1)), x=float(m.group(2)), values=arrays[m.group(3)],
                          derivs=arrays[m.group(4)]))
    return dict(erf=erf, erf_tolerance=1.0e-15, erf_source=ERF_TEST, bspline=cases,
                bspline_tolerance=1.0e-6, bspline_source=BSPLINE_TEST)


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    prm = parse_prm(os.path.join(ref_root, PRM))
    out = {}
    for name, xyz_file, key_file in (("dhfr", "dhfr.xyz", "dhfr.key"),
                                     ("ubiquitin", "ubiquitin.xyz", "ubiquitin.key")):
        out[name] = build(ref_root, name, xyz_file, key_file, prm)
        print(name, json.dumps(out[name]))
    out["numerics"] = numerics_known_answers(ref_root)
    print("numerics", len(out["numerics"]["erf"]), "erf cases,", len(out["numerics"]["bspline"]), "bspline cases")
    with open(os.path.join(HERE, "fixtures.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
