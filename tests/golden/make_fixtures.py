"""Generate the reference-pinned golden fixtures from the Force Field X source tree.

Run in a container that has the reference checked out (it is read here as data):

    python tests/golden/make_fixtures.py /path/to/forcefieldx

It parses the reference's own test inputs (modules/potential/src/test/resources/
dhfr.{xyz,key}, ubiquitin.{xyz,key}) and its AMOEBA_BIO_2009 parameter file with
forcefieldx_b200.ffxio (a restatement of Force Field X's input formats and atom
typing rules), and writes:

  tests/golden/<name>_system.npz   resolved per-atom system (AmoebaSystem.save_npz)
  tests/golden/fixtures.json       keys (box, cutoffs, PME grid) and the golden
                                   per-term energies and interaction counts that
                                   EnergyTest.java asserts for the same inputs.

The assignment rules and their reference lines are listed in forcefieldx_b200/ffxio.py.
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

from forcefieldx_b200.ffxio import read_key, read_prm, read_xyz, space_group, system_from_types  # noqa: E402
from forcefieldx_b200.system import pme_grid_dim  # noqa: E402

PRM = "modules/potential/src/main/java/ffx/potential/parameters/ff/AMOEBA_BIO_2009"
PRM_PROTEIN = "modules/potential/src/main/java/ffx/potential/parameters/ff/AMOEBA_PROTEIN_2004"
RES = "modules/potential/src/test/resources"
ENERGY_TEST = "modules/potential/src/test/java/ffx/potential/commands/EnergyTest.java"


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
    xyz, types, bonds = read_xyz(os.path.join(ref_root, RES, xyz_file))
    key = read_key(os.path.join(ref_root, RES, key_file))
    system = system_from_types(xyz, types, bonds, prm)
    n = system.n_atoms
    ip11 = system.ip11
    sym = all(i in ip11[k] for i in range(n) for k in ip11[i])
    system.save_npz(os.path.join(HERE, f"{name}_system.npz"))
    box = [float(key["a-axis"][0]), float(key.get("b-axis", key["a-axis"])[0]),
           float(key.get("c-axis", key["a-axis"])[0])]
    density = float(key.get("pme-mesh-density", ["1.2"])[0])
    grid = [pme_grid_dim(b, density) for b in box]
    keys = dict(box=box, vdw_cutoff=float(key["vdw-cutoff"][0]), ewald_cutoff=float(key["ewald-cutoff"][0]),
                ewald_alpha=float(key["ewald-alpha"][0]), pme_order=int(key.get("pme-order", ["5"])[0]),
                pme_grid=grid, polar_eps=float(key.get("polar-eps", ["1e-6"])[0]))
    return dict(keys=keys, golden=golden_from_energy_test(os.path.join(ref_root, ENERGY_TEST), xyz_file),
                n_atoms=n, ip11_symmetric=bool(sym), space_group=space_group(key),
                frames={str(f): int((system.frame == f).sum()) for f in range(6)})


def build_crystal(ref_root, name):
    """A small-molecule crystal of EnergyTest (its .xyz asymmetric unit, .properties keys and
    the .patch parameter file they name): cell edges and angles, space group, cutoffs; the
    Ewald coefficient is the key's or the reference's default 0.545 (EwaldParameters.java:70),
    the PME mesh ReciprocalSpace.initConvolution's on the unit cell (ReciprocalSpace.java:
    909-975)."""
    res = os.path.join(ref_root, RES)
    key = read_key(os.path.join(res, f"{name}.properties"))
    prm = read_prm(os.path.join(res, key["parameters"][0]))
    xyz, types, bonds = read_xyz(os.path.join(res, f"{name}.xyz"))
    system = system_from_types(xyz, types, bonds, prm)
    system.save_npz(os.path.join(HERE, f"{name}_system.npz"))
    box = [float(key["a-axis"][0]), float(key.get("b-axis", key["a-axis"])[0]),
           float(key.get("c-axis", key["a-axis"])[0])]
    angles = [float(key.get(a, ["90.0"])[0]) for a in ("alpha", "beta", "gamma")]
    density = float(key.get("pme-mesh-density", ["1.2"])[0])
    keys = dict(box=box, angles=angles, vdw_cutoff=float(key["vdw-cutoff"][0]),
                ewald_cutoff=float(key["ewald-cutoff"][0]),
                ewald_alpha=float(key.get("ewald-alpha", ["0.545"])[0]), pme_order=5,
                pme_grid=[pme_grid_dim(b, density) for b in box],
                polar_eps=float(key.get("polar-eps", ["1e-6"])[0]))
    return dict(keys=keys, golden=golden_from_energy_test(os.path.join(ref_root, ENERGY_TEST), f"{name}.xyz"),
                n_atoms=system.n_atoms, space_group=space_group(key))


CRYSTALS = ("methylparaben", "paracetamol", "phenacetin", "ethylparaben", "acetanilide")

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
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FFX_REFERENCE_ROOT", "")
    if not ref_root or not os.path.isdir(ref_root):
        sys.exit("usage: make_fixtures.py <reference checkout> (or set FFX_REFERENCE_ROOT)")
    prm = read_prm(os.path.join(ref_root, PRM))
    out = {}
    for name, xyz_file, key_file in (("dhfr", "dhfr.xyz", "dhfr.key"),
                                     ("ubiquitin", "ubiquitin.xyz", "ubiquitin.key")):
        out[name] = build(ref_root, name, xyz_file, key_file, prm)
        print(name, json.dumps(out[name]))
    # SNARE in P212121 (EnergyTest.java:70-104): the asymmetric unit; tests expand it to
    # the P1 cell of its four mates (forcefieldx_b200.ffxio.expand_system).
    prm_protein = read_prm(os.path.join(ref_root, PRM_PROTEIN))
    out["snare"] = build(ref_root, "snare", "1n7s.P212121.xyz", "1n7s.P212121.key", prm_protein)
    print("snare", json.dumps(out["snare"]))
    # Small-molecule crystals in P21/c (monoclinic cells) and Pbca (EnergyTest.java:437-616).
    for name in CRYSTALS:
        out[name] = build_crystal(ref_root, name)
        print(name, json.dumps(out[name]))
    out["numerics"] = numerics_known_answers(ref_root)
    print("numerics", len(out["numerics"]["erf"]), "erf cases,", len(out["numerics"]["bspline"]), "bspline cases")
    with open(os.path.join(HERE, "fixtures.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
