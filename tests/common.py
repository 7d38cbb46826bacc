"""Shared helpers for the parity tests."""
import os

from forcefieldx_b200.ffxio import expand_system
from forcefieldx_b200.system import AmoebaParams, AmoebaSystem

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_system(name, fixtures, **overrides):
    """A reference test system (dhfr, ubiquitin, snare, the small-molecule crystals) and its
    keys from fixtures.json; a space-group system comes expanded to the P1 cell of its mates
    (n_symm set)."""
    s = AmoebaSystem.load_npz(os.path.join(GOLDEN, f"{name}_system.npz"))
    k = fixtures[name]["keys"]
    sg = fixtures[name].get("space_group", "P1")
    angles = tuple(k.get("angles", (90.0, 90.0, 90.0)))
    if sg != "P1":
        s = expand_system(s, k["box"], sg, angles)
    else:
        s.n_symm = 1
    p = dict(box=k["box"], angles=angles, vdw_cutoff=k["vdw_cutoff"], ewald_cutoff=k["ewald_cutoff"],
             ewald_alpha=k["ewald_alpha"], pme_grid=k["pme_grid"], pme_order=k["pme_order"],
             polar_eps=k["polar_eps"])
    p.update(overrides)
    return s, AmoebaParams(**p)


CRYSTALS = ("methylparaben", "paracetamol", "phenacetin", "ethylparaben", "acetanilide")


def ewald_coefficient(cutoff, precision=1.0e-8):
    """EwaldParameters.ewaldCoefficient (nonbonded/pme/EwaldParameters.java:132-166): the
    smallest coefficient with erfc(alpha cutoff) / cutoff below the precision, by doubling
    and 60 extra bisection steps."""
    import math
    eps = precision if precision < 0.1 else 1.0e-8
    ratio, x, i = eps + 1.0, 0.5, 0
    while ratio >= eps:
        i += 1
        x *= 2.0
        ratio = math.erfc(x * cutoff) / cutoff
    lo, hi = 0.0, x
    for _ in range(i + 60):
        x = (lo + hi) / 2.0
        if math.erfc(x * cutoff) / cutoff >= eps:
            lo = x
        else:
            hi = x
    return x
