"""Shared helpers for the parity tests."""
import os

from forcefieldx_b200.ffxio import expand_system
from forcefieldx_b200.system import AmoebaParams, AmoebaSystem

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_system(name, fixtures, **overrides):
    """A reference test system (dhfr, ubiquitin, snare) and its keys from fixtures.json;
    a space-group system comes expanded to the P1 cell of its mates (n_symm set)."""
    s = AmoebaSystem.load_npz(os.path.join(GOLDEN, f"{name}_system.npz"))
    k = fixtures[name]["keys"]
    sg = fixtures[name].get("space_group", "P1")
    if sg != "P1":
        s = expand_system(s, k["box"], sg)
    else:
        s.n_symm = 1
    p = dict(box=k["box"], vdw_cutoff=k["vdw_cutoff"], ewald_cutoff=k["ewald_cutoff"],
             ewald_alpha=k["ewald_alpha"], pme_grid=k["pme_grid"], pme_order=k["pme_order"],
             polar_eps=k["polar_eps"])
    p.update(overrides)
    return s, AmoebaParams(**p)
