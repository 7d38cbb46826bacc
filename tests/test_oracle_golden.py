"""Pin the CPU oracle to the reference's own golden energies and interaction counts.

EnergyTest.java (modules/potential/src/test/java/ffx/potential/commands/EnergyTest.java)
asserts per-term energies to 1e-2 kcal/mol and exact interaction counts for DHFR
(:147-182), ubiquitin (:363-398) and SNARE in P212121 (:70-104, AMOEBA_PROTEIN_2004),
and per-term energies for five small-molecule crystals (:437-616): methylparaben,
paracetamol, phenacetin and ethylparaben in P21/c (monoclinic cells) and acetanilide in
Pbca; tests/golden/make_fixtures.py resolved the same inputs into tests/golden/*_system.npz.
"""
import dataclasses

import pytest

from oracle import binding as ob
from tests.common import CRYSTALS, ewald_coefficient, golden_system


@pytest.mark.parametrize("name", ["ubiquitin", "dhfr", "snare"])
def test_oracle_matches_reference_golden(name, fixtures):
    """SNARE (EnergyTest.java:70-104) is the P212121 asymmetric unit, evaluated as the P1
    cell of its four mates: energies and counts per asymmetric unit."""
    system, params = golden_system(name, fixtures)
    g = fixtures[name]["golden"]
    tol = g["tolerance"]
    r = ob.energy(system, params, gradient=False)
    assert r["status"] == 0
    t, c = r["terms"] / system.n_symm, r["counts"]
    assert abs(t[0] - g["vdw"]) < tol
    assert abs(t[1] - g["permanent"]) < tol
    assert abs(t[2] - g["polarization"]) < tol
    assert c[0] == system.n_symm * g["n_vdw"]
    assert c[1] == system.n_symm * g["n_permanent"]


@pytest.mark.parametrize("name", CRYSTALS)
def test_oracle_matches_crystal_goldens(name, fixtures):
    """The P1 cell of the mates of each asymmetric unit, with lists of every lattice image
    (the cells are narrower than twice the cutoffs); energies per asymmetric unit at the
    reference test's 1e-2 kcal/mol.  (The reference counts interactions with images of the
    asymmetric unit by its own bookkeeping, so counts are not compared.)"""
    system, params = golden_system(name, fixtures)
    g = fixtures[name]["golden"]
    r = ob.energy(system, params, gradient=False)
    assert r["status"] == 0
    t = r["terms"] / system.n_symm
    assert abs(t[0] - g["vdw"]) < 1.0e-8 * max(1.0, abs(g["vdw"]))     # the vdW term has no mesh: exact
    assert abs(t[1] - g["permanent"]) < g["tolerance"]
    assert abs(t[2] - g["polarization"]) < g["tolerance"]


def test_oracle_methylparaben_at_the_cutoff_derived_ewald_coefficient(fixtures):
    """Methylparaben's golden permanent energy is reproduced to 1e-6 with the Ewald
    coefficient EwaldParameters.ewaldCoefficient derives from its 8 A cutoff at 1e-8."""
    system, params = golden_system("methylparaben", fixtures)
    params = dataclasses.replace(params, ewald_alpha=ewald_coefficient(params.ewald_cutoff), polarization=0)
    r = ob.energy(system, params, gradient=False)
    assert abs(r["terms"][1] / system.n_symm - fixtures["methylparaben"]["golden"]["permanent"]) < 1.0e-5