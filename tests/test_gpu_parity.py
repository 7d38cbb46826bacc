"""Parity of the CUDA path (through the C ABI) with the CPU FP64 oracle.

Bar (plain FP64 form): bit-identical neighbour pair set, every energy term within
1e-8 relative, gradient RMS within 1e-6 kcal/mol/A, identical interaction counts and
PCG iteration counts, induced dipoles within 1e-8 e*A RMS.  The oracle is pinned to
the reference's golden energies (tests/test_oracle_golden.py), and the reference
goldens are checked here directly as well.
"""
import numpy as np
import pytest

from forcefieldx_b200.energy import EnergyException, ForceFieldEnergy
from forcefieldx_b200.system import WATER_24K, WATER_648, water_box, water_params
from oracle import binding as ob
from tests.common import golden_system

pytestmark = pytest.mark.gpu

E_REL = 1.0e-8       # per-term relative energy tolerance
G_RMS = 1.0e-6       # gradient RMS tolerance, kcal/mol/A
U_RMS = 1.0e-8       # induced dipole RMS tolerance, e*A


def compare(system, params, check_pairs=True):
    ref = ob.energy(system, params)
    assert ref["status"] == 0
    with ForceFieldEnergy(system, params) as ffe:
        e, g = ffe.energy_and_gradient(system.xyz)
        terms, counts = ffe.terms.copy(), ffe.counts.copy()
        u, ucr = ffe.get_induced_dipoles()
        pairs = ffe.neighbor_pairs() if check_pairs else None
    rel = np.abs(terms - ref["terms"]) / np.maximum(np.abs(ref["terms"]), 1.0)
    assert rel.max() < E_REL, (terms, ref["terms"], rel)
    rms = float(np.sqrt(np.mean((g - ref["grad"]) ** 2)))
    assert rms < G_RMS, rms
    assert counts[0] == ref["counts"][0]          # vdW interactions
    assert counts[1] == ref["counts"][1]          # permanent interactions
    assert counts[2] == ref["counts"][2]          # PCG iterations
    assert np.sqrt(np.mean((u - ref["induced"]) ** 2)) < U_RMS
    assert np.sqrt(np.mean((ucr - ref["induced_cr"]) ** 2)) < U_RMS
    if check_pairs:
        ref_pairs = ob.neighbor_pairs(system, params)
        a = np.unique(pairs[:, 0].astype(np.int64) * system.n_atoms + pairs[:, 1])
        b = np.unique(ref_pairs[:, 0].astype(np.int64) * system.n_atoms + ref_pairs[:, 1])
        assert a.size == pairs.shape[0]
        assert np.array_equal(a, b)
    return terms, counts, g, ref


def test_water_648():
    s = water_box(6, 18.643, seed=21)
    p = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 20))
    compare(s, p)


def test_water_648_buffered_list_beyond_half_box():
    """The reference's CPU-runnable case (216 waters, 18.643 A, 9 A vdW, 7 A Ewald, PME 20^3):
    the 11 A buffered list is longer than half the edge, where the reference switches to
    replicate cells; every interaction cutoff is shorter, so each pair has one image."""
    s = water_box(WATER_648["n_side"], WATER_648["edge"], seed=3)
    p = water_params(WATER_648["edge"], pme_grid=WATER_648["grid"])
    compare(s, p)


@pytest.mark.parametrize("name", ["ubiquitin", "dhfr", "snare"])
def test_reference_golden(name, fixtures):
    """DHFR and ubiquitin in P1; SNARE in P212121 as the P1 cell of its four mates, whose
    energy per asymmetric unit is the reference's P212121 golden."""
    s, p = golden_system(name, fixtures)
    terms, counts, _, _ = compare(s, p)
    gold = fixtures[name]["golden"]
    m = s.n_symm
    assert abs(terms[0] / m - gold["vdw"]) < gold["tolerance"]
    assert abs(terms[1] / m - gold["permanent"]) < gold["tolerance"]
    assert abs(terms[2] / m - gold["polarization"]) < gold["tolerance"]
    assert counts[0] == m * gold["n_vdw"] and counts[1] == m * gold["n_permanent"]


def test_water_24k():
    s = water_box(WATER_24K["n_side"], WATER_24K["edge"])
    p = water_params(WATER_24K["edge"], pme_grid=WATER_24K["grid"])
    compare(s, p)


def test_repeated_calls_and_list_reuse():
    s = water_box(6, 18.643, seed=4)
    p = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 20))
    with ForceFieldEnergy(s, p) as ffe:
        e1, g1 = ffe.energy_and_gradient(s.xyz)
        assert ffe.count("list_builds") == 1
        e2, g2 = ffe.energy_and_gradient(s.xyz)
        assert ffe.count("list_builds") == 0          # no motion: list kept
        assert abs(e1 - e2) < 1e-9 * abs(e1)
        x = s.xyz + 0.3                               # small move: list kept, energies change
        e3, _ = ffe.energy_and_gradient(x)
        assert ffe.count("list_builds") == 0
        ref = ob.energy(s, p, xyz=x)
        assert abs(e3 - ref["terms"][9]) < 1e-8 * abs(e3)
        x = s.xyz.copy()
        x[0] += 1.5                                   # beyond half the buffer: rebuild
        ffe.energy_and_gradient(x)
        assert ffe.count("list_builds") == 1


def test_fd_gradient_gpu():
    s = water_box(6, 18.643, seed=9)
    p = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 20))
    rng = np.random.default_rng(1)
    h = 1.0e-5
    with ForceFieldEnergy(s, p) as ffe:
        _, g = ffe.energy_and_gradient(s.xyz)
        for atom in rng.choice(s.n_atoms, 4, replace=False):
            for d in range(3):
                x = s.xyz.copy()
                x[atom, d] += h
                ep = ffe.energy(x)
                x[atom, d] -= 2 * h
                em = ffe.energy(x)
                assert abs((ep - em) / (2 * h) - g[atom, d]) < 1.0e-2


def test_error_status_codes():
    s = water_box(4, 12.4, seed=2)
    with pytest.raises(EnergyException) as ei:
        ForceFieldEnergy(s, water_params(12.4, pme_grid=(16, 16, 16), pme_order=4))   # only order 5
    assert ei.value.status == 1
    s = water_box(6, 18.643, seed=2)
    p = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 20), max_scf_iter=1)
    with ForceFieldEnergy(s, p) as ffe:
        with pytest.raises(EnergyException) as ei:
            ffe.energy(s.xyz)
        assert ei.value.status == 4                                       # SCF_MAXITER
        x = s.xyz.copy()
        x[3, 1] = np.nan
        with pytest.raises(EnergyException) as ei:
            ffe.energy(x)
        assert ei.value.status == 5                                       # NONFINITE
    p = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 4))
    with pytest.raises(EnergyException) as ei:
        ForceFieldEnergy(s, p)                                            # a mesh shorter than the B-spline order
    assert ei.value.status == 1


@pytest.mark.parametrize("precision", [0, 1])
def test_mesh_with_prime_factors_above_seven(precision):
    """Mesh lengths 22 = 2 x 11, 26 = 2 x 13 and 33 = 3 x 11 take the general radix pass, as
    the reference's Complex transforms any length (Complex.java:173-330)."""
    s = water_box(6, 18.643, seed=61)
    p = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(22, 26, 33), precision=precision)
    if precision == 0:
        compare(s, p, check_pairs=False)
        return
    # Mixed form: this box's total cancels to ~50 kcal/mol, so the terms are held to 1e-5 of
    # the largest term's magnitude, the gradient to the mixed bar's 1e-3 RMS.
    ref = ob.energy(s, p)
    with ForceFieldEnergy(s, p) as ffe:
        e, g = ffe.energy_and_gradient(s.xyz)
        terms = ffe.terms.copy()
    assert np.abs(terms - ref["terms"]).max() < 1e-5 * np.abs(ref["terms"]).max(), (terms, ref["terms"])
    assert float(np.sqrt(np.mean((g - ref["grad"]) ** 2))) < 1e-3


@pytest.mark.parametrize("precision", [0, 1])
def test_graph_replay_matches_direct_launches(precision):
    """The captured graph (PCG loop as a device-side while node) gives the direct path's
    results: bitwise in the mixed form, to FP64 rounding in the plain form (its mesh
    spreading uses floating-point atomics)."""
    s = water_box(6, 18.643, seed=5)
    p = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 20), precision=precision)
    rng = np.random.default_rng(7)
    xs = [s.xyz + rng.normal(0.0, 0.05, s.xyz.shape) for _ in range(3)]
    res = {}
    for mode in (True, False):
        with ForceFieldEnergy(s, p) as ffe:
            ffe.set_graph_mode(mode)
            out = []
            for x in [s.xyz] + xs:
                e, g = ffe.energy_and_gradient(x)
                out.append((ffe.terms.copy(), g.copy(), int(ffe.count("scf_iter"))))
            res[mode] = out
    for (ta, ga, ia), (tb, gb, ib) in zip(res[True], res[False]):
        assert ia == ib
        if precision == 1:
            assert np.array_equal(ta, tb) and np.array_equal(ga, gb)
        else:
            assert np.max(np.abs(ta - tb) / np.maximum(np.abs(tb), 1.0)) < 1e-11
            assert np.max(np.abs(ga - gb)) < 1e-9


def test_graph_replay_reports_scf_errors():
    s = water_box(6, 18.643, seed=2)
    p = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 20), max_scf_iter=2)
    with ForceFieldEnergy(s, p) as ffe:
        for _ in range(3):                      # the first call builds the list; later ones replay
            with pytest.raises(EnergyException) as ei:
                ffe.energy(s.xyz)
            assert ei.value.status == 4         # SCF_MAXITER, decided on the device


def test_crystal_energy_p212121(fixtures):
    """CrystalEnergy on the SNARE asymmetric unit: energy per asymmetric unit and its
    gradient, against the oracle's P1 cell of the four mates."""
    from forcefieldx_b200.energy import CrystalEnergy
    from forcefieldx_b200.system import AmoebaSystem
    from tests.common import GOLDEN
    import os
    asu = AmoebaSystem.load_npz(os.path.join(GOLDEN, "snare_system.npz"))
    cell, p = golden_system("snare", fixtures)
    ref = ob.energy(cell, p)
    with CrystalEnergy(asu, p, "P212121") as ce:
        e, g = ce.energy_and_gradient(asu.xyz)
    assert abs(e - ref["terms"][9] / 4) < 1e-8 * abs(ref["terms"][9] / 4)
    assert float(np.sqrt(np.mean((g - ref["grad"][:asu.n_atoms]) ** 2))) < 1e-6
