"""General cells and space groups on the GPU against the oracle and the reference's goldens.

* The five small-molecule crystals of EnergyTest (:437-616): methylparaben, paracetamol,
  phenacetin and ethylparaben in P21/c (monoclinic cells, beta up to 147 degrees) and
  acetanilide in Pbca, each as the P1 cell of its symmetry mates with lists of every lattice
  image.  FP64 form: bit-identical image-pair set, 1e-8 per term, 1e-6 gradient RMS and
  identical counts against the oracle, and the goldens per asymmetric unit (vdW to 1e-8, the
  electrostatic terms at the reference test's 1e-2).  Mixed form: every term within 1e-5 of
  the largest term, 1e-3 gradient RMS.
* A triclinic water box whose widths exceed twice the cutoffs: minimum-image lists from the
  cell builder on fractional cells, against the oracle with a bit-identical pair set.
* ffxg_set_box from a cube to a monoclinic cell of the same atoms against a new handle.
"""
import math

import numpy as np
import pytest

from forcefieldx_b200.energy import ForceFieldEnergy
from forcefieldx_b200.ffxio import cell_matrices
from forcefieldx_b200.system import PRECISION_FP64, PRECISION_MIXED, water_box, water_params
from oracle import binding as ob
from tests.common import CRYSTALS, golden_system

pytestmark = pytest.mark.gpu


def _rows_set(rows):
    return {tuple(int(v) for v in r) for r in rows}


def _parity(s, p, ref):
    with ForceFieldEnergy(s, p) as ffe:
        for _ in range(2):                     # direct launches, then the captured graph
            e, g = ffe.energy_and_gradient(s.xyz)
            terms, counts = ffe.terms.copy(), ffe.counts.copy()
            if p.precision == PRECISION_FP64:
                rel = np.abs(terms - ref["terms"]) / np.maximum(np.abs(ref["terms"]), 1.0)
                assert rel.max() < 1e-8, (terms, ref["terms"])
                assert float(np.sqrt(np.mean((g - ref["grad"]) ** 2))) < 1e-6
                assert counts[2] == ref["counts"][2]
            else:
                assert np.abs(terms - ref["terms"]).max() < 1e-5 * np.abs(ref["terms"]).max(), (terms, ref["terms"])
                assert float(np.sqrt(np.mean((g - ref["grad"]) ** 2))) < 1e-3
            assert counts[0] == ref["counts"][0] and counts[1] == ref["counts"][1]
        rows = ffe.neighbor_images()
    return terms, rows


@pytest.mark.parametrize("name", CRYSTALS)
def test_crystal_fp64_against_oracle_and_golden(name, fixtures):
    s, p = golden_system(name, fixtures)
    ref = ob.energy(s, p)
    assert ref["status"] == 0
    terms, rows = _parity(s, p, ref)
    got = _rows_set(rows)
    assert len(got) == len(rows) and got == _rows_set(ob.neighbor_images(s, p))
    g, m = fixtures[name]["golden"], s.n_symm
    assert abs(terms[0] / m - g["vdw"]) < 1e-8 * max(1.0, abs(g["vdw"]))
    assert abs(terms[1] / m - g["permanent"]) < g["tolerance"]
    assert abs(terms[2] / m - g["polarization"]) < g["tolerance"]


@pytest.mark.parametrize("name", ["paracetamol", "ethylparaben"])
def test_crystal_mixed_against_oracle(name, fixtures):
    s, p = golden_system(name, fixtures, precision=PRECISION_MIXED)
    _parity(s, p, ob.energy(s, p))


def _triclinic_water(seed):
    """512 waters of a 24.8 A cube recast on the lattice a, b, c + a/3 + b/4 (same fractional
    coordinates): a general triclinic cell whose widths exceed twice the 9 A cutoff."""
    edge = 24.8
    s = water_box(8, edge, seed=seed)
    a, b, c = np.eye(3) * edge
    c2 = c + a / 3 + b / 4
    lens = [float(np.linalg.norm(v)) for v in (a, b, c2)]
    ang = lambda u, v: math.degrees(math.acos(float(u @ v) / (np.linalg.norm(u) * np.linalg.norm(v))))  # noqa
    angles = (ang(b, c2), ang(a, c2), ang(a, b))
    ai, _ = cell_matrices(lens, angles)
    s.xyz = (s.xyz @ np.linalg.inv(np.array([a, b, c2]))) @ ai
    return s, lens, angles


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_MIXED])
def test_triclinic_water_minimum_image(precision):
    s, lens, angles = _triclinic_water(77)
    p = water_params(lens[0], vdw_cutoff=9.0, ewald_cutoff=7.0, pme_grid=(24, 24, 30), precision=precision)
    p = type(p)(**{**p.__dict__, "box": tuple(lens), "angles": angles})
    ref = ob.energy(s, p)
    assert ref["status"] == 0
    _parity(s, p, ref)
    with ForceFieldEnergy(s, p) as ffe:
        ffe.energy(s.xyz)
        pairs = ffe.neighbor_pairs()
    want = ob.neighbor_pairs(s, p)
    n = s.n_atoms
    a = np.unique(pairs[:, 0].astype(np.int64) * n + pairs[:, 1])
    b = np.unique(want[:, 0].astype(np.int64) * n + want[:, 1])
    assert a.size == pairs.shape[0] and np.array_equal(a, b)


def test_set_box_to_a_monoclinic_cell():
    s = water_box(8, 24.8, seed=79)
    p0 = water_params(24.8, vdw_cutoff=9.0, ewald_cutoff=7.0, pme_grid=(24, 24, 24))
    box, angles = (24.8, 24.8, 25.3), (90.0, 101.0, 90.0)
    ai, _ = cell_matrices(box, angles)
    x = (s.xyz / 24.8) @ ai
    p = type(p0)(**{**p0.__dict__, "box": box, "angles": angles})
    ref = ob.energy(s, p, xyz=x)
    with ForceFieldEnergy(s, p0) as ffe:
        ffe.energy_and_gradient(s.xyz)
        ffe.set_crystal(box, angles=angles)
        e, g = ffe.energy_and_gradient(x)
        terms = ffe.terms.copy()
    rel = np.abs(terms - ref["terms"]) / np.maximum(np.abs(ref["terms"]), 1.0)
    assert rel.max() < 1e-8, (terms, ref["terms"])
    assert float(np.sqrt(np.mean((g - ref["grad"]) ** 2))) < 1e-6
