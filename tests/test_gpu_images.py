"""Multi-image lists of the CUDA library (boxes at most twice an interaction cutoff)
against the oracle, whose multi-image sum is pinned to the replicate supercell
(tests/test_oracle_images.py).

Bar as for the minimum-image parity tests: bit-identical image-pair set of the list,
1e-8 relative per energy term and 1e-6 gradient RMS in the plain FP64 form, identical
interaction and PCG iteration counts; in the mixed form every term within 1e-5 of the
total energy's magnitude and 1e-3 gradient RMS (the bar of the 24k-atom mixed test).
"""
import numpy as np
import pytest

from forcefieldx_b200.energy import ForceFieldEnergy
from forcefieldx_b200.system import PRECISION_FP64, PRECISION_MIXED, WATER_648, replicate, small_water_box, \
    water_box, water_params
from oracle import binding as ob

pytestmark = pytest.mark.gpu


def _rows_set(rows):
    return {tuple(int(v) for v in r) for r in rows}


def _check(s, p, e_rel, g_rms, all_images=False, graph_repeats=2):
    ref = ob.energy(s, p, all_images=all_images)
    assert ref["status"] == 0
    with ForceFieldEnergy(s, p) as ffe:
        if all_images:
            ffe.set_image_mode(True)
        for _ in range(graph_repeats):        # direct launches, then the captured graph
            e, g = ffe.energy_and_gradient(s.xyz)
            terms, counts = ffe.terms.copy(), ffe.counts.copy()
            if p.precision == PRECISION_FP64:
                rel = np.abs(terms - ref["terms"]) / np.maximum(np.abs(ref["terms"]), 1.0)
            else:   # the mixed-form bar: every term within e_rel of the total's magnitude
                rel = np.abs(terms - ref["terms"]) / abs(ref["terms"][9])
            assert rel.max() < e_rel, (terms, ref["terms"], rel)
            rms = float(np.sqrt(np.mean((g - ref["grad"]) ** 2)))
            assert rms < g_rms, rms
            assert counts[0] == ref["counts"][0] and counts[1] == ref["counts"][1]
            if p.precision == PRECISION_FP64:
                assert counts[2] == ref["counts"][2]
        rows = ffe.neighbor_images()
    want = ob.neighbor_images(s, p, all_images=all_images)
    got = _rows_set(rows)
    assert len(got) == len(rows)
    assert got == _rows_set(want)


@pytest.mark.parametrize("n_atoms,grid,seed", [(96, 10, 3), (96, 9, 5), (150, 10, 7), (300, 12, 9)])
def test_small_box_fp64(n_atoms, grid, seed):
    s, edge = small_water_box(n_atoms, seed=seed)
    p = water_params(edge, pme_grid=(grid,) * 3, precision=PRECISION_FP64)
    _check(s, p, 1e-8, 1e-6)


@pytest.mark.parametrize("n_atoms,grid,seed", [(96, 10, 3), (300, 12, 9)])
def test_small_box_mixed(n_atoms, grid, seed):
    s, edge = small_water_box(n_atoms, seed=seed)
    p = water_params(edge, pme_grid=(grid,) * 3, precision=PRECISION_MIXED)
    _check(s, p, 1e-5, 1e-3)


def test_forced_images_water_648():
    s = water_box(WATER_648["n_side"], WATER_648["edge"], seed=5)
    p = water_params(WATER_648["edge"], pme_grid=WATER_648["grid"], precision=PRECISION_FP64)
    _check(s, p, 1e-8, 1e-6, all_images=True)


def test_small_box_equals_supercell_on_gpu():
    """The library's own multi-image energy against its own minimum-image energy of the
    2x2x2 replicate supercell (per copy)."""
    s, edge = small_water_box(96, seed=13)
    p = water_params(edge, pme_grid=(10, 10, 10), precision=PRECISION_FP64)
    big = replicate(s, edge)
    P = water_params(2 * edge, pme_grid=(20, 20, 20), precision=PRECISION_FP64)
    with ForceFieldEnergy(s, p) as a:
        ea, ga = a.energy_and_gradient(s.xyz)
        ta = a.terms.copy()
    with ForceFieldEnergy(big, P) as b:
        eb, gb = b.energy_and_gradient(big.xyz)
        tb = b.terms.copy()
    rel = np.abs(tb / 8 - ta) / np.maximum(np.abs(ta), 1.0)
    assert rel.max() < 1e-9, rel
    assert np.abs(gb[:96] - ga).max() < 1e-8 * np.abs(ga).max()
