"""Multi-image lists of the oracle (boxes at most twice an interaction cutoff).

The reference handles such boxes with a replicate supercell (C/ReplicatesCrystal.java:
172-202): the energy of the unit cell is that of the supercell of its copies divided by
the number of copies.  The oracle instead sums every lattice image inside the cutoffs.
Pins:

1. a 96-atom water box (9.86 A edge, 9 A vdW, 7 A real space, PME 10^3) against the
   minimum-image oracle on its 2x2x2 replicate supercell (19.7 A, PME 20^3): every energy
   term x 8 and the gradient of every copy.  Even grids keep the supercell's PME grid a
   refinement-free copy of the small one (the grid origin sits half a box from the
   coordinate origin, so an odd K would shift the supercell's points by half a spacing);
2. the 648-atom box, where the minimum image suffices, with multi-image lists forced;
3. the image-pair set of the list builder against a numpy enumeration of all images.
"""
import itertools

import numpy as np
import pytest

from forcefieldx_b200.system import PRECISION_FP64, WATER_648, replicate, small_water_box, water_box, \
    water_params
from oracle import binding as ob


@pytest.mark.parametrize("n_atoms,seed", [(96, 3), (150, 7)])
def test_small_box_equals_replicate_supercell(n_atoms, seed):
    s, edge = small_water_box(n_atoms, seed=seed)
    p = water_params(edge, pme_grid=(10, 10, 10), precision=PRECISION_FP64)
    big = replicate(s, edge)
    P = water_params(2 * edge, pme_grid=(20, 20, 20), precision=PRECISION_FP64)
    r = ob.energy(s, p)
    R = ob.energy(big, P)
    assert r["status"] == 0 and R["status"] == 0
    rel = np.abs(R["terms"] / 8 - r["terms"]) / np.maximum(np.abs(r["terms"]), 1e-9)
    assert rel.max() < 1e-10, rel
    gmax = np.abs(r["grad"]).max()
    for m in range(8):
        gm = R["grad"][m * n_atoms:(m + 1) * n_atoms]
        assert np.abs(gm - r["grad"]).max() < 1e-9 * gmax
    # Interactions inside the cutoffs: the same image pairs, eight copies of each.
    assert R["counts"][0] == 8 * r["counts"][0] and R["counts"][1] == 8 * r["counts"][1]


def test_forced_images_match_minimum_image():
    s = water_box(WATER_648["n_side"], WATER_648["edge"], seed=5)
    p = water_params(WATER_648["edge"], pme_grid=WATER_648["grid"], precision=PRECISION_FP64)
    a = ob.energy(s, p)
    b = ob.energy(s, p, all_images=True)
    rel = np.abs(a["terms"] - b["terms"]) / np.maximum(np.abs(a["terms"]), 1e-9)
    assert rel.max() < 1e-11, rel
    assert np.abs(a["grad"] - b["grad"]).max() < 1e-9
    assert list(a["counts"][:3]) == list(b["counts"][:3])


def _reduced(s):
    xyz = s.xyz.copy()
    for i in range(s.n_atoms):
        r, f = s.red_parent[i], s.red_factor[i]
        if r != i or f != 0.0:
            xyz[i] = f * (s.xyz[i] - s.xyz[r]) + s.xyz[r]
    return xyz


def test_image_pairs_match_enumeration():
    s, edge = small_water_box(96, seed=11)
    p = water_params(edge, pme_grid=(10, 10, 10), precision=PRECISION_FP64)
    rows = ob.neighbor_images(s, p)
    got = {tuple(int(v) for v in r) for r in rows}
    assert len(got) == len(rows)
    rl = max(p.vdw_cutoff, p.ewald_cutoff) + p.list_buffer
    x = _reduced(s)
    want = set()
    shifts = np.array(list(itertools.product(range(-3, 4), repeat=3)))[:, ::-1]   # (nx, ny, nz)
    for i in range(s.n_atoms):
        for k in range(i, s.n_atoms):
            d = x[k] - x[i] + shifts * edge
            d2 = (d * d).sum(1)
            for (nx, ny, nz), ok, dd in zip(shifts, d2 <= rl * rl, d2):
                if not ok or abs(dd - rl * rl) < 1e-9:
                    continue
                if k == i and not (nz > 0 or (nz == 0 and (ny > 0 or (ny == 0 and nx > 0)))):
                    continue
                want.add((i, k, int(nx), int(ny), int(nz)))
    boundary = {r for r in got - want}
    assert not (want - got), sorted(want - got)[:5]
    for (i, k, nx, ny, nz) in boundary:      # only pairs within rounding of the list radius
        d = x[k] - x[i] + np.array([nx, ny, nz]) * edge
        assert abs(float(d @ d) - rl * rl) < 1e-9
