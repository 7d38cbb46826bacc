"""General (monoclinic, triclinic) cells in the oracle, pinned independently of the reference's
crystal goldens: one lattice described by two bases gives the same lattice sums.

A 216-water cube (edge L) is also the lattice spanned by a = (L, 0, 0), b = (0, L, 0) and
c' = (L, 0, L): a monoclinic cell with c' = sqrt(2) L and beta = 45 degrees.  With lists of
every lattice image inside the cutoffs, the vdW and real-space sums are exact lattice sums,
so they agree to rounding between the two descriptions; the reciprocal terms differ only by
the PME discretisation of the two meshes.  A general triclinic basis of the same lattice
(c'' = c + a + b) exercises the general branch of Crystal.updateCrystal the same way.
"""
import math

import numpy as np
import pytest

from forcefieldx_b200.ffxio import cell_matrices, expand_coordinates
from forcefieldx_b200.system import water_box, water_params
from oracle import binding as ob

EDGE = 18.643


def _cell_of_vectors(a, b, c):
    """(edges, angles in degrees) of the cell spanned by the lattice vectors a, b, c."""
    la, lb, lc = (float(np.linalg.norm(v)) for v in (a, b, c))
    ang = lambda u, v: math.degrees(math.acos(float(np.dot(u, v)) / (np.linalg.norm(u) * np.linalg.norm(v))))  # noqa
    return (la, lb, lc), (ang(b, c), ang(a, c), ang(a, b))


@pytest.mark.parametrize("basis", ["monoclinic", "triclinic"])
def test_same_lattice_two_bases(basis):
    s = water_box(6, EDGE, seed=71)
    a, b, c = np.array([EDGE, 0, 0]), np.array([0, EDGE, 0]), np.array([0, 0, EDGE])
    c2 = c + a if basis == "monoclinic" else c + a + b
    box2, ang2 = _cell_of_vectors(a, b, c2)
    ai, _ = cell_matrices(box2, ang2)
    # The reference's cell of these edges and angles spans the same lattice (rotated into its
    # a-along-x, b-in-xy frame, which is the identity here since a and b lie on x and y).
    assert np.allclose(ai[2], c2) if basis == "monoclinic" else abs(np.linalg.det(ai) - EDGE ** 3) < 1e-9
    # The coordinates in the reference frame of the second cell (a along x, b in the xy
    # plane): the same fractional coordinates in the new basis.
    x2 = (s.xyz @ np.linalg.inv(np.array([a, b, c2]))) @ ai
    for g1, g2, exact in (((20, 20, 20), (20, 20, 28), True), ((64, 64, 64), (64, 64, 90), False)):
        p1 = water_params(EDGE, vdw_cutoff=9.0, ewald_cutoff=7.0, pme_grid=g1)
        p2 = water_params(EDGE, vdw_cutoff=9.0, ewald_cutoff=7.0, pme_grid=g2)
        p2 = type(p2)(**{**p2.__dict__, "box": box2, "angles": ang2})
        r1 = ob.energy(s, p1, all_images=True)
        r2 = ob.energy(s, p2, xyz=x2, all_images=True)
        assert r1["status"] == 0 and r2["status"] == 0
        if exact:   # lattice sums: vdW, permanent real space, self; interaction counts
            for t in (0, 3, 4):
                assert abs(r1["terms"][t] - r2["terms"][t]) < 1e-9 * abs(r1["terms"][t]), t
            assert r1["counts"][0] == r2["counts"][0] and r1["counts"][1] == r2["counts"][1]
        else:       # the meshes converge to one Ewald sum
            assert abs(r1["terms"][9] - r2["terms"][9]) < 5e-5 * abs(r1["terms"][9])
            if basis == "monoclinic":   # a and b on x and y in both frames: gradients comparable
                assert float(np.sqrt(np.mean((r1["grad"] - r2["grad"]) ** 2))) < 5e-3


def test_right_angles_are_the_orthorhombic_cell():
    s = water_box(6, EDGE, seed=73)
    p = water_params(EDGE, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 20))
    q = type(p)(**{**p.__dict__, "angles": (0.0, 0.0, 0.0)})     # 0 reads as 90
    r, t = ob.energy(s, p), ob.energy(s, q)
    # (the oracle's threaded mesh sums add in thread order: equal to rounding)
    assert np.max(np.abs(r["terms"] - t["terms"]) / np.maximum(np.abs(r["terms"]), 1.0)) < 1e-12
    assert np.max(np.abs(r["grad"] - t["grad"])) < 1e-10


def test_space_group_expansion_in_a_monoclinic_cell():
    """P21/c mates of a point: fractional x' = R x + t in the monoclinic cell's coordinates."""
    box, ang = (10.0, 12.0, 14.0), (90.0, 110.0, 90.0)
    ai, a = cell_matrices(box, ang)
    f = np.array([[0.1, 0.2, 0.3]])
    x = f @ ai
    mates = expand_coordinates(x, box, "P21/C", ang) @ a
    want = np.array([[0.1, 0.2, 0.3], [-0.1, -0.2, -0.3], [-0.1, 0.7, 0.2], [0.1, 0.3, 0.8]])
    assert np.allclose(mates, want, atol=1e-12)


def test_triclinic_minimum_image_equals_every_image():
    """A triclinic cell wider than twice the cutoffs: the cell-list minimum-image path (fractional
    cells, Crystal.image's general round trip) gives the sums of the every-image lists."""
    edge = 24.8
    s = water_box(8, edge, seed=77)
    a, b, c = np.eye(3) * edge
    c2 = c + a / 3 + b / 4
    box2, ang2 = _cell_of_vectors(a, b, c2)
    ai, _ = cell_matrices(box2, ang2)
    x2 = (s.xyz @ np.linalg.inv(np.array([a, b, c2]))) @ ai
    p = water_params(edge, vdw_cutoff=9.0, ewald_cutoff=7.0, pme_grid=(24, 24, 30))
    p = type(p)(**{**p.__dict__, "box": box2, "angles": ang2})
    r1, r2 = ob.energy(s, p, xyz=x2), ob.energy(s, p, xyz=x2, all_images=True)
    assert r1["status"] == 0 and r2["status"] == 0
    assert np.max(np.abs(r1["terms"] - r2["terms"]) / np.maximum(np.abs(r1["terms"]), 1.0)) < 1e-11
    assert np.max(np.abs(r1["grad"] - r2["grad"])) < 1e-9
    assert np.array_equal(r1["counts"][:3], r2["counts"][:3])
