"""Force Field X input formats (forcefieldx_b200/ffxio.py).

1. A water box written as XYZ + key + AMOEBA parameter records and read back resolves
   to the same per-atom system as the generator's own parameters, and evaluates to the
   same oracle energy.
2. The reference's own DHFR inputs (XYZ, key, AMOEBA_BIO_2009), where present, resolve to
   the committed golden system (tests/golden/dhfr_system.npz) exactly.
3. Its SNARE asymmetric unit in P212121, expanded by the four symmetry operators, is the
   reference's own P1 file of the same crystal (1n7s.P1.xyz) up to lattice translations.
"""
import os

import numpy as np
import pytest

from forcefieldx_b200.ffxio import load_system, read_key, read_xyz, write_xyz
from forcefieldx_b200.system import (WATER_H_MPOLE_BOHR, WATER_O_MPOLE_BOHR, WATER_POLAR, WATER_THOLE, WATER_VDW,
                                     AmoebaSystem, water_box, water_params)
from oracle import binding as ob

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# The reference checkout, when present (tests that read its files skip otherwise).
REFERENCE = os.environ.get("FFX_REFERENCE_ROOT", "")


def _mpole_records(t, frame_types, m):
    q, d, Q = m
    return [f"multipole {t} {' '.join(str(f) for f in frame_types)} {q}",
            f"    {d[0]} {d[1]} {d[2]}",
            f"    {Q[0][0]}",
            f"    {Q[1][0]} {Q[1][1]}",
            f"    {Q[2][0]} {Q[2][1]} {Q[2][2]}"]


def _water_prm():
    lines = ['atom 1 1 O "AMOEBA Water O" 8 15.999 2',
             'atom 2 2 H "AMOEBA Water H" 1 1.008 1',
             f"vdw 1 {WATER_VDW[0][0]} {WATER_VDW[0][1]}",
             f"vdw 2 {WATER_VDW[1][0]} {WATER_VDW[1][1]} {WATER_VDW[1][2]}"]
    lines += _mpole_records(1, (-2, -2), WATER_O_MPOLE_BOHR)
    lines += _mpole_records(2, (1, 2), WATER_H_MPOLE_BOHR)
    lines += [f"polarize 1 {WATER_POLAR[0]} {WATER_THOLE} 2", f"polarize 2 {WATER_POLAR[1]} {WATER_THOLE} 1"]
    return "\n".join(lines) + "\n"


def test_water_files_round_trip(tmp_path):
    s = water_box(3, 9.3215, seed=4)
    n = s.n_atoms
    types = np.where(np.arange(n) % 3 == 0, 1, 2)
    bonds = [(3 * w, 3 * w + 1) for w in range(n // 3)] + [(3 * w, 3 * w + 2) for w in range(n // 3)]
    write_xyz(tmp_path / "w.xyz", s.xyz, types, bonds, names=["O" if t == 1 else "H" for t in types], title="water")
    (tmp_path / "w.prm").write_text(_water_prm())
    (tmp_path / "w.key").write_text("parameters w.prm\na-axis 18.643\nvdw-cutoff 9.0\newald-cutoff 7.0\n"
                                    "ewald-alpha 0.545\npme-grid 20 20 20\npolar-eps 1e-6\n")
    xyz, t2, b2 = read_xyz(tmp_path / "w.xyz")
    assert np.allclose(xyz, s.xyz, atol=5e-7) and list(t2) == list(types)
    assert read_key(tmp_path / "w.key")["pme-grid"] == ["20", "20", "20"]
    got, p = load_system(tmp_path / "w.xyz", tmp_path / "w.key")
    assert p.box == [18.643, 18.643, 18.643] and list(p.pme_grid) == [20, 20, 20]
    for f in ("multipole", "frame", "axis", "polarizability", "thole", "pdamp", "vdw_type", "red_parent",
              "red_factor", "vdw_inv_rmin", "vdw_eps"):
        assert np.array_equal(np.asarray(getattr(got, f)), np.asarray(getattr(s, f))), f
    for f in ("n12", "n13", "n14", "n15", "ip11"):
        assert [list(v) for v in getattr(got, f)] == [list(v) for v in getattr(s, f)], f
    # Same energy from the file-built system (coordinates rounded to the XYZ format's 6 decimals).
    s_file = AmoebaSystem(**{**s.__dict__, "xyz": xyz})
    params = water_params(18.643, pme_grid=(20, 20, 20))
    e1 = ob.energy(got, params)["terms"]
    e2 = ob.energy(s_file, params)["terms"]
    assert np.array_equal(e1, e2)


@pytest.mark.skipif(not os.path.isdir(REFERENCE), reason="reference source tree not present")
def test_dhfr_reference_inputs_resolve_to_golden_system():
    res = os.path.join(REFERENCE, "modules/potential/src/test/resources")
    prm = os.path.join(REFERENCE, "modules/potential/src/main/java/ffx/potential/parameters/ff/AMOEBA_BIO_2009")
    got, p = load_system(os.path.join(res, "dhfr.xyz"), os.path.join(res, "dhfr.key"), prm_path=prm)
    want = AmoebaSystem.load_npz(os.path.join(GOLDEN, "dhfr_system.npz"))
    for f in ("xyz", "multipole", "frame", "axis", "polarizability", "thole", "pdamp", "vdw_type", "red_parent",
              "red_factor", "vdw_inv_rmin", "vdw_eps"):
        assert np.array_equal(np.asarray(getattr(got, f)), np.asarray(getattr(want, f))), f
    assert [list(v) for v in got.ip11] == [list(v) for v in want.ip11]
    assert p.ewald_cutoff == 6.7 and p.ewald_alpha == 0.57


@pytest.mark.skipif(not os.path.isdir(REFERENCE), reason="reference source tree not present")
def test_p212121_expansion_is_the_reference_p1_cell():
    """The P212121 asymmetric unit expanded by the four symmetry operators gives the atoms
    of the reference's own P1 file (1n7s.P1.xyz), mate after mate, up to lattice
    translations of whole atoms."""
    from forcefieldx_b200.ffxio import expand_coordinates, read_key
    res = os.path.join(REFERENCE, "modules/potential/src/test/resources")
    xyz, types, _ = read_xyz(os.path.join(res, "1n7s.P212121.xyz"))
    key = read_key(os.path.join(res, "1n7s.P212121.key"))
    box = np.array([float(key["a-axis"][0]), float(key["b-axis"][0]), float(key["c-axis"][0])])
    cell = expand_coordinates(xyz, box, "P212121")
    ref, rtypes, _ = read_xyz(os.path.join(res, "1n7s.P1.xyz"))
    d = (cell - ref) / box
    assert np.abs(d - np.round(d)).max() < 1e-6
    assert list(rtypes) == list(types) * 4
