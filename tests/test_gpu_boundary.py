"""The drop-in boundary's state changes: a new cell (ForceFieldEnergy.setCrystal, behind
OpenMMEnergy.setCrystal, OpenMMEnergy.java:585) and new parameter values
(OpenMMEnergy.updateParameters, :623), each checked against a freshly created handle and
the oracle at the parity bar (1e-8 relative per term, 1e-6 gradient RMS).
"""
import dataclasses

import numpy as np
import pytest

from forcefieldx_b200.energy import ForceFieldEnergy
from forcefieldx_b200.system import PRECISION_FP64, PRECISION_MIXED, WATER_24K, Alchemy, water_box, water_params
from oracle import binding as ob

pytestmark = pytest.mark.gpu

E_REL = 1.0e-8
G_RMS = 1.0e-6


def _against(ffe, s, p, x, check_oracle=True, fresh_rel=1e-11):
    e, g = ffe.energy_and_gradient(x)
    terms = ffe.terms.copy()
    with ForceFieldEnergy(s, p) as fresh:
        ef, gf = fresh.energy_and_gradient(x)
        tf = fresh.terms.copy()
    assert np.max(np.abs(terms - tf) / np.maximum(np.abs(tf), 1.0)) < fresh_rel, (terms, tf)
    g_tol = 1e-6 if p.precision == PRECISION_MIXED else 1e-9
    assert np.max(np.abs(g - gf)) < g_tol
    if check_oracle:
        ref = ob.energy(s, p, xyz=x)
        assert ref["status"] == 0
        rel = np.abs(terms - ref["terms"]) / np.maximum(np.abs(ref["terms"]), 1.0)
        # Mixed form: every term within 1e-5 of the largest term's magnitude (the perturbed
        # systems' totals cancel to a small fraction of their terms).
        bar = E_REL if p.precision == PRECISION_FP64 else 1e-5 * np.abs(ref["terms"]).max()
        if p.precision == PRECISION_FP64:
            assert rel.max() < bar, (terms, ref["terms"])
            assert float(np.sqrt(np.mean((g - ref["grad"]) ** 2))) < G_RMS
        else:
            assert np.abs(terms - ref["terms"]).max() < bar
            assert float(np.sqrt(np.mean((g - ref["grad"]) ** 2))) < 1e-3


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_MIXED])
def test_set_box_keeps_or_changes_the_mesh(precision):
    s = water_box(6, 18.643, seed=51)
    p0 = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 20), precision=precision)
    with ForceFieldEnergy(s, p0) as ffe:
        ffe.energy_and_gradient(s.xyz)
        ffe.energy_and_gradient(s.xyz)                    # a captured graph now exists
        for edge, grid in ((18.9, None), (19.2, (24, 24, 24)), (18.5, (20, 20, 20))):
            ffe.set_crystal(edge, grid)
            p = water_params(edge, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=grid or (20, 20, 20),
                             precision=precision)
            x = s.xyz * (edge / 18.643)
            _against(ffe, s, p, x)
            assert ffe.count("list_builds") == 1         # a new cell rebuilds the list


def test_set_box_into_multi_image_lists():
    """18.643 A with 9 A vdW: one image per pair; 17.5 A: some pairs interact through two."""
    s = water_box(6, 18.643, seed=53)
    p0 = water_params(18.643, pme_grid=(20, 20, 20))
    with ForceFieldEnergy(s, p0) as ffe:
        ffe.energy_and_gradient(s.xyz)
        ffe.set_crystal(17.5)
        x = s.xyz * (17.5 / 18.643)
        _against(ffe, s, water_params(17.5, pme_grid=(20, 20, 20)), x)
        ffe.set_crystal(18.643)
        _against(ffe, s, p0, s.xyz)


def test_set_box_water_24k_barostat_step():
    s = water_box(WATER_24K["n_side"], WATER_24K["edge"])
    p0 = water_params(WATER_24K["edge"], pme_grid=WATER_24K["grid"])
    with ForceFieldEnergy(s, p0) as ffe:
        ffe.energy_and_gradient(s.xyz)
        ffe.energy_and_gradient(s.xyz)
        edge = 62.31
        ffe.set_crystal(edge)
        x = s.xyz * (edge / WATER_24K["edge"])
        _against(ffe, s, water_params(edge, pme_grid=WATER_24K["grid"]), x)


def _perturbed(s, seed):
    rng = np.random.default_rng(seed)
    mp = s.multipole * (1.0 + 0.1 * rng.uniform(-1, 1, s.multipole.shape))
    mp[:, 0] = s.multipole[:, 0] * 1.05                  # charges scaled: the cell stays neutral
    pol = s.polarizability * 0.9
    thole = s.thole * 1.05
    pdamp = np.where(thole == 0.0, 0.0, pol ** (1.0 / 6.0))
    eps = s.vdw_eps * 1.2
    inv = s.vdw_inv_rmin * 0.98
    red = np.where(s.red_factor > 0, s.red_factor * 0.95, 0.0)
    return dataclasses.replace(s, multipole=mp, polarizability=pol, thole=thole, pdamp=pdamp, vdw_eps=eps,
                               vdw_inv_rmin=inv, red_factor=red)


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_MIXED])
def test_update_parameters(precision):
    s = water_box(6, 18.643, seed=57)
    p = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 20), precision=precision)
    with ForceFieldEnergy(s, p) as ffe:
        ffe.energy_and_gradient(s.xyz)
        ffe.energy_and_gradient(s.xyz)
        t = _perturbed(s, 3)
        ffe.update_parameters(t)
        _against(ffe, t, p, s.xyz)
        ffe.update_parameters(s)                          # and back
        _against(ffe, s, p, s.xyz, check_oracle=False)


def test_update_parameters_under_electrostatic_lambda():
    s = water_box(6, 18.643, seed=59)
    p = water_params(18.643, pme_grid=(20, 20, 20))
    soft = np.zeros(s.n_atoms, dtype=np.int32)
    soft[:30] = 1
    a = Alchemy(soft=soft, molecule=np.arange(s.n_atoms) // 3, elec=True)
    t = _perturbed(s, 5)
    with ForceFieldEnergy(s, p) as ffe:
        ffe.set_alchemy(a)
        ffe.set_lambda(0.8)
        ffe.energy_and_gradient(s.xyz)
        ffe.update_parameters(t)
        e, g = ffe.energy_and_gradient(s.xyz)
        d1, d2, lg = ffe.get_dEdL()
    ref = ob.energy(t, p, alchemy=a, lam=0.8)
    assert np.all(np.abs(ffe.terms - ref["terms"]) < E_REL * np.maximum(np.abs(ref["terms"]), 1.0))
    assert abs(d1 - ref["dEdL"]) < E_REL * max(1.0, abs(ref["dEdL"]))
    assert float(np.sqrt(np.mean((g - ref["grad"]) ** 2))) < G_RMS
    assert float(np.sqrt(np.mean((lg - ref["dEdXdL"]) ** 2))) < G_RMS


def test_bad_boundary_arguments():
    from forcefieldx_b200.energy import EnergyException
    s = water_box(4, 12.4, seed=2)
    with ForceFieldEnergy(s, water_params(12.4, pme_grid=(16, 16, 16))) as ffe:
        with pytest.raises(EnergyException) as ei:
            ffe.set_crystal(-1.0)
        assert ei.value.status == 1
        with pytest.raises(EnergyException) as ei:
            ffe.set_crystal(12.4, (4, 16, 16))           # a mesh shorter than the B-spline order
        assert ei.value.status == 1
        w = water_box(5, 15.5, seed=2)
        with pytest.raises(EnergyException) as ei:
            ffe.update_parameters(w)                       # other atom count
        assert ei.value.status == 1
