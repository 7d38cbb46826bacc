"""The oracle's vdW softcore lambda path against central finite differences.

The reference tests its lambda derivatives the same way (finite differences of the
energy in lambda and of dU/dL in the coordinates).  System: 216 waters with a 30-atom
(10-water) soft subset, lambda in {0.1, 0.5, 0.9}.
"""
import numpy as np
import pytest

from forcefieldx_b200.system import PRECISION_FP64, Alchemy, water_box, water_params
from oracle import binding as ob


def _setup():
    s = water_box(6, 18.643, seed=11)
    p = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 20), polarization=0,
                     precision=PRECISION_FP64)
    soft = np.zeros(s.n_atoms, dtype=np.int32)
    soft[:30] = 1
    return s, p, Alchemy(soft=soft, molecule=np.arange(s.n_atoms) // 3)


@pytest.mark.parametrize("lam", [0.1, 0.5, 0.9])
def test_dEdL_matches_finite_difference(lam):
    s, p, a = _setup()
    h = 1.0e-5
    r0 = ob.energy(s, p, alchemy=a, lam=lam)
    ep = ob.energy(s, p, alchemy=a, lam=lam + h, gradient=False)
    em = ob.energy(s, p, alchemy=a, lam=lam - h, gradient=False)
    fd = (ep["terms"][9] - em["terms"][9]) / (2 * h)
    assert abs(fd - r0["dEdL"]) < 1e-6 * max(1.0, abs(fd)), (fd, r0["dEdL"])
    fd2 = (ep["dEdL"] - em["dEdL"]) / (2 * h)
    assert abs(fd2 - r0["d2EdL2"]) < 1e-5 * max(1.0, abs(fd2)), (fd2, r0["d2EdL2"])


def test_dEdXdL_matches_finite_difference():
    s, p, a = _setup()
    lam, h = 0.5, 1.0e-5
    r0 = ob.energy(s, p, alchemy=a, lam=lam)
    assert np.abs(r0["dEdXdL"]).max() > 0.0
    for atom in (0, 4, 40):          # soft O, soft H, a hard atom near the soft waters
        for d in range(3):
            x = s.xyz.copy()
            x[atom, d] += h
            dp = ob.energy(s, p, xyz=x, alchemy=a, lam=lam, gradient=False)["dEdL"]
            x[atom, d] -= 2 * h
            dm = ob.energy(s, p, xyz=x, alchemy=a, lam=lam, gradient=False)["dEdL"]
            fd = (dp - dm) / (2 * h)
            assert abs(fd - r0["dEdXdL"][atom, d]) < 1e-5 * max(1.0, abs(fd)), (atom, d, fd, r0["dEdXdL"][atom, d])


def test_lambda_one_is_the_plain_energy():
    s, p, a = _setup()
    plain = ob.energy(s, p)
    soft = ob.energy(s, p, alchemy=a, lam=1.0)
    assert abs(plain["terms"][0] - soft["terms"][0]) < 1e-10 * abs(plain["terms"][0])
    assert np.abs(plain["grad"] - soft["grad"]).max() < 1e-10


# ---------------------------------------------------------------------------
# Electrostatic lambda (elec-lambdaterm, OST: condensed, condensed without the soft atoms,
# soft atoms in vacuum; ParticleMeshEwald.java:897-935, 1609-1796).

def _setup_elec(polarization=2):
    s = water_box(6, 18.643, seed=11)
    p = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 20), polarization=polarization,
                     precision=PRECISION_FP64)
    soft = np.zeros(s.n_atoms, dtype=np.int32)
    soft[:30] = 1
    return s, p, Alchemy(soft=soft, molecule=np.arange(s.n_atoms) // 3, elec=True)


def test_elec_lambda_one_is_the_plain_energy():
    s, p, a = _setup_elec()
    plain = ob.energy(s, p)
    full = ob.energy(s, p, alchemy=a, lam=1.0)
    assert np.abs(plain["terms"] - full["terms"]).max() < 1e-10 * np.abs(plain["terms"]).max()
    assert np.abs(plain["grad"] - full["grad"]).max() < 1e-10


# The reference's dU/dL takes the polarization energy's lambda dependence through its scale
# only: inside the polarization window (lambda >= polarization-lambda-start, 0.75) the
# softcore shift also moves the polarization energy of soft pairs, a term its dU/dL omits
# (RealSpaceEnergyRegion.java:2153-2176), so finite differences there are checked with
# polarization off.
@pytest.mark.parametrize("lam,polarization", [(0.1, 2), (0.5, 2), (0.6, 2), (0.8, 0), (0.9, 0)])
def test_elec_dEdL_matches_finite_difference(lam, polarization):
    s, p, a = _setup_elec(polarization)
    h = 1.0e-5
    r0 = ob.energy(s, p, alchemy=a, lam=lam)
    ep = ob.energy(s, p, alchemy=a, lam=lam + h, gradient=False)
    em = ob.energy(s, p, alchemy=a, lam=lam - h, gradient=False)
    fd = (ep["terms"][9] - em["terms"][9]) / (2 * h)
    assert abs(fd - r0["dEdL"]) < 1e-6 * max(1.0, abs(fd)), (fd, r0["dEdL"])
    fd2 = (ep["dEdL"] - em["dEdL"]) / (2 * h)
    assert abs(fd2 - r0["d2EdL2"]) < 1e-5 * max(1.0, abs(fd2)), (fd2, r0["d2EdL2"])


@pytest.mark.parametrize("lam,polarization", [(0.5, 2), (0.9, 0)])
def test_elec_dEdXdL_matches_finite_difference(lam, polarization):
    s, p, a = _setup_elec(polarization)
    h = 1.0e-5
    r0 = ob.energy(s, p, alchemy=a, lam=lam)
    for atom in (0, 4, 40):          # soft O, soft H, a hard atom near the soft waters
        for d in range(3):
            x = s.xyz.copy()
            x[atom, d] += h
            dp = ob.energy(s, p, xyz=x, alchemy=a, lam=lam, gradient=False)["dEdL"]
            x[atom, d] -= 2 * h
            dm = ob.energy(s, p, xyz=x, alchemy=a, lam=lam, gradient=False)["dEdL"]
            fd = (dp - dm) / (2 * h)
            assert abs(fd - r0["dEdXdL"][atom, d]) < 1e-5 * max(1.0, abs(fd)), (atom, d, fd, r0["dEdXdL"][atom, d])


def test_elec_gradient_matches_finite_difference():
    s, p, a = _setup_elec()
    lam, h = 0.6, 1.0e-5
    r0 = ob.energy(s, p, alchemy=a, lam=lam)
    for atom in (1, 5, 40):
        for d in range(3):
            x = s.xyz.copy()
            x[atom, d] += h
            ep = ob.energy(s, p, xyz=x, alchemy=a, lam=lam, gradient=False)["terms"][9]
            x[atom, d] -= 2 * h
            em = ob.energy(s, p, xyz=x, alchemy=a, lam=lam, gradient=False)["terms"][9]
            fd = (ep - em) / (2 * h)
            assert abs(fd - r0["grad"][atom, d]) < 1e-5 * max(1.0, abs(fd)), (atom, d, fd, r0["grad"][atom, d])
