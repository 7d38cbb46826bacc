"""Differentiation on the 24,000-atom water box (the config of the reference's
testLambdaGradient and GradientUtils checks, at this box's scale).

* Electrostatic (OST) plus vdW softcore lambda on a seeded 30-atom soft subset at lambda
  in {0.1, 0.5, 0.9}: energy terms, dU/dL, d2U/dL2, dU/dX dL and the gradient against the
  oracle, FP64 at 1e-8 relative (1e-6 RMS for gradient-like outputs) and the mixed form at
  1e-5 relative (1e-3 RMS).  Reference: commands/EnergyTest.java testLambdaGradient;
  ParticleMeshEwald.java:897-935; VanDerWaals.java:1723-1880.
* Central finite differences (h = 1e-5 A) of the FP64 energy at 64 seeded random
  coordinates against the FP64 analytic gradient (GradientUtils.testGradient,
  utils/GradientUtils.java:78-206), and the mixed form's analytic gradient against the
  same differences.  A mixed-form difference at this step would drown in FP32 noise.
"""
import numpy as np
import pytest

from forcefieldx_b200.energy import ForceFieldEnergy
from forcefieldx_b200.system import PRECISION_FP64, PRECISION_MIXED, WATER_24K, Alchemy, water_box, water_params
from oracle import binding as ob

pytestmark = pytest.mark.gpu

LAMBDAS = [0.1, 0.5, 0.9]


def _box():
    return water_box(WATER_24K["n_side"], WATER_24K["edge"])


def _alchemy(n, seed=404):
    rng = np.random.default_rng(seed)
    soft = np.zeros(n, dtype=np.int32)
    for w in rng.choice(n // 3, 10, replace=False):   # ten whole waters: 30 soft atoms
        soft[3 * w:3 * w + 3] = 1
    return Alchemy(soft=soft, molecule=np.arange(n) // 3, elec=True)


@pytest.fixture(scope="module")
def oracle_lambda():
    s = _box()
    a = _alchemy(s.n_atoms)
    p = water_params(WATER_24K["edge"], pme_grid=WATER_24K["grid"], precision=PRECISION_FP64)
    return {lam: ob.energy(s, p, alchemy=a, lam=lam) for lam in LAMBDAS}


@pytest.mark.parametrize("precision,rel,rms_tol", [(PRECISION_FP64, 1e-8, 1e-6), (PRECISION_MIXED, 1e-5, 1e-3)])
def test_elec_and_vdw_lambda_water_24k(oracle_lambda, precision, rel, rms_tol):
    s = _box()
    a = _alchemy(s.n_atoms)
    p = water_params(WATER_24K["edge"], pme_grid=WATER_24K["grid"], precision=precision)
    with ForceFieldEnergy(s, p) as ffe:
        ffe.set_alchemy(a)
        for lam in LAMBDAS:
            ffe.set_lambda(lam)
            ref = oracle_lambda[lam]
            assert ref["status"] == 0
            e, g = ffe.energy_and_gradient(s.xyz)
            d1, d2, lg = ffe.get_dEdL()
            scale = max(abs(ref["terms"][9]), 1.0)
            terr = np.abs(ffe.terms - ref["terms"])
            report = f"lambda {lam}: term errors {terr}, dEdL {d1} vs {ref['dEdL']}, d2EdL2 {d2} vs {ref['d2EdL2']}"
            if precision == PRECISION_FP64:
                assert np.all(terr < rel * np.maximum(np.abs(ref["terms"]), 1.0)), report
            else:
                assert terr.max() < rel * scale, report
            assert abs(d1 - ref["dEdL"]) < rel * max(1.0, abs(ref["dEdL"]), 0 if precision == PRECISION_FP64 else scale), report
            assert abs(d2 - ref["d2EdL2"]) < 10 * rel * max(1.0, abs(ref["d2EdL2"]),
                                                             0 if precision == PRECISION_FP64 else scale), report
            assert float(np.sqrt(np.mean((g - ref["grad"]) ** 2))) < rms_tol, report
            assert float(np.sqrt(np.mean((lg - ref["dEdXdL"]) ** 2))) < rms_tol, report


def test_finite_difference_gradient_water_24k():
    s = _box()
    rng = np.random.default_rng(64)
    coords = [(int(a), int(d)) for a, d in zip(rng.choice(s.n_atoms, 64, replace=False), rng.integers(0, 3, 64))]
    h = 1.0e-5
    p64 = water_params(WATER_24K["edge"], pme_grid=WATER_24K["grid"], precision=PRECISION_FP64, polar_eps=1e-8)
    fd = np.zeros(len(coords))
    with ForceFieldEnergy(s, p64) as ffe:
        _, g64 = ffe.energy_and_gradient(s.xyz)
        for q, (atom, d) in enumerate(coords):
            x = s.xyz.copy()
            x[atom, d] += h
            ep = ffe.energy(x)
            x[atom, d] -= 2 * h
            em = ffe.energy(x)
            fd[q] = (ep - em) / (2 * h)
    pm = water_params(WATER_24K["edge"], pme_grid=WATER_24K["grid"], precision=PRECISION_MIXED, polar_eps=1e-8)
    with ForceFieldEnergy(s, pm) as ffe:
        _, gm = ffe.energy_and_gradient(s.xyz)
    an64 = np.array([g64[a, d] for a, d in coords])
    anm = np.array([gm[a, d] for a, d in coords])
    err64, errm = np.abs(an64 - fd), np.abs(anm - fd)
    print(f"FD (h=1e-5) vs analytic, 64 coordinates: FP64 max {err64.max():.3e} RMS "
          f"{np.sqrt(np.mean(err64 ** 2)):.3e}; mixed max {errm.max():.3e} RMS {np.sqrt(np.mean(errm ** 2)):.3e}")
    assert err64.max() < 1e-4
    assert errm.max() < 1e-3
