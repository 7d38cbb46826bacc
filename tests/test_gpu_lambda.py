"""vdW softcore lambda path of the CUDA library against the oracle.

A 30-atom (10-water) soft subset at lambda in {0.1, 0.5, 0.9}: energies, dU/dL, d2U/dL2
and dU/dX dL.  Plain FP64 form to 1e-8 relative (gradient-like outputs to 1e-6 RMS), the
mixed form to 1e-5 relative / 1e-3 RMS.  The oracle's lambda path is itself pinned by
finite differences (tests/test_oracle_lambda.py).
"""
import numpy as np
import pytest

from forcefieldx_b200.energy import ForceFieldEnergy
from forcefieldx_b200.system import PRECISION_FP64, PRECISION_MIXED, WATER_24K, WATER_648, Alchemy, water_box, \
    water_params
from oracle import binding as ob

pytestmark = pytest.mark.gpu


def _alchemy(n):
    soft = np.zeros(n, dtype=np.int32)
    soft[:30] = 1
    return Alchemy(soft=soft, molecule=np.arange(n) // 3)


def _check(s, p, lams, rel, rms_tol):
    a = _alchemy(s.n_atoms)
    with ForceFieldEnergy(s, p) as ffe:
        ffe.set_alchemy(a)
        for lam in lams:
            ffe.set_lambda(lam)
            for _ in range(2):                       # direct launches, then the captured graph
                e, g = ffe.energy_and_gradient(s.xyz)
                d1, d2, lg = ffe.get_dEdL()
                ref = ob.energy(s, p, alchemy=a, lam=lam)
                assert abs(ffe.terms[0] - ref["terms"][0]) < rel * abs(ref["terms"][0])
                assert abs(d1 - ref["dEdL"]) < rel * max(1.0, abs(ref["dEdL"])), (lam, d1, ref["dEdL"])
                assert abs(d2 - ref["d2EdL2"]) < 10 * rel * max(1.0, abs(ref["d2EdL2"])), (lam, d2, ref["d2EdL2"])
                assert float(np.sqrt(np.mean((lg - ref["dEdXdL"]) ** 2))) < rms_tol
                assert float(np.sqrt(np.mean((g - ref["grad"]) ** 2))) < rms_tol


def test_lambda_fp64_water_648():
    s = water_box(WATER_648["n_side"], WATER_648["edge"], seed=8)
    p = water_params(WATER_648["edge"], pme_grid=WATER_648["grid"], precision=PRECISION_FP64)
    _check(s, p, [0.1, 0.5, 0.9], 1e-8, 1e-6)


def test_lambda_mixed_water_648():
    s = water_box(WATER_648["n_side"], WATER_648["edge"], seed=8)
    p = water_params(WATER_648["edge"], pme_grid=WATER_648["grid"], precision=PRECISION_MIXED)
    _check(s, p, [0.1, 0.5, 0.9], 1e-5, 1e-3)


def test_lambda_fp64_water_24k():
    s = water_box(WATER_24K["n_side"], WATER_24K["edge"])
    p = water_params(WATER_24K["edge"], pme_grid=WATER_24K["grid"], precision=PRECISION_FP64)
    _check(s, p, [0.5], 1e-8, 1e-6)


def test_lambda_cleared_restores_plain_energy():
    s = water_box(WATER_648["n_side"], WATER_648["edge"], seed=8)
    p = water_params(WATER_648["edge"], pme_grid=WATER_648["grid"])
    with ForceFieldEnergy(s, p) as ffe:
        e0, _ = ffe.energy_and_gradient(s.xyz)
        ffe.set_alchemy(_alchemy(s.n_atoms))
        ffe.set_lambda(0.3)
        e1, _ = ffe.energy_and_gradient(s.xyz)
        assert abs(e1 - e0) > 1e-6
        ffe.set_alchemy(None)
        e2, _ = ffe.energy_and_gradient(s.xyz)
        assert abs(e2 - e0) < 1e-9 * abs(e0)
        assert ffe.get_dEdL()[0] == 0.0


# ---------------------------------------------------------------------------
# Electrostatic lambda (OST: condensed, condensed without the soft atoms, soft atoms in
# vacuum) against the oracle's restatement, which finite differences pin
# (tests/test_oracle_lambda.py).

def _elec(n):
    soft = np.zeros(n, dtype=np.int32)
    soft[:30] = 1
    return Alchemy(soft=soft, molecule=np.arange(n) // 3, elec=True)


def _check_elec(s, p, lams, rel, rms_tol):
    a = _elec(s.n_atoms)
    with ForceFieldEnergy(s, p) as ffe:
        ffe.set_alchemy(a)
        for lam in lams:
            ffe.set_lambda(lam)
            for _ in range(2):
                e, g = ffe.energy_and_gradient(s.xyz)
                d1, d2, lg = ffe.get_dEdL()
                ref = ob.energy(s, p, alchemy=a, lam=lam)
                scale = abs(ref["terms"][9])
                terr = np.abs(ffe.terms - ref["terms"])
                assert terr.max() < rel * max(scale, 1.0), (lam, ffe.terms, ref["terms"])
                assert abs(d1 - ref["dEdL"]) < rel * max(1.0, abs(ref["dEdL"]), scale), (lam, d1, ref["dEdL"])
                assert abs(d2 - ref["d2EdL2"]) < 10 * rel * max(1.0, abs(ref["d2EdL2"]), scale), (lam, d2, ref["d2EdL2"])
                assert float(np.sqrt(np.mean((g - ref["grad"]) ** 2))) < rms_tol, lam
                assert float(np.sqrt(np.mean((lg - ref["dEdXdL"]) ** 2))) < rms_tol, lam


def test_elec_lambda_fp64_water_648():
    s = water_box(WATER_648["n_side"], WATER_648["edge"], seed=8)
    p = water_params(WATER_648["edge"], pme_grid=WATER_648["grid"], precision=PRECISION_FP64)
    _check_elec(s, p, [0.3, 0.6, 0.85, 1.0], 1e-8, 1e-6)


def test_elec_lambda_mixed_water_648():
    s = water_box(WATER_648["n_side"], WATER_648["edge"], seed=8)
    p = water_params(WATER_648["edge"], pme_grid=WATER_648["grid"], precision=PRECISION_MIXED)
    _check_elec(s, p, [0.6, 0.85], 1e-5, 1e-3)


def test_elec_lambda_one_is_plain():
    s = water_box(WATER_648["n_side"], WATER_648["edge"], seed=8)
    p = water_params(WATER_648["edge"], pme_grid=WATER_648["grid"], precision=PRECISION_FP64)
    with ForceFieldEnergy(s, p) as ffe:
        e0, g0 = ffe.energy_and_gradient(s.xyz)
        ffe.set_alchemy(_elec(s.n_atoms))
        ffe.set_lambda(1.0)
        e1, g1 = ffe.energy_and_gradient(s.xyz)
        assert abs(e1 - e0) < 1e-9 * abs(e0)
        assert np.abs(g1 - g0).max() < 1e-8
        ffe.set_alchemy(None)
        e2, _ = ffe.energy_and_gradient(s.xyz)
        assert abs(e2 - e0) < 1e-9 * abs(e0)
