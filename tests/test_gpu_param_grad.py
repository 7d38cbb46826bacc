"""Parameter gradients on the device (ffxg_param_grad) against the oracle's, which finite
differences pin (tests/test_oracle_param_grad.py): dE/dM of every atom's local multipole and
dE/dalpha, the 648-atom water box in three polarization models and the 24,000-atom box
(both forms).
FP64 form: 1e-8 relative to the largest component; mixed form: 1e-4.
"""
import numpy as np
import pytest

from forcefieldx_b200.energy import ForceFieldEnergy
from forcefieldx_b200.system import PRECISION_FP64, PRECISION_MIXED, WATER_24K, WATER_648, water_box, water_params
from oracle import binding as ob

pytestmark = pytest.mark.gpu


_ORACLE = {}


def _check(s, p, tol, key=None):
    with ForceFieldEnergy(s, p) as ffe:
        ffe.energy_and_gradient(s.xyz)
        dM, dA = ffe.param_gradients()
    if key is None or key not in _ORACLE:
        # The oracle's FP64 parameter gradients (the same for both device forms).
        pr = type(p)(**{**p.__dict__, "precision": PRECISION_FP64})
        res = ob.param_gradients(s, pr)
        if key is not None:
            _ORACLE[key] = res
    rM, rA = _ORACLE[key] if key is not None else res
    scale = np.abs(rM).max()
    assert np.abs(dM - rM).max() < tol * scale, (np.abs(dM - rM).max(), scale)
    if np.abs(rA).max() > 0:
        assert np.abs(dA - rA).max() < tol * np.abs(rA).max()
    else:
        assert np.abs(dA).max() == 0.0


@pytest.mark.parametrize("polarization", [0, 1, 2])
def test_param_grad_fp64_water_648(polarization):
    s = water_box(WATER_648["n_side"], WATER_648["edge"], seed=6)
    p = water_params(WATER_648["edge"], pme_grid=WATER_648["grid"], polarization=polarization,
                     precision=PRECISION_FP64)
    _check(s, p, 1e-8)


def test_param_grad_mixed_water_648():
    s = water_box(WATER_648["n_side"], WATER_648["edge"], seed=6)
    p = water_params(WATER_648["edge"], pme_grid=WATER_648["grid"], precision=PRECISION_MIXED)
    _check(s, p, 1e-4)


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_MIXED])
def test_param_grad_water_24k(precision):
    s = water_box(WATER_24K["n_side"], WATER_24K["edge"])
    p = water_params(WATER_24K["edge"], pme_grid=WATER_24K["grid"], precision=precision)
    _check(s, p, 1e-8 if precision == PRECISION_FP64 else 1e-4, key="24k")
