"""Parameter gradients of the oracle against central finite differences.

dE/dM for each atom's local-frame multipole components and dE/dalpha for its
polarizability (Thole damping held fixed), in all three polarization models.  The
reference has no analytic parameter gradient to compare with, so finite differences are
the pin (step 1e-6 in the parameter, PCG converged to 1e-12 D so the solve error stays
below the difference quotient's).
"""
import dataclasses

import numpy as np
import pytest

from forcefieldx_b200.system import PRECISION_FP64, water_box, water_params
from oracle import binding as ob


def _setup(polarization):
    s = water_box(3, 9.3215, seed=4)
    p = water_params(9.3215, vdw_cutoff=4.5, ewald_cutoff=4.5, pme_grid=(12, 12, 12), polar_eps=1e-12,
                     precision=PRECISION_FP64, polarization=polarization)
    return s, p


def _fd(s, p, field, atom, comp, h=1e-6):
    vals = []
    for sign in (1, -1):
        arr = getattr(s, field).copy()
        if comp is None:
            arr[atom] += sign * h
        else:
            arr[atom, comp] += sign * h
        vals.append(ob.energy(dataclasses.replace(s, **{field: arr}), p, gradient=False)["terms"][9])
    return (vals[0] - vals[1]) / (2 * h)


@pytest.mark.parametrize("polarization", [0, 1, 2])
def test_multipole_gradients(polarization):
    s, p = _setup(polarization)
    dM, _ = ob.param_gradients(s, p)
    for atom in (0, 1, 5):
        for c in range(10):
            fd = _fd(s, p, "multipole", atom, c)
            assert abs(fd - dM[atom, c]) < 1e-5 * max(1.0, abs(fd)), (atom, c, fd, dM[atom, c])


@pytest.mark.parametrize("polarization", [1, 2])
def test_polarizability_gradients(polarization):
    s, p = _setup(polarization)
    _, dA = ob.param_gradients(s, p)
    for atom in (0, 1, 2, 9):
        fd = _fd(s, p, "polarizability", atom, None)
        assert abs(fd - dA[atom]) < 1e-5 * max(1.0, abs(fd)), (atom, fd, dA[atom])
