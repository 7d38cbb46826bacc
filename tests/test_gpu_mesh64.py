"""64 x 64 x 64 meshes and the near list's fallback.

1. FP64 form on a 64^3 mesh (the compile-time-length FFT passes) against the oracle at the
   parity bar: 1e-8 relative per term, 1e-6 gradient RMS, identical counts.
2. Mixed form on the same mesh (X and Y passes fused by four-CTA clusters, the double
   accumulation mesh cleared by its reader) at the mixed bar, bit for bit on repeated
   calls: a mesh left dirty by one call would change the next.
3. A hydrogen whose vdW reduction factor is 0.5 (its reduced site half-way to the
   oxygen, 0.48 A from the atom): the offset exceeds the near list's 0.25 A margin, so
   every evaluation takes the fallback (Ewald sub-lists from the buffered rows), which
   must match the oracle with identical pair counts.
"""
import numpy as np
import pytest

from forcefieldx_b200.system import PRECISION_MIXED, AmoebaSystem, water_box, water_params
from tests.test_gpu_parity import compare
from tests.test_gpu_precision_mixed import compare_mixed

pytestmark = pytest.mark.gpu

N_WATERS = 1500
EDGE = (N_WATERS * 29.915) ** (1.0 / 3.0)    # 35.52 A at the water boxes' density


def _box(seed):
    return water_box(12, EDGE, seed=seed, n_waters=N_WATERS)


def test_fp64_mesh64_against_oracle():
    s = _box(41)
    compare(s, water_params(EDGE, pme_grid=(64, 64, 64)), check_pairs=False)


def test_fp64_repeat_agrees_to_rounding():
    """The FP64 form adds the mesh and the real-space k-side force and torque with FP64
    atomics in arrival order, so repeated calls agree to rounding, not bit for bit (the
    mixed form's quantised sums do repeat exactly)."""
    from forcefieldx_b200.energy import ForceFieldEnergy
    s = _box(45)
    with ForceFieldEnergy(s, water_params(EDGE, pme_grid=(64, 64, 64))) as ffe:
        e1, g1 = ffe.energy_and_gradient(s.xyz)
        t1 = ffe.terms.copy()
        e2, g2 = ffe.energy_and_gradient(s.xyz)
        t2 = ffe.terms.copy()
    assert np.max(np.abs(t1 - t2) / np.maximum(np.abs(t1), 1.0)) < 1e-12
    assert np.max(np.abs(g1 - g2)) < 1e-9


def test_mixed_mesh64_against_oracle_and_repeatable():
    s = _box(43)
    compare_mixed(s, water_params(EDGE, pme_grid=(64, 64, 64), precision=PRECISION_MIXED))


def test_near_list_fallback_matches_oracle():
    s = _box(47)
    o, h = 0, 1                                   # water 0: oxygen 0, hydrogen 1
    red = np.array(s.red_factor, dtype=np.float64).copy()
    red[h] = 0.5
    assert (1.0 - red[h]) * np.linalg.norm(s.xyz[h] - s.xyz[o]) > 0.25
    t = AmoebaSystem(**{**s.__dict__, "red_factor": red})
    compare(t, water_params(EDGE, pme_grid=(40, 40, 40)), check_pairs=False)
