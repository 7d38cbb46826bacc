"""Direct and no polarization against the oracle, in both precision forms.

The real-space energy kernel has two layouts: half rows (each pair once, atom k's force and
torque by atomics) for mutual and no polarization, and full rows (atom i's share only) for
direct polarization, whose extra terms are compiled in only there.  The mutual form is
covered by the other parity tests; these cover the other two modes in the FP64 form
(1e-8 relative per term, 1e-6 gradient RMS) and direct polarization in the mixed form
(its own bar, with bitwise repeatability).
"""
import pytest

from forcefieldx_b200.system import POLAR_DIRECT, POLAR_NONE, PRECISION_MIXED, water_box, water_params
from tests.test_gpu_parity import compare
from tests.test_gpu_precision_mixed import compare_mixed

pytestmark = pytest.mark.gpu

EDGE = 18.643


def _params(polarization, **kw):
    return water_params(EDGE, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 20),
                        polarization=polarization, **kw)


@pytest.mark.parametrize("polarization", [POLAR_DIRECT, POLAR_NONE])
def test_fp64_polarization_mode(polarization):
    compare(water_box(6, EDGE, seed=23), _params(polarization), check_pairs=False)


def test_mixed_direct_polarization():
    # The mixed bar bounds each term by 1e-5 of the total energy.  Without polarization this
    # box's total is a near cancellation (76 kcal/mol), which makes that per-term bound
    # tighter than the form's FP32 rounding (8e-4 on a ~1e3 real-space term).  That mode
    # runs the half-row layout which the mutual mixed tests already cover.
    compare_mixed(water_box(6, EDGE, seed=29), _params(POLAR_DIRECT, precision=PRECISION_MIXED))
