"""The mixed-precision form (FFXG_PRECISION_MIXED) against the FP64 oracle.

Bar: total energy within 1e-5 relative, each energy term within 1e-5 of the total's
magnitude, gradient RMS within 1e-3 kcal/mol/A, identical interaction counts (the
neighbour list, the cutoff tests and the exclusion masks are FP64 in both forms), and
bitwise-identical results on repeated calls (fixed-point mesh accumulation and
fixed-order reductions).
"""
import numpy as np
import pytest

from forcefieldx_b200.energy import ForceFieldEnergy
from forcefieldx_b200.system import PRECISION_MIXED, WATER_24K, water_box, water_params
from oracle import binding as ob
from tests.common import golden_system

pytestmark = pytest.mark.gpu

E_TOTAL_REL = 1.0e-5    # total energy, relative
G_RMS = 1.0e-3          # gradient RMS, kcal/mol/A
U_RMS = 1.0e-5          # induced dipole RMS, e*A


def compare_mixed(system, params, xyz=None):
    x = system.xyz if xyz is None else xyz
    ref = ob.energy(system, params, xyz=x)
    assert ref["status"] == 0
    with ForceFieldEnergy(system, params) as ffe:
        e, g = ffe.energy_and_gradient(x)
        assert ffe.last_status == 0                  # no fixed-point sum left its exact range
        terms, counts = ffe.terms.copy(), ffe.counts.copy()
        u, _ = ffe.get_induced_dipoles()
        e2, g2 = ffe.energy_and_gradient(x)
        terms2 = ffe.terms.copy()
    total = ref["terms"][9]
    term_err = np.abs(terms - ref["terms"])
    rms = float(np.sqrt(np.mean((g - ref["grad"]) ** 2)))
    report = f"term errors {term_err}, total {total}, gradient RMS error {rms}"
    assert abs(terms[9] - total) < E_TOTAL_REL * abs(total), report
    assert term_err.max() < E_TOTAL_REL * abs(total), report
    assert rms < G_RMS, report
    assert counts[0] == ref["counts"][0] and counts[1] == ref["counts"][1]
    assert abs(int(counts[2]) - int(ref["counts"][2])) <= 1          # PCG iterations
    assert float(np.sqrt(np.mean((u - ref["induced"]) ** 2))) < U_RMS
    # Deterministic: the second call reproduces the first bit for bit.
    assert np.array_equal(terms, terms2) and np.array_equal(g, g2)
    return term_err, rms


def test_mixed_water_648():
    s = water_box(6, 18.643, seed=21)
    p = water_params(18.643, pme_grid=(20, 20, 20), precision=PRECISION_MIXED)
    compare_mixed(s, p)


@pytest.mark.parametrize("name", ["ubiquitin", "dhfr"])
def test_mixed_reference_golden(name, fixtures):
    s, p = golden_system(name, fixtures, precision=PRECISION_MIXED)
    compare_mixed(s, p)


def test_mixed_water_24k_configurations():
    s = water_box(WATER_24K["n_side"], WATER_24K["edge"])
    p = water_params(WATER_24K["edge"], pme_grid=WATER_24K["grid"], precision=PRECISION_MIXED)
    rng = np.random.default_rng(300)
    for c in range(2):
        x = s.xyz + rng.normal(0.0, 0.02, s.xyz.shape)   # thermal-scale displacements
        compare_mixed(s, p, x)
