"""Failure and recovery paths of the CUDA library, provoked from the host with inputs alone.

* List regrowth: a handle sized for a dilute box meets a configuration at twice its
  density; the rows overflow their capacity, the library grows them and repeats the
  evaluation (from a replayed graph as well as from direct launches), and the result is
  the oracle's.
* SCF divergence: with Thole damping off, intramolecular O-H pairs of AMOEBA water sit
  inside the polarization catastrophe radius (r^6 < 4 alpha_i alpha_k), the polarization
  matrix is indefinite and the residual grows: FFXG_ERR_SCF_DIVERGED, as the reference
  throws it (PCGSolver.java:547-559).
* The mixed form's fixed-point range: a close contact drives real-space forces above
  2^20 kcal/mol/A; the call completes and returns FFXG_ERR_RANGE.
* List regrowth inside a batch graph (stage by stage and as branches): the overflowing
  system is repeated directly and the batch graph rebuilt on the grown lists.
* The FFT's shared-memory limit is process-wide: a mesh whose longest axis comes first
  needs more than 48 KB per line batch, and creating a handle with smaller axes later
  must not take that limit away from the first handle.
"""
import dataclasses
import warnings

import numpy as np
import pytest

from forcefieldx_b200 import cabi
from forcefieldx_b200.energy import EnergyException, ForceFieldEnergy
from forcefieldx_b200.system import POLAR_NONE, PRECISION_FP64, PRECISION_MIXED, water_box, water_params
from oracle import binding as ob
from tests.common import golden_system

pytestmark = pytest.mark.gpu

E_REL = 1.0e-8
G_RMS = 1.0e-6


def _dilute_and_compact(seed):
    """216 waters: compact at 1 g/cm^3 (an 18.643 A cube) and the same molecules spread
    rigidly over a 24 A cube (0.47 g/cm^3), both in a 24 A periodic box."""
    s = water_box(6, 18.643, seed=seed)
    o = s.xyz[0::3]
    shift = np.repeat(o * (24.0 / 18.643 - 1.0), 3, axis=0)
    dilute = dataclasses.replace(s, xyz=s.xyz + shift)
    return dilute, s.xyz.copy()


@pytest.mark.parametrize("graph", [True, False])
def test_list_overflow_regrows_and_matches_oracle(graph):
    dilute, compact = _dilute_and_compact(seed=17)
    p = water_params(24.0, pme_grid=(24, 24, 24), precision=PRECISION_FP64)
    ref = ob.energy(dilute, p, xyz=compact)
    assert ref["status"] == 0
    with ForceFieldEnergy(dilute, p) as ffe:
        ffe.set_graph_mode(graph)
        ffe.energy_and_gradient(dilute.xyz)          # lists sized for the dilute density
        assert ffe.count("list_growths") == 0
        ffe.energy_and_gradient(dilute.xyz)          # (graph mode: captured and replayed)
        e, g = ffe.energy_and_gradient(compact)       # rows overflow: grow and repeat
        assert ffe.count("list_growths") >= 1
        assert ffe.count("list_builds") == 1
        terms = ffe.terms.copy()
        rel = np.abs(terms - ref["terms"]) / np.maximum(np.abs(ref["terms"]), 1.0)
        assert rel.max() < E_REL, (terms, ref["terms"])
        assert float(np.sqrt(np.mean((g - ref["grad"]) ** 2))) < G_RMS
        assert ffe.counts[2] == ref["counts"][2]
        e2, g2 = ffe.energy_and_gradient(compact)     # the grown lists hold: no further growth
        assert ffe.count("list_growths") == 0
        assert abs(e2 - e) < 1e-9 * abs(e)


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_MIXED])
@pytest.mark.parametrize("graph", [True, False])
def test_scf_divergence_is_reported(precision, graph):
    s = water_box(6, 18.643, seed=21)
    s = dataclasses.replace(s, thole=np.zeros_like(s.thole), pdamp=np.zeros_like(s.pdamp))
    p = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 20), max_scf_iter=200,
                     precision=precision)
    assert ob.energy(s, p)["status"] == 3
    with ForceFieldEnergy(s, p) as ffe:
        ffe.set_graph_mode(graph)
        for _ in range(2):                           # list build, then (graph mode) the replay
            with pytest.raises(EnergyException) as ei:
                ffe.energy(s.xyz)
            assert ei.value.status == 3              # FFXG_ERR_SCF_DIVERGED


def test_fixed_point_range_is_reported():
    s = water_box(6, 18.643, seed=23)
    x = s.xyz.copy()
    x[4] = x[0] + np.array([0.02, 0.0, 0.0])        # an H of water 1 on the O of water 0
    out = {}
    for precision in (PRECISION_FP64, PRECISION_MIXED):
        p = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 20),
                         polarization=POLAR_NONE, precision=precision)
        with ForceFieldEnergy(s, p) as ffe:
            ffe.energy_and_gradient(s.xyz)
            assert ffe.last_status == 0
            with warnings.catch_warnings(record=True) as w:
                warnings.simplefilter("always")
                e, g = ffe.energy_and_gradient(x)
            out[precision] = (ffe.last_status, e, g, len(w))
    st64, e64, g64, _ = out[PRECISION_FP64]
    stm, em, gm, nw = out[PRECISION_MIXED]
    assert st64 == 0
    assert np.abs(g64).max() >= 2.0 ** 20          # the contact's forces are beyond the range
    assert stm == cabi.STATUS_RANGE and nw == 1      # mixed: reported, outputs complete
    assert np.all(np.isfinite(gm)) and np.isfinite(em)


def test_fft_long_first_axis_mesh():
    """A (160, 48, 64) mesh: the first axis's line batch needs 80 KB of shared memory."""
    s = water_box(6, 18.643, seed=29)
    p = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(160, 48, 64))
    ref = ob.energy(s, p)
    with ForceFieldEnergy(s, p) as ffe:
        e, g = ffe.energy_and_gradient(s.xyz)
        terms = ffe.terms.copy()
    rel = np.abs(terms - ref["terms"]) / np.maximum(np.abs(ref["terms"]), 1.0)
    assert rel.max() < E_REL, (terms, ref["terms"])
    assert float(np.sqrt(np.mean((g - ref["grad"]) ** 2))) < G_RMS


@pytest.mark.parametrize("graph", [True, False])
def test_fft_limit_survives_later_handles(fixtures, graph):
    """SNARE's (48, 64, 160) mesh, then handles with 64^3 and 20^3 meshes, then SNARE again."""
    s, p = golden_system("snare", fixtures)
    ref = ob.energy(s, p)
    with ForceFieldEnergy(s, p) as big:
        big.set_graph_mode(graph)
        big.energy_and_gradient(s.xyz)
        first = big.terms.copy()
        w = water_box(6, 18.643, seed=2)
        for grid in ((64, 64, 64), (20, 20, 20)):
            with ForceFieldEnergy(w, water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=grid)) as small:
                small.energy_and_gradient(w.xyz)
        e, g = big.energy_and_gradient(s.xyz)
        terms = big.terms.copy()
    rel = np.abs(terms - ref["terms"]) / np.maximum(np.abs(ref["terms"]), 1.0)
    assert rel.max() < E_REL, (terms, ref["terms"])
    assert np.max(np.abs(terms - first) / np.maximum(np.abs(first), 1.0)) < 1e-11
    assert float(np.sqrt(np.mean((g - ref["grad"]) ** 2))) < G_RMS


@pytest.mark.parametrize("mode", ["graph", "branches"])
def test_list_overflow_inside_a_batch_graph(mode):
    """One system of a batch meets a configuration at twice its density while the batch
    replays its graph: the system's rows overflow, the batch drops its graph, grows that
    system's lists and repeats it directly, and every system's result is the oracle's; the
    next call rebuilds the batch graph on the grown lists."""
    from forcefieldx_b200.batch import BatchEnergy
    dilute, compact = _dilute_and_compact(seed=23)
    other = water_box(6, 18.643, seed=29)
    p24 = water_params(24.0, pme_grid=(24, 24, 24), precision=PRECISION_FP64)
    p18 = water_params(18.643, pme_grid=(20, 20, 20), precision=PRECISION_FP64)
    with BatchEnergy([dilute, other], [p24, p18]) as b:
        b.set_mode(mode)
        for _ in range(2):                          # lists built, then the batch graph
            b.energy_and_gradient([dilute.xyz, other.xyz])
        builds = b.graph_builds
        for call in range(2):
            e, grads = b.energy_and_gradient([compact, other.xyz])
            for j, (s, p, x) in enumerate([(dilute, p24, compact), (other, p18, other.xyz)]):
                ref = ob.energy(s, p, xyz=x)
                rel = np.abs(b.terms[j] - ref["terms"]) / np.maximum(np.abs(ref["terms"]), 1.0)
                assert rel.max() < E_REL, (mode, call, j, b.terms[j], ref["terms"])
                assert float(np.sqrt(np.mean((grads[j] - ref["grad"]) ** 2))) < G_RMS
            if call == 0:
                assert b.counts[0][5] >= 1           # the dense system's lists grew
        assert b.graph_builds > builds               # rebuilt on the grown lists
