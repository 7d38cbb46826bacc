"""Batches (ffxg_batch_*) on the device.

1. Every system of a batch (multi-image and minimum-image boxes, 96-1,200 atoms, odd and
   even PME grids) gives the energy terms and gradient of its own single-system handle,
   in GRAPH mode (stage by stage: one launch per kernel for all systems), BRANCHES mode
   (one graph branch per system) and LOOP mode, on first and repeated calls and after the
   coordinates move: bit for bit in the mixed form, to rounding (1e-11) in the plain FP64
   form, whose mesh atomics add in arrival order.  A batch that mixes the two forms and a
   softcore system (different kernel instances in the same stages) does the same.
2. The plain FP64 batch against the oracle at the parity bar (1e-8 relative per term,
   1e-6 gradient RMS).
3. A lambda change on one system's handle makes the batch recapture its graph.
"""
import numpy as np
import pytest

from forcefieldx_b200.batch import BatchEnergy, batch_workload
from forcefieldx_b200.energy import ForceFieldEnergy
from forcefieldx_b200.system import PRECISION_FP64, PRECISION_MIXED, Alchemy
from oracle import binding as ob

pytestmark = pytest.mark.gpu


def _single(s, p, xs):
    """Results of one handle over the coordinate history xs (lists built at xs[0], as in
    the batch: the moves stay inside the list buffer, so summation orders agree)."""
    out = []
    with ForceFieldEnergy(s, p) as f:
        for x in xs:
            e, g = f.energy_and_gradient(x)
            out.append((f.terms.copy(), g.copy()))
    return out


@pytest.mark.parametrize("precision", [PRECISION_MIXED, PRECISION_FP64])
def test_batch_matches_single_system_handles(precision):
    w = batch_workload(n_systems=10, seed=31, n_min=96, n_max=1200, precision=precision)
    systems, params = [s for s, _ in w], [p for _, p in w]
    rng = np.random.default_rng(4)
    moved = [s.xyz + rng.normal(scale=0.05, size=s.xyz.shape) for s in systems]
    hist = [_single(s, p, [s.xyz, s.xyz, x]) for s, p, x in zip(systems, params, moved)]
    with BatchEnergy(systems, params) as b:
        for mode in ("graph", "loop", "branches", "graph"):
            b.set_mode(mode)
            for k, xs in enumerate(([s.xyz for s in systems], moved, moved)):
                e, grads = b.energy_and_gradient(xs)
                for j in range(len(systems)):
                    _same(precision, b.terms[j], grads[j], hist[j][1 if k == 0 else 2], (mode, k, j))
            if mode == "graph":
                assert b.stages() > 50
                chosen, times = b.tuning()
                assert chosen in (1, 2, 4, 8) and chosen in times and min(times, key=times.get) == chosen
        assert b.graph_builds >= 1
        for groups in (3, 1):     # a fixed number of groups: the same results
            b.set_groups(groups)
            e, grads = b.energy_and_gradient(moved)
            for j in range(len(systems)):
                _same(precision, b.terms[j], grads[j], hist[j][2], ("groups", groups, j))
            assert b.tuning()[0] == groups


def _same(precision, terms, grad, ref, tag):
    if precision == PRECISION_MIXED:     # deterministic form: bit for bit
        assert np.array_equal(terms, ref[0]), (tag, terms, ref[0])
        assert np.array_equal(grad, ref[1]), tag
    else:   # FP64 mesh atomics add in arrival order: rounding-level differences
        rel = np.abs(terms - ref[0]) / np.maximum(np.abs(ref[0]), 1.0)
        assert rel.max() < 1e-11, (tag, rel)
        assert np.abs(grad - ref[1]).max() < 1e-9, tag


def test_staged_batch_of_mixed_forms_and_a_softcore_system():
    w = batch_workload(n_systems=6, seed=41, n_min=96, n_max=900, precision=PRECISION_MIXED)
    systems = [s for s, _ in w]
    params = [p if j % 2 else type(p)(**{**p.__dict__, "precision": PRECISION_FP64}) for j, (_, p) in enumerate(w)]
    soft = np.zeros(systems[1].n_atoms, dtype=np.int32)
    soft[:6] = 1
    alch = Alchemy(soft=soft, molecule=np.arange(systems[1].n_atoms) // 3)
    hist = []
    for j, (s, p) in enumerate(zip(systems, params)):
        with ForceFieldEnergy(s, p) as f:
            if j == 1:
                f.set_alchemy(alch)
                f.set_lambda(0.6)
            f.energy_and_gradient(s.xyz)
            e, g = f.energy_and_gradient(s.xyz)
            hist.append((f.terms.copy(), g.copy()))
    with BatchEnergy(systems, params) as b:
        sf = b.system_energy(1)
        sf.set_alchemy(alch)
        sf.set_lambda(0.6)
        for _ in range(3):
            e, grads = b.energy_and_gradient()
            for j in range(len(systems)):
                _same(params[j].precision, b.terms[j], grads[j], hist[j], j)
        assert b.stages() > 50


def test_batch_fp64_against_oracle():
    w = batch_workload(n_systems=6, seed=7, n_min=96, n_max=600, precision=PRECISION_FP64)
    systems, params = [s for s, _ in w], [p for _, p in w]
    with BatchEnergy(systems, params) as b:
        for _ in range(2):
            e, grads = b.energy_and_gradient()
            for j, (s, p) in enumerate(w):
                ref = ob.energy(s, p)
                rel = np.abs(b.terms[j] - ref["terms"]) / np.maximum(np.abs(ref["terms"]), 1.0)
                assert rel.max() < 1e-8, (j, rel)
                assert float(np.sqrt(np.mean((grads[j] - ref["grad"]) ** 2))) < 1e-6
                assert b.counts[j][2] == ref["counts"][2]


def test_lambda_change_recaptures_batch_graph():
    w = batch_workload(n_systems=4, seed=17, n_min=96, n_max=300, precision=PRECISION_FP64)
    systems, params = [s for s, _ in w], [p for _, p in w]
    with BatchEnergy(systems, params) as b:
        b.energy_and_gradient()
        e0, _ = b.energy_and_gradient()
        builds = b.graph_builds
        s0 = systems[0]
        soft = np.zeros(s0.n_atoms, dtype=np.int32)
        soft[:6] = 1
        a = Alchemy(soft=soft, molecule=np.arange(s0.n_atoms) // 3)
        f = b.system_energy(0)
        f.set_alchemy(a)
        f.set_lambda(0.5)
        e1, g1 = b.energy_and_gradient()
        assert b.graph_builds == builds + 1
        ref = ob.energy(s0, params[0], alchemy=a, lam=0.5)
        assert abs(e1[0] - ref["terms"][9]) < 1e-8 * abs(ref["terms"][9])
        assert np.all(np.abs(e1[1:] - e0[1:]) < 1e-11 * np.abs(e0[1:]))   # the other systems unchanged


@pytest.mark.parametrize("precision", [PRECISION_MIXED, PRECISION_FP64])
def test_staged_batch_of_the_reference_crystals(precision, fixtures):
    """The five small-molecule crystals (P1 cells of their mates, monoclinic and
    orthorhombic, every lattice image listed) as one stage-by-stage batch against their
    own handles."""
    from tests.common import CRYSTALS, golden_system
    pairs = [golden_system(name, fixtures, precision=precision) for name in CRYSTALS]
    systems, params = [s for s, _ in pairs], [p for _, p in pairs]
    hist = []
    for s, p in pairs:
        with ForceFieldEnergy(s, p) as f:
            f.energy_and_gradient(s.xyz)
            e, g = f.energy_and_gradient(s.xyz)
            hist.append((f.terms.copy(), g.copy()))
    with BatchEnergy(systems, params) as b:
        for _ in range(3):
            e, grads = b.energy_and_gradient()
            for j in range(len(systems)):
                _same(precision, b.terms[j], grads[j], hist[j], CRYSTALS[j])
        assert b.stages() > 50


def test_large_batch_host_copies_and_nonfinite_coordinates():
    """A batch of ~180,000 atoms, whose coordinate and gradient copies are split over
    several host threads: every system's result is its own handle's (bit for bit, mixed
    form); a NaN in the last system's coordinates is rejected (NONFINITE) without running,
    after which there are no coordinates to reuse (a NULL pointer: BAD_ARG); valid
    coordinates then give the first results again."""
    import ctypes
    from forcefieldx_b200.energy import EnergyException
    w = batch_workload(n_systems=64, seed=53, n_min=2700, n_max=3000, precision=PRECISION_MIXED)
    systems, params = [s for s, _ in w], [p for _, p in w]
    assert 3 * sum(s.n_atoms for s in systems) >= 2 * (1 << 18)   # at least two copy threads
    checked = [0, 31, 63]
    hist = {j: _single(systems[j], params[j], [systems[j].xyz, systems[j].xyz])[1] for j in checked}
    with BatchEnergy(systems, params) as b:
        xs = [s.xyz for s in systems]
        for _ in range(2):
            e0, grads = b.energy_and_gradient(xs)
        for j in checked:
            _same(PRECISION_MIXED, b.terms[j], grads[j], hist[j], j)
        bad = [x.copy() for x in xs]
        bad[-1][-1, 2] = np.nan
        with pytest.raises(EnergyException) as ei:
            b.energy_and_gradient(bad)
        assert ei.value.status == 5                     # FFXG_ERR_NONFINITE
        D = ctypes.POINTER(ctypes.c_double)
        st = b.lib.ffxg_batch_energy(b._b, None, 1, b.terms.ctypes.data_as(D), b._grad.ctypes.data_as(D), None, None)
        assert st == 1                                  # FFXG_ERR_BAD_ARG: nothing to reuse
        e1, grads = b.energy_and_gradient(xs)
        assert np.array_equal(e1, e0)
        for j in checked:
            _same(PRECISION_MIXED, b.terms[j], grads[j], hist[j], j)
