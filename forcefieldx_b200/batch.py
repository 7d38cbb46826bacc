"""Batches of independent periodic systems, and their partition over ranks.

The reference evaluates a set of systems (conformers, rotamers, lambda windows) one
``ForceFieldEnergy.energyAndGradient`` call at a time
(modules/potential/src/main/java/ffx/potential/ForceFieldEnergy.java:1843-1890).
``BatchEnergy`` evaluates the whole set through ``ffxg_batch_*`` (include/ffxcuda.h): one
coordinate upload, one CUDA-graph launch holding every system's evaluation, one gradient
download.  ``evaluate_partitioned`` spreads a set over ranks (one GPU each): systems are
assigned by atom count with the longest-processing-time greedy rule, every rank
evaluates its share with no exchange, and one all-reduce of the zero-padded per-system
results gives every rank the full table.
"""
from __future__ import annotations

import ctypes
import math
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from . import cabi
from .energy import EnergyException, ForceFieldEnergy, library
from .system import PRECISION_MIXED, AmoebaParams, AmoebaSystem, params_struct, small_water_box, water_params

BATCH_GRAPH, BATCH_LOOP, BATCH_BRANCHES = 0, 1, 2
_MODES = {"graph": BATCH_GRAPH, "loop": BATCH_LOOP, "branches": BATCH_BRANCHES}


def smooth235(n: int) -> int:
    """Smallest integer >= n whose prime factors are 2, 3 and 5."""
    m = max(1, int(n))
    while True:
        k = m
        for f in (2, 3, 5):
            while k % f == 0:
                k //= f
        if k == 1:
            return m
        m += 1


def pme_grid_for(edge: float, spacing: float = 1.2, minimum: int = 5) -> int:
    """Grid points per edge at <= ``spacing`` A, rounded up to 2,3,5-smooth (no minimum of
    16 as the reference's default sizing applies, ReciprocalSpace.java:938-947)."""
    return smooth235(max(minimum, int(math.ceil(edge / spacing - 1e-9))))


def batch_workload(n_systems: int = 512, seed: int = 2026, n_min: int = 96, n_max: int = 3000,
                   precision: int = PRECISION_MIXED, spacing: float = 1.2) -> List[Tuple[AmoebaSystem, AmoebaParams]]:
    """Water boxes of atom counts drawn uniformly from {n_min, n_min + 3, ..., n_max} at
    29.915 A^3 per molecule, each with its own PME grid, and the keys of the water
    configurations (9 A vdW, 7 A real space, alpha 0.545, order 5, PCG 1e-6 D)."""
    rng = np.random.default_rng(seed)
    counts = 3 * rng.integers(n_min // 3, n_max // 3 + 1, size=n_systems)
    out = []
    for j, n in enumerate(counts):
        s, edge = small_water_box(int(n), seed=seed + 1 + j)
        g = pme_grid_for(edge, spacing)
        out.append((s, water_params(edge, pme_grid=(g, g, g), precision=precision)))
    return out


class BatchEnergy:
    """Energy and gradient of many independent systems on one B200 (ffxg_batch_*)."""

    def __init__(self, systems: Sequence[AmoebaSystem], params: Sequence[AmoebaParams]):
        if len(systems) != len(params) or not systems:
            raise ValueError("one params per system, at least one system")
        self.lib = library()
        self.systems = list(systems)
        self.params = list(params)
        S = len(systems)
        sarr = (cabi.FfxgSystem * S)()
        parr = (cabi.FfxgParams * S)()
        keep = []
        for j, (s, p) in enumerate(zip(systems, params)):
            cs, k = s.c_struct(cabi)
            keep.append((cs, k))
            sarr[j] = cs
            parr[j] = params_struct(p, cabi)
        b = ctypes.c_void_p()
        st = self.lib.ffxg_batch_create(S, sarr, parr, ctypes.byref(b))
        if st != 0:
            raise EnergyException(st, self.lib.ffxg_batch_last_error(None).decode())
        self._b = b
        self.offsets = np.zeros(S + 1, dtype=np.int64)
        self.lib.ffxg_batch_atoms(b, self.offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        self.n_atoms = int(self.offsets[-1])
        self.terms = np.zeros((S, cabi.N_TERMS))
        self.counts = np.zeros((S, cabi.N_COUNTS), dtype=np.int64)
        self.status = np.zeros(S, dtype=np.int32)
        self._xyz = np.ascontiguousarray(np.concatenate([s.xyz for s in systems]), dtype=np.float64)
        self._grad = np.zeros((self.n_atoms, 3))

    def __len__(self):
        return len(self.systems)

    def close(self):
        if getattr(self, "_b", None):
            self.lib.ffxg_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_mode(self, mode) -> None:
        """"graph" (default: one CUDA graph, stage by stage), "branches" (one graph of
        per-system branches) or "loop" (single-system launches one after another).  A bool
        selects "loop" (True) or "graph" (False)."""
        if isinstance(mode, bool):
            mode = "loop" if mode else "graph"
        st = self.lib.ffxg_batch_set_mode(self._b, _MODES[mode])
        if st != 0:
            raise EnergyException(st, self.lib.ffxg_batch_last_error(self._b).decode())

    @property
    def graph_builds(self) -> int:
        return int(self.lib.ffxg_batch_graph_builds(self._b))

    def tuning(self):
        """(chosen number of groups, {groups: ms per batch} of the candidates timed) of the
        stage-by-stage graph's autotuning; (0, {}) before the first build."""
        import ctypes
        cand = (ctypes.c_int32 * 4)()
        ms = (ctypes.c_double * 4)()
        chosen = int(self.lib.ffxg_batch_tuning(self._b, cand, ms))
        return chosen, {int(cand[k]): float(ms[k]) for k in range(4) if cand[k] > 0}

    def set_groups(self, groups: int) -> None:
        """Fix the number of concurrent groups of the stage-by-stage graph (0: autotune)."""
        st = self.lib.ffxg_batch_set_groups(self._b, int(groups))
        if st != 0:
            raise EnergyException(st, "bad number of groups")

    def stages(self, gradient: bool = True) -> int:
        """Stages (one launch each for all systems) of the stage-by-stage graph; 0 when the
        batch runs as branches or has not been evaluated yet."""
        return int(self.lib.ffxg_batch_stages(self._b, 1 if gradient else 0))

    def system_energy(self, i: int) -> ForceFieldEnergy:
        """A non-owning ForceFieldEnergy on system i's handle (induced dipoles, lambda ...)."""
        h = self.lib.ffxg_batch_system(self._b, int(i))
        if not h:
            raise IndexError(i)
        return ForceFieldEnergy(self.systems[i], self.params[i], _handle=h)

    def split(self, flat: np.ndarray) -> List[np.ndarray]:
        return [flat[self.offsets[j]:self.offsets[j + 1]] for j in range(len(self))]

    def energy_and_gradient(self, xyz: Optional[Sequence[np.ndarray]] = None, gradient: bool = True,
                            raise_on_error: bool = True):
        """Returns (energies[S], gradients: list of [n_s, 3] views, or None)."""
        if xyz is not None:
            self._xyz = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.float64).reshape(-1, 3)
                                                             for x in xyz]))
            if self._xyz.shape[0] != self.n_atoms:
                raise ValueError("coordinates do not match the batch")
        D = ctypes.POINTER(ctypes.c_double)
        st = self.lib.ffxg_batch_energy(
            self._b, self._xyz.ctypes.data_as(D), 1 if gradient else 0, self.terms.ctypes.data_as(D),
            self._grad.ctypes.data_as(D) if gradient else None,
            self.counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            self.status.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        if st != 0 and raise_on_error:
            raise EnergyException(st, self.lib.ffxg_batch_last_error(self._b).decode())
        return self.terms[:, 9].copy(), (self.split(self._grad) if gradient else None)


def partition_lpt(sizes: Sequence[int], n_parts: int) -> List[List[int]]:
    """Longest-processing-time greedy: systems in decreasing size, each to the part with
    the least work so far (ties to the lower part); within a part, original order."""
    load = [0] * n_parts
    parts: List[List[int]] = [[] for _ in range(n_parts)]
    for j in sorted(range(len(sizes)), key=lambda t: (-sizes[t], t)):
        r = min(range(n_parts), key=lambda q: (load[q], q))
        parts[r].append(j)
        load[r] += int(sizes[j])
    return [sorted(p) for p in parts]


def evaluate_partitioned(systems: Sequence[AmoebaSystem], params: Sequence[AmoebaParams],
                         evaluate: Callable[[List[AmoebaSystem], List[AmoebaParams]], np.ndarray], width: int,
                         rank: int, world: int, all_reduce: Callable[[np.ndarray], np.ndarray]) -> np.ndarray:
    """Per-system result rows [S, width] for the whole set on every rank.  ``evaluate`` maps
    this rank's systems to a [k, width] array (e.g. the energy terms); ``all_reduce`` sums an
    array over ranks, called exactly once on every rank.  Rows of other ranks' systems are
    zero before the sum, so the sum is exact."""
    parts = partition_lpt([s.n_atoms for s in systems], world)
    mine = parts[rank]
    table = np.zeros((len(systems), width))
    if mine:
        local = np.asarray(evaluate([systems[j] for j in mine], [params[j] for j in mine]), dtype=np.float64)
        table[mine] = local.reshape(len(mine), width)
    return all_reduce(table)


def torch_all_reduce(group=None) -> Callable[[np.ndarray], np.ndarray]:
    """Sum over the ranks of a torch.distributed group (NCCL on GPUs, gloo on CPUs)."""
    import torch
    import torch.distributed as dist

    def reduce(a: np.ndarray) -> np.ndarray:
        dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return t.cpu().numpy()

    return reduce
