"""Host logic of batches: the workload generator, the per-system PME grid rule, the
longest-processing-time partition, and the partitioned evaluation over two gloo ranks
(CPU processes; each rank evaluates its share with the oracle, one all-reduce gathers
the table) against a serial evaluation."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from forcefieldx_b200.batch import batch_workload, evaluate_partitioned, partition_lpt, pme_grid_for, smooth235, \
    torch_all_reduce
from forcefieldx_b200.system import PRECISION_FP64
from oracle import binding as ob


def test_smooth235():
    assert [smooth235(n) for n in (1, 7, 11, 13, 17, 26, 49, 97)] == [1, 8, 12, 15, 18, 27, 50, 100]


def test_pme_grid_rule():
    # 96 atoms: 9.86 A edge -> ceil(8.2) = 9; 3000 atoms: 31.03 A -> 26 -> 27.
    assert pme_grid_for(9.8555) == 9
    assert pme_grid_for(31.03) == 27
    assert pme_grid_for(62.08) == 54


def test_workload_shapes():
    w = batch_workload(n_systems=40, seed=5)
    sizes = [s.n_atoms for s, _ in w]
    assert all(96 <= n <= 3000 and n % 3 == 0 for n in sizes)
    for s, p in w:
        edge = p.box[0]
        assert abs(s.n_atoms / 3 * 29.915 - edge ** 3) < 1e-6 * edge ** 3
        assert edge / p.pme_grid[0] <= 1.2 + 1e-12
        assert smooth235(p.pme_grid[0]) == p.pme_grid[0]


def test_partition_lpt_covers_and_balances():
    rng = np.random.default_rng(0)
    sizes = 3 * rng.integers(32, 1001, size=512)
    for world in (1, 2, 3, 8):
        parts = partition_lpt(sizes, world)
        flat = sorted(j for p in parts for j in p)
        assert flat == list(range(512))
        loads = [int(sizes[p].sum()) for p in parts]
        # LPT bound: max load <= mean + largest item.
        assert max(loads) <= sum(loads) / world + sizes.max()


def _workload():
    return batch_workload(n_systems=5, seed=9, n_min=96, n_max=240, precision=PRECISION_FP64)


def _oracle_terms(systems, params):
    return np.array([ob.energy(s, p, gradient=False, nthreads=1)["terms"] for s, p in zip(systems, params)])


def _rank(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = _workload()
        table = evaluate_partitioned([s for s, _ in w], [p for _, p in w], _oracle_terms, 10, rank, world,
                                     torch_all_reduce())
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), table)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partitioned_evaluation_two_gloo_ranks(tmp_path):
    mp.spawn(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    w = _workload()
    serial = _oracle_terms([s for s, _ in w], [p for _, p in w])
    for r in range(2):
        table = np.load(tmp_path / f"rank{r}.npy")
        assert np.array_equal(table, serial)
