"""Host logic of the multi-GPU path on CPU: two gloo ranks (no GPU).

bench.py under torchrun runs one process per GPU with no collective on the data path:
timings are reduced to the slowest rank, and conformer batches shard by molecules.  These
tests run that host logic with world_size 2 over gloo on 127.0.0.1."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _sizes():
    rng = np.random.default_rng(11)
    return [int(round(np.exp(rng.uniform(np.log(20), np.log(300))))) for _ in range(200)]


def _worker(rank, world, port):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from curcuma_b200.sharding import shard_by_cost, shard_costs

        # slowest rank's time
        assert bench.max_over_ranks(1.5 + rank, dist, "cpu") == 1.5 + (world - 1)
        # every rank computes the same partition and takes its own shard
        sizes = _sizes()
        mine = shard_by_cost(sizes, world)[rank]
        got = [None] * world
        dist.all_gather_object(got, mine)
        flat = sorted(i for s in got for i in s)
        assert flat == list(range(len(sizes))), "shards must partition the batch"
        c = shard_costs(sizes, got)
        assert max(c) / min(c) < 1.02, c
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    mp.spawn(_worker, args=(2, _free_port()), nprocs=2, join=True)


def test_shard_by_cost_single_process():
    from curcuma_b200.sharding import molecule_cost, shard_by_cost, shard_costs

    sizes = _sizes()
    for k in (1, 3, 8):
        sh = shard_by_cost(sizes, k)
        assert sorted(i for s in sh for i in s) == list(range(len(sizes)))
        c = shard_costs(sizes, sh)
        # LPT bound: no shard exceeds the mean by more than the largest single molecule
        assert max(c) - sum(c) / k <= max(molecule_cost(n) for n in sizes) + 1e-9
    assert shard_by_cost(sizes, 4) == shard_by_cost(list(sizes), 4)   # deterministic


def _ensemble():
    from curcuma_b200 import workloads
    return workloads.conformer_batch(12, 33, lo=20, hi=80)


def _shard_worker(rank, world, port, out_path):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from curcuma_b200.sharding import gather_ensemble, shard_by_cost
        from tests.oracle_api import Oracle

        ens = _ensemble()
        sizes = [len(z) for z, _ in ens]
        idx = shard_by_cost(sizes, world)[rank]
        # this rank's shard evaluated by the CPU oracle (the per-rank evaluator on CPU)
        E, G = [], []
        for m in idx:
            z, x = ens[m]
            T, g, q, cn = Oracle(z, x).engrad(x, 1)
            E.append(T["total"])
            G.append(g)
        E_all, G_all = gather_ensemble(idx, E, np.concatenate(G), sizes, dist.all_gather_object, world)
        if rank == 0:
            np.savez(out_path, E=E_all, G=G_all)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_ensemble_shards_gather_to_the_single_process_result(tmp_path):
    """One ensemble split over two gloo ranks (shard_by_cost), each shard evaluated on its
    rank, energies and gradients gathered in ensemble order: equal to the one-process
    evaluation of the whole ensemble."""
    out = tmp_path / "gathered.npz"
    mp.spawn(_shard_worker, args=(2, _free_port(), str(out)), nprocs=2, join=True)
    got = np.load(out)
    from tests.oracle_api import Oracle
    E, G = [], []
    for z, x in _ensemble():
        T, g, q, cn = Oracle(z, x).engrad(x, 1)
        E.append(T["total"])
        G.append(g)
    assert np.array_equal(got["E"], np.array(E))
    assert np.array_equal(got["G"], np.concatenate(G))


def test_gather_rejects_incomplete_shards():
    from curcuma_b200.sharding import gather_ensemble

    def fake_all_gather(parts, obj):   # one rank's shard only: the other is missing
        parts[0] = obj
        parts[1] = ([], np.zeros(0), np.zeros((0, 3)))
    import pytest
    with pytest.raises(RuntimeError):
        gather_ensemble([0], [1.0], np.zeros((2, 3)), [2, 3], fake_all_gather, 2)
