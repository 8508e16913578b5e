"""Molecule batches over several GPUs (one process per GPU, no collective on the data path).

Molecules of a conformer batch are independent (block-diagonal EEQ, no terms between
molecules), so one ensemble shards by molecules: every rank sets up and evaluates its own
subset with ``GFNFF.setMoleculeBatch`` and the host gathers energies and gradients in
ensemble order (``gather_ensemble``; one all-gather of host objects after the evaluation).
The subsets are balanced by the per-molecule cost N^3/3 + N^2 (the EEQ factorisation
dominates small molecules; pair work grows as N^2).
"""
from __future__ import annotations

import heapq

import numpy as np


def molecule_cost(n_atoms: int) -> float:
    return n_atoms ** 3 / 3.0 + n_atoms ** 2


def shard_by_cost(sizes, nshard: int):
    """Partition molecule indices 0..len(sizes)-1 into ``nshard`` lists of similar total cost.

    Longest-processing-time greedy: molecules in decreasing cost (ties by index) go to the
    currently cheapest shard (ties by shard number), so every rank computes the same
    partition from the same sizes.  Each shard's indices are returned in increasing order.
    """
    if nshard < 1:
        raise ValueError("nshard must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-molecule_cost(sizes[i]), i))
    heap = [(0.0, r) for r in range(nshard)]
    shards = [[] for _ in range(nshard)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + molecule_cost(sizes[i]), r))
    return [sorted(s) for s in shards]


def shard_costs(sizes, shards):
    return [sum(molecule_cost(sizes[i]) for i in s) for s in shards]


def gather_ensemble(idx, energies, grad, sizes, all_gather_object, world: int):
    """Energies and gradients of one ensemble evaluated in shards, in ensemble order.

    idx: ensemble indices of this rank's molecules, in the order they were evaluated;
    energies: one per molecule of this rank; grad: their gradients concatenated (sum of
    their atom counts x 3); sizes: atom counts of the whole ensemble;
    all_gather_object: ``torch.distributed.all_gather_object`` (or a stand-in with its
    signature).  Every rank receives the whole ensemble: (energies[n_mol], grad[n_atoms x 3]).
    """
    parts = [None] * world
    all_gather_object(parts, (list(map(int, idx)), np.asarray(energies, dtype=np.float64),
                              np.asarray(grad, dtype=np.float64).reshape(-1, 3)))
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    E = np.full(len(sizes), np.nan)
    G = np.full((int(off[-1]), 3), np.nan)
    for ids, e, g in parts:
        a = 0
        for k, m in enumerate(ids):
            E[m] = e[k]
            G[off[m]:off[m + 1]] = g[a:a + sizes[m]]
            a += sizes[m]
    if np.isnan(E).any():
        raise RuntimeError("gather_ensemble: the shards do not cover the ensemble")
    return E, G
