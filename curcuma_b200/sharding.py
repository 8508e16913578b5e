"""Molecule batches over several GPUs (one process per GPU, no collective on the data path).

Molecules of a conformer batch are independent (block-diagonal EEQ, no terms between
molecules), so a batch shards by molecules: every rank sets up and evaluates its own subset
with ``GFNFF.setMoleculeBatch`` and the host gathers energies and gradients.  The subsets are
balanced by the per-molecule cost N^3/3 + N^2 (the EEQ factorisation dominates small
molecules; pair work grows as N^2).
"""
from __future__ import annotations

import heapq


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
