"""Replica sharding across GPUs (one process per GPU).

Replicas of a titration sweep are independent Markov chains, so they shard
with no data-path collective: each rank owns a contiguous block of replicas
balanced by estimated cost (particles x trials + mesh points), runs them on
its own GPU, and the ranks only exchange their per-replica results (a few
bytes each) once at the end.  The reference has no multi-GPU path.
"""
import numpy as np


def replica_cost(n_particles, mesh):
    """Per-sweep cost estimate: N trials + one mesh rebuild per ~32 trials."""
    m = int(np.prod(mesh))
    return float(n_particles) * (1.0 + m / (32.0 * 1.0e4))


def partition(costs, world):
    """Contiguous blocks of replicas with near-equal summed cost.
    Returns a list of (start, stop) per rank; every replica is owned once."""
    costs = np.asarray(costs, np.float64)
    n = len(costs)
    if world <= 1 or n == 0:
        return [(0, n)] + [(n, n)] * max(0, world - 1)
    target = costs.sum() / world
    bounds, start, acc = [], 0, 0.0
    for i, c in enumerate(costs):
        acc += c
        if len(bounds) < world - 1 and acc >= target * (len(bounds) + 1) and n - (i + 1) >= world - 1 - len(bounds):
            bounds.append((start, i + 1))
            start = i + 1
    bounds.append((start, n))
    while len(bounds) < world:
        bounds.append((n, n))
    return bounds


def gather_results(local, world, group=None):
    """All-gather of per-replica result dicts (host objects, gloo or nccl)."""
    if world <= 1:
        return list(local)
    import torch.distributed as dist
    out = [None] * world
    dist.all_gather_object(out, list(local), group=group)
    return [r for part in out for r in part]
