"""Placement of independent scenes on the ranks of a multi-GPU job.

Scenes never exchange data, so a job over N GPUs runs one process per GPU and
splits the scenes between them; no collective touches the data path. Every
rank computes the same split from the same list (no communication): longest
processing time first, each scene going to the rank with the least assigned
work so far (ties to the lower rank), with a scene's work taken as its
particle count (times its step count, when those differ).
"""
from __future__ import annotations

from typing import Sequence


def footprint_bytes(n_particles: int, precision: int) -> int:
    """Device bytes a scene of n particles holds in a batch: two particle
    buffers (23 real planes, 9 double planes, an int32 id), sort buffers, and
    its share of the grid (about one 4x4x4 block per 32 particles, with 2x
    headroom). precision: 0 FP64, 1 mixed."""
    real = 8 if precision == 0 else 4
    per_particle = 2 * (23 * real + 9 * 8 + 4) + 16 + 26 * 8 // 4
    grid = 2 * ((n_particles + 31) // 32) * 64 * 13 * real
    return n_particles * per_particle + grid + (1 << 16)


def shard(work: Sequence[float], world: int, rank: int) -> list[int]:
    """Indices (ascending) of the scenes that rank `rank` of `world` runs."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    order = sorted(range(len(work)), key=lambda i: (-work[i], i))
    load = [0.0] * world
    owner = [0] * len(work)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += work[i]
    return [i for i in range(len(work)) if owner[i] == rank]


def imbalance(work: Sequence[float], world: int) -> float:
    """Largest rank's work over the mean (1.0 is a perfect split)."""
    loads = [sum(work[i] for i in shard(work, world, r)) for r in range(world)]
    mean = sum(loads) / world
    return max(loads) / mean if mean > 0 else 1.0
