"""Sharding independent scenes of a batch across GPUs (one process per GPU).

Scenes of a batch share nothing, so a multi-GPU batch is a partition of the scenes: each rank
creates a BatchDOM of its own scenes and updates it with no collective on the data path. The
partition balances an estimated per-frame cost (longest-processing-time first, deterministic,
so every rank computes the same partition without communicating).

Cost model of one steady frame of a scene (units: bytes-or-evaluations, proportional terms):
particle stages ~ 300 B per persistent particle + 100 B per birth + 60 B per cell (the per-frame
algorithmic bytes of the particle and cell stages), evidence ~ in-support kernel evaluations =
points x (in-grid ray length / res) x pi (ls / res)^2 cells per unit length, weighted by the
measured cost ratio of one evaluation to one HBM byte.
"""
from __future__ import annotations

import math

# one in-support evaluation costs about as much time as this many bytes of HBM traffic
# (k_bgki: ~1e8 evaluations/ms; particle stages: ~1.5e9 bytes/ms)
EVAL_BYTES = 15.0


def scene_cost(params, n_points: int) -> float:
    """Estimated cost of one steady frame of a scene (params: k3dom_params or a dict)."""
    get = (lambda k: params[k]) if isinstance(params, dict) else (lambda k: getattr(params, k))
    res = float(get("resolution"))
    G = int(float(get("size")) / res)
    Gz = int(float(get("size_z")) / res)
    C = G * G * Gz
    P = int(get("particle_count"))
    B = int(get("new_born_particle_count"))
    ls = float(get("ls"))
    ray_cells = min(G * math.sqrt(2.0) / 2.0 + Gz, G)  # in-grid length of a ray from the centre [cells]
    evals = n_points * ray_cells * math.pi * (ls / res) ** 2
    return 300.0 * P + 100.0 * B + 60.0 * C + EVAL_BYTES * evals


def partition(costs, n_ranks: int) -> list[list[int]]:
    """Scenes -> ranks, longest-processing-time first: scenes in decreasing cost (ties by index)
    each go to the currently least-loaded rank (ties by rank). Every rank gets its scenes in
    increasing index order. Deterministic: every rank computes the same result."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * n_ranks
    out: list[list[int]] = [[] for _ in range(n_ranks)]
    for i in order:
        r = min(range(n_ranks), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += float(costs[i])
    return [sorted(x) for x in out]


def my_scenes(costs, rank: int, world: int) -> list[int]:
    return partition(costs, world)[rank]
