"""Batched ensembles across GPUs: independent systems shard by system.

An ensemble of independent systems (the batched configuration: 256 Plummer
spheres of uneven N) needs no exchange between GPUs.  Each rank evaluates
its own share of the systems on its own GPU with fmm_evaluate_batched; the
only communication is a host-side gather of timings and statistics.  The
reference has no ensemble mode; its one multi-rank path splits a single
system's tree into coarse branches per rank
(src/system_updaters/tree_components/parallel_tree.cpp:54), which is the
same idea one level up: whole independent units per rank, balanced by work.

The share of each rank is chosen by the longest-processing-time rule:
systems in order of decreasing cost, each to the rank with the least cost so
far (ties to the lower rank), which keeps the largest load within 4/3 of
the best possible.  The cost of a system of n particles is n * log2(n),
the FMM pass's work (the tree sort dominates the growth beyond linear).
"""
import math

import numpy as np


def system_cost(n):
    """Work estimate of one force pass of n particles."""
    n = max(int(n), 1)
    return n * max(math.log2(n), 1.0)


def partition_systems(sizes, world):
    """Assigns every system to one of `world` ranks (longest processing time
    first).  Returns, per rank, the ascending list of its system indices."""
    if world < 1:
        raise ValueError("world must be >= 1")
    sizes = [int(s) for s in sizes]
    order = sorted(range(len(sizes)), key=lambda i: (-system_cost(sizes[i]), i))
    load = [0.0] * world
    share = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        share[r].append(i)
        load[r] += system_cost(sizes[i])
    return [sorted(s) for s in share]


def rank_loads(sizes, shares):
    """Total cost per rank of a partition."""
    return [sum(system_cost(sizes[i]) for i in s) for s in shares]


def gather_systems(pos, mass, offsets, systems):
    """The particles of `systems` (indices into offsets, which has one entry
    more than the ensemble has systems) stored one after another, as
    fmm_evaluate_batched takes them: (positions, masses, local offsets)."""
    offsets = np.asarray(offsets, dtype=np.int64)
    parts_p, parts_m, loc = [], [], [0]
    for s in systems:
        a, b = int(offsets[s]), int(offsets[s + 1])
        parts_p.append(pos[a:b])
        parts_m.append(mass[a:b])
        loc.append(loc[-1] + (b - a))
    dim = pos.shape[1]
    p = np.concatenate(parts_p) if parts_p else np.zeros((0, dim))
    m = np.concatenate(parts_m) if parts_m else np.zeros(0)
    return np.ascontiguousarray(p), np.ascontiguousarray(m), np.asarray(loc, dtype=np.int64)
