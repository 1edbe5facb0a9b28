"""Multi-GPU sharding of a screened sweep.

Shell quartets are independent and write disjoint output blocks, so a sweep shards with no
data exchange: every rank builds the same plan (deterministic from the same inputs), takes the
chunks `assign_chunks` gives it, and the only collectives are a barrier around the timed region
and a max-reduction of the step time (`max_over_ranks`).
"""
from __future__ import annotations


def assign_chunks(costs, nranks: int):
    """Longest-first greedy assignment of chunks (by cost estimate) to ranks.

    Returns owner[c] for every chunk; identical on every rank for identical costs.
    """
    order = sorted(range(len(costs)), key=lambda c: (-costs[c], c))
    load = [0.0] * nranks
    owner = [0] * len(costs)
    for c in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        owner[c] = r
        load[r] += costs[c]
    return owner


def chunks_of(owner, rank: int):
    return [c for c, r in enumerate(owner) if r == rank]


def chunk_doubles_for(nintegrals: int, world: int, cap: int, per_rank: int = 16, floor: int = 1 << 22) -> int:
    """Chunk size (output doubles) for a sweep of `nintegrals` split over `world` ranks: `cap` on
    one rank (fewest launches), else small enough that every rank gets about `per_rank` chunks.
    A screened plan orders its quartets by kernel class, so a chunk holds one or a few classes and
    the flop estimate the assignment balances is off by a class-dependent factor (2-3x between
    the one-lane s/p classes and the f classes); with many chunks per class the longest-first
    assignment deals each class's chunks out over all ranks, so every rank gets a similar class
    mix and those factors cancel.  Never below `floor`."""
    if world <= 1 or nintegrals <= 0:
        return cap
    want = -(-int(nintegrals) // (per_rank * world))
    return int(min(cap, max(floor, want)))


def plan_digest(plan, world: int) -> dict:
    """What a rank needs to agree on with the others before it takes its share of a sweep: the
    plan's chunk sizes, each chunk's kernel-class segments and a hash of its quartet list, and the
    chunk assignment for `world` ranks with each rank's integral count."""
    import hashlib

    import numpy as np
    st = plan.stats
    h = hashlib.sha256()
    sizes, segs = [], []
    for c in range(st.nchunks):
        sizes.append(plan.chunk_size(c))
        cls, nq, fl = plan.segments(c)
        segs.append([tuple(int(v) for v in cl) + (int(n),) for cl, n in zip(cls, nq)])
        h.update(np.ascontiguousarray(plan.chunk_quartets(c)).tobytes())
    owner = assign_chunks([float(plan.segments(c)[2].sum()) for c in range(st.nchunks)], world)
    shard_ints = [sum(sizes[c] for c in chunks_of(owner, r)) for r in range(world)]
    return {"nquartets": int(st.nquartets), "nintegrals": int(st.nintegrals), "chunk_sizes": sizes,
            "segments": segs, "quartets_sha256": h.hexdigest(), "owner": owner, "shard_integrals": shard_ints}


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar over the default process group (the value itself when the
    group is not initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
