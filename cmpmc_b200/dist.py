"""Multi-GPU run_events: events shard across ranks, one process per GPU.

Events are independent and seed-addressed (event i draws from Rng::for_stream(seed, i),
transport/parallel.hpp:102-109), so rank r of a world of size W owns the contiguous event
range [r * n, (r + 1) * n) and runs it on its own device with no collective on the data
path. The only exchange is the merge of the per-rank results on rank 0, in rank order:
hit counts -> global hit_offsets, hit records concatenated, SimStats summed (integer
counters exactly; FP64 ledgers in rank order), as run_events merges its chunks
(parallel.hpp:133-145). Timing is the maximum over ranks.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence

import numpy as np

from . import _ffi


def first_event(rank: int, events_per_rank: int) -> int:
    return rank * events_per_rank


def merge_results(parts: Sequence[dict]) -> dict:
    """Merges per-rank results (dicts with 'hits', 'hit_offsets', 'stats' records) in rank order."""
    hits = np.concatenate([p["hits"] for p in parts]) if parts else np.zeros(0, _ffi.HIT_DTYPE)
    offs = [np.zeros(1, dtype=np.uint64)]
    base = 0
    for p in parts:
        o = np.asarray(p["hit_offsets"], dtype=np.uint64)
        offs.append(o[1:] + np.uint64(base))
        base += int(o[-1])
    stats = np.zeros((), dtype=_ffi.STATS_DTYPE)
    for p in parts:
        for name in _ffi.STATS_DTYPE.names:
            stats[name] = stats[name] + p["stats"][name]
    return {"hits": hits, "hit_offsets": np.concatenate(offs), "stats": stats}


def gather_to_root(part: dict, group=None) -> Optional[dict]:
    """Gathers every rank's result on rank 0 and merges them there (None on other ranks)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    objs = [None] * world if dist.get_rank(group) == 0 else None
    dist.gather_object(part, objs, dst=0, group=group)
    if dist.get_rank(group) != 0:
        return None
    return merge_results(objs)


def max_over_ranks(x: float, group=None, device=None) -> float:
    """Maximum of a per-rank time over the process group."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def run_sharded(engine, workload, events_per_rank: int, options, rank: int,
                runner: Optional[Callable] = None) -> dict:
    """Generates and transports this rank's event range; returns its result as a dict.

    `runner(packed, options)` transports the packed events (default: the device run of
    `engine`); it returns a RunResult."""
    fe = first_event(rank, events_per_rank)
    packed = engine.generate(workload, events_per_rank, options.seed, first_event=fe)
    res = (runner or engine.run_packed)(packed, options)
    return {"hits": res.hits, "hit_offsets": res.hit_offsets, "stats": res.stats.record(), "first_event": fe}
