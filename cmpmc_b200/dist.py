"""Multi-GPU run_events: events shard across ranks, one process per GPU.

Events are independent and seed-addressed (event i draws from Rng::for_stream(seed, i),
transport/parallel.hpp:102-109), so rank r of a world of size W owns the contiguous event
range [r * n, (r + 1) * n) and runs it on its own device with no collective inside the
transport. The data-path exchange is the merge of run_events (parallel.hpp:133-145), done
with collectives on the tensors the ranks hold (NCCL between GPUs, gloo on CPU):

  1. an all-gather of every rank's per-event hit counts, from which every rank has the
     global hit_offsets (exclusive scan in rank order);
  2. a gather of the hit records to the root in rank order (point-to-point sends into the
     root's output buffer at each rank's offset);
  3. an all-gather of the per-rank SimStats records, summed on the root in rank order
     (integer counters exactly, FP64 ledgers in rank order).

The adjoint reduces its histogram, value, gradient and their variance estimates with one
all-reduce (every primary belongs to exactly one rank, so all of them are sums). Timing is
the maximum over ranks.
"""
from __future__ import annotations

from dataclasses import replace
from typing import Callable, Optional, Sequence

import numpy as np

from . import _ffi

HIT_BYTES = 56
STATS_BYTES = 208


def first_event(rank: int, events_per_rank: int) -> int:
    return rank * events_per_rank


def sum_stats(records: Sequence[np.ndarray]) -> np.ndarray:
    """SimStats records summed in the given (rank) order."""
    stats = np.zeros((), dtype=_ffi.STATS_DTYPE)
    for r in records:
        for name in _ffi.STATS_DTYPE.names:
            stats[name] = stats[name] + r[name]
    return stats


def merge_results(parts: Sequence[dict]) -> dict:
    """Merges per-rank host results (dicts with 'hits', 'hit_offsets', 'stats' records) in
    rank order: the same result as exchange() gives on the root."""
    hits = np.concatenate([p["hits"] for p in parts]) if parts else np.zeros(0, _ffi.HIT_DTYPE)
    offs = [np.zeros(1, dtype=np.uint64)]
    base = 0
    for p in parts:
        o = np.asarray(p["hit_offsets"], dtype=np.uint64)
        offs.append(o[1:] + np.uint64(base))
        base += int(o[-1])
    return {"hits": hits, "hit_offsets": np.concatenate(offs), "stats": sum_stats([p["stats"] for p in parts])}


def exchange(hits, hit_offsets, stats, group=None, dst: int = 0) -> Optional[dict]:
    """The run_events merge across ranks on the ranks' own tensors.

    hits: uint8 tensor of this rank's SensorHit records (56 B each), hit_offsets: int64
    tensor [n_events + 1] (this rank's events), stats: uint8 tensor of its SimStats record
    (208 B); all on the device of the process group's backend (CUDA for NCCL, CPU for
    gloo). Every rank takes part in every collective. Returns, on every rank, the global
    hit_offsets (int64 tensor), and on `dst` also the hits of all ranks in rank order
    (uint8 tensor) and the summed SimStats record (numpy); other ranks get hits None."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = hits.device
    n_ev = hit_offsets.numel() - 1
    if hits.numel() % HIT_BYTES or stats.numel() != STATS_BYTES:
        raise ValueError("hits must hold whole 56-byte records and stats one 208-byte record")
    n_h = hits.numel() // HIT_BYTES
    # sizes of every rank: events and hits
    sz = torch.tensor([n_ev, n_h], dtype=torch.int64, device=dev)
    all_sz = [torch.empty_like(sz) for _ in range(world)]
    dist.all_gather(all_sz, sz, group=group)
    sizes = torch.stack(all_sz).cpu().tolist()
    n_evs, n_hs = [int(s[0]) for s in sizes], [int(s[1]) for s in sizes]
    # 1. per-event hit counts, padded to the largest rank -> global offsets on every rank
    m = max(max(n_evs), 1)
    cnt = torch.zeros(m, dtype=torch.int64, device=dev)
    if n_ev:
        cnt[:n_ev] = hit_offsets[1:] - hit_offsets[:-1]
    all_cnt = [torch.empty_like(cnt) for _ in range(world)]
    dist.all_gather(all_cnt, cnt, group=group)
    counts = torch.cat([all_cnt[r][:n_evs[r]] for r in range(world)])
    offsets = torch.zeros(counts.numel() + 1, dtype=torch.int64, device=dev)
    if counts.numel():
        offsets[1:] = torch.cumsum(counts, 0)
    # 3. SimStats records
    all_st = [torch.empty_like(stats) for _ in range(world)]
    dist.all_gather(all_st, stats, group=group)
    # 2. hits to dst, in rank order
    if rank == dst:
        out = torch.empty(sum(n_hs) * HIT_BYTES, dtype=torch.uint8, device=dev)
        base = 0
        for r in range(world):
            seg = out[base * HIT_BYTES:(base + n_hs[r]) * HIT_BYTES]
            if r == rank:
                seg.copy_(hits)
            elif n_hs[r]:
                dist.recv(seg, src=r, group=group)
            base += n_hs[r]
        recs = [t.cpu().numpy().view(_ffi.STATS_DTYPE)[0] for t in all_st]
        return {"hits": out, "hit_offsets": offsets, "stats": sum_stats(recs)}
    if n_h:
        dist.send(hits.contiguous(), dst=dst, group=group)
    return {"hits": None, "hit_offsets": offsets, "stats": None}


def exchange_result(res, group=None, dst: int = 0, device=None) -> Optional[dict]:
    """exchange() of a RunResult (host arrays), moved to `device` first (the rank's GPU for
    NCCL; None keeps them on the CPU for gloo). Returns host arrays on dst, None elsewhere."""
    import torch
    hits = torch.from_numpy(np.ascontiguousarray(res.hits).view(np.uint8).reshape(-1).copy())
    offs = torch.from_numpy(np.asarray(res.hit_offsets, dtype=np.uint64).view(np.int64).copy())
    st = torch.from_numpy(np.array(res.stats.record()).reshape(1).view(np.uint8).copy())
    if device is not None:
        hits, offs, st = hits.to(device), offs.to(device), st.to(device)
    m = exchange(hits, offs, st, group=group, dst=dst)
    if m["hits"] is None:
        return None
    return {"hits": m["hits"].cpu().numpy().view(_ffi.HIT_DTYPE),
            "hit_offsets": m["hit_offsets"].cpu().numpy().view(np.uint64), "stats": m["stats"]}


def allreduce_adjoint(res, group=None, device=None):
    """An AdjointResult summed over ranks: histogram, value, gradient and their variance
    estimates (sums over disjoint primaries) with one all-reduce; SimStats summed alongside.
    Every rank gets the global result."""
    import torch
    import torch.distributed as dist
    from .api import SimStats
    nb = len(res.hist)
    st = np.array(res.stats.record()).reshape(1)
    ints = [n for n in _ffi.STATS_DTYPE.names if _ffi.STATS_DTYPE[n].kind == "u"]
    flts = [n for n in _ffi.STATS_DTYPE.names if _ffi.STATS_DTYPE[n].kind == "f"]
    v = np.concatenate([res.hist, [res.value], res.grad, [res.value_var], res.grad_var, [res.n_primaries],
                        [float(st[n][0]) for n in flts]]).astype(np.float64)
    t = torch.from_numpy(v)
    ti = torch.from_numpy(np.array([int(st[n][0]) for n in ints], dtype=np.int64))
    if device is not None:
        t, ti = t.to(device), ti.to(device)
    dist.all_reduce(t, group=group)
    dist.all_reduce(ti, group=group)
    v, iv = t.cpu().numpy(), ti.cpu().numpy()
    rec = np.zeros((), dtype=_ffi.STATS_DTYPE)
    for k, n in enumerate(ints):
        rec[n] = iv[k]
    for k, n in enumerate(flts):
        rec[n] = v[nb + 11 + k]
    return replace(res, hist=v[:nb].copy(), value=float(v[nb]), grad=v[nb + 1:nb + 5].copy(),
                   value_var=float(v[nb + 5]), grad_var=v[nb + 6:nb + 10].copy(), n_primaries=int(v[nb + 10]),
                   stats=SimStats(rec), per_primary=None)


def gather_to_root(part: dict, group=None, device=None) -> Optional[dict]:
    """Merges every rank's host result (run_sharded's dict) on rank 0 through exchange()."""
    import torch
    hits = torch.from_numpy(np.ascontiguousarray(part["hits"]).view(np.uint8).reshape(-1).copy())
    offs = torch.from_numpy(np.asarray(part["hit_offsets"], dtype=np.uint64).view(np.int64).copy())
    st = torch.from_numpy(np.array(part["stats"]).reshape(1).view(np.uint8).copy())
    if device is not None:
        hits, offs, st = hits.to(device), offs.to(device), st.to(device)
    m = exchange(hits, offs, st, group=group)
    if m["hits"] is None:
        return None
    return {"hits": m["hits"].cpu().numpy().view(_ffi.HIT_DTYPE),
            "hit_offsets": m["hit_offsets"].cpu().numpy().view(np.uint64), "stats": m["stats"]}


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
