"""Multi-GPU: one process per GPU, spectra sharded across ranks.

The jerk search has no data-path exchange: spectra (and, for one very long
spectrum, rstep ranges) are independent, and the kernel bank is replicated.
Ranks only agree on timing (the max over ranks) and, for a job that wants
one list of results, hand their results to rank 0 -- the host merge: whole
spectra's candidate lists unchanged, or, for one spectrum split by rstep
ranges, the raw hits, which rank 0 sorts into the reference's insertion
order and inserts (jerk_merge_hits).  Everything here is torch.distributed
plumbing that works with the "nccl" backend on GPUs and "gloo" on CPUs.
"""

from __future__ import annotations

import os
from dataclasses import dataclass
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np


@dataclass(frozen=True)
class RankEnv:
    rank: int
    world: int
    local: int


def rank_env() -> RankEnv:
    return RankEnv(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                   int(os.environ.get("LOCAL_RANK", "0")))


def shard(items: Sequence, rank: int, world: int) -> List:
    """Round-robin share of a job's spectra for one rank (every item exactly
    once over all ranks)."""
    return [x for i, x in enumerate(items) if i % world == rank]


def contiguous_ranges(n: int, world: int) -> List[Tuple[int, int]]:
    """(first, count) ranges covering 0..n-1, one per rank, sizes differing by
    at most one."""
    base, extra = divmod(n, world)
    out, first = [], 0
    for r in range(world):
        k = base + (1 if r < extra else 0)
        out.append((first, k))
        first += k
    return out


def rstep_ranges(nrsteps: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous (first, count) rstep ranges covering one spectrum, one per
    rank, for a spectrum searched by several GPUs."""
    return contiguous_ranges(nrsteps, world)


def dm_ranges(numdms: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous (first, count) DM-trial ranges, one per rank, for subband
    dedispersion over several GPUs: each rank builds its dedisperser from its
    rows of the offsets table and reads the same subband blocks.  Contiguous
    rows keep neighbouring DMs, whose windows overlap, in one rank's groups.
    With more ranks than DMs the last ranks get count 0: such a rank has no
    trials and must not build a dedisperser (jerk_dedisperser_create rejects
    zero rows); it only takes part in the collectives."""
    return contiguous_ranges(numdms, world)


def max_over_ranks(value: float, dist=None, device: Optional[str] = None) -> float:
    """The largest value over ranks (a job's time is its slowest rank's)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(local: Dict[int, list], dist=None) -> Optional[Dict[int, list]]:
    """Per-spectrum results of all ranks on rank 0 (None elsewhere).  Keys are
    global spectrum ids; a rank's lists are merged unchanged (each spectrum is
    searched by exactly one rank, so nothing needs re-ordering)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(local)
    world = dist.get_world_size()
    parts = [None] * world if dist.get_rank() == 0 else None
    dist.gather_object(local, parts, dst=0)
    if dist.get_rank() != 0:
        return None
    merged: Dict[int, list] = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise ValueError(f"spectrum {k} searched by two ranks")
            merged[k] = v
    return merged


def _rank_world(dist) -> Tuple[int, int]:
    if dist is None or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(), dist.get_world_size()


def split_search(search: Callable[[int, int], Tuple[np.ndarray, np.ndarray]], obs,
                 fundamental, first: int, count: int, dist=None) -> Optional[np.ndarray]:
    """One spectrum searched by all ranks: rank r takes the r-th contiguous
    share of rsteps [first, first + count) and calls search(first_r, count_r),
    which returns that range's raw hits (keys, powers) -- for a plan,
    ``lambda f, n: plan.search(spec, f, n, want_hits=True)[1:]``.  Rank 0
    gathers every rank's hits and merges them in the reference's insertion
    order (sort by key, then the ordered insertion: jerk_merge_hits), so its
    list equals a one-rank search of the whole range; the others get None.
    A rank whose share is empty searches nothing."""
    from . import jerk

    rank, world = _rank_world(dist)
    f, n = rstep_ranges(count, world)[rank]
    if n:
        k, p = search(first + f, n)
    else:
        k, p = np.zeros(0, np.uint64), np.zeros(0, np.float32)
    part = (np.ascontiguousarray(k, dtype=np.uint64), np.ascontiguousarray(p, dtype=np.float32))
    if world == 1:
        parts = [part]
    else:
        parts = [None] * world if rank == 0 else None
        dist.gather_object(part, parts, dst=0)
        if rank != 0:
            return None
    keys = np.concatenate([q[0] for q in parts])
    pows = np.concatenate([q[1] for q in parts])
    if len(np.unique(keys)) != len(keys):
        raise ValueError("two ranks reported the same hit: overlapping rstep ranges")
    return jerk.merge_hits(obs, fundamental, keys, pows)
