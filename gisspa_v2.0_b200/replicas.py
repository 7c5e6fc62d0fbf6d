"""Replica scheduling of micrographs over devices / ranks (the reference's multi-GPU mode).

The reference splits micrographs [first, last) into contiguous intervals, one per device
(work_intervals, helper.cu:23-33), searches them independently and concatenates the
per-device pick lists in device order (main.cu:51-90).  Micrographs never exchange data,
so there is no collective on the data path; with torch.distributed the only
communication is gathering the finished pick lists on rank 0.
"""
from __future__ import annotations


def work_intervals(first: int, last: int, n: int) -> list[tuple[int, int]]:
    """Contiguous intervals of round((last - first) / n) micrographs (at least 1); the last
    interval absorbs the remainder (helper.cu:23-33)."""
    out = []
    total = float(last - first)
    per = max(int(_round_half_away(total / n)), 1)
    i = 0
    while i < n and first < last:
        out.append((first, min(first + per, last)))
        first += per
        i += 1
    if out:
        out[-1] = (out[-1][0], last)
    return out


def _round_half_away(x: float) -> float:
    # std::round semantics (half away from zero)
    import math
    return math.floor(x + 0.5) if x >= 0 else math.ceil(x - 0.5)


def run_replicas(search, first: int, last: int, rank: int, world: int, gather=None):
    """Search this rank's interval with `search(i) -> list`, then (optionally) gather every
    rank's results on all ranks with `gather(obj) -> list_of_objs_in_rank_order`; returns the
    concatenation in micrograph order (device order, as main.cu:87-89)."""
    iv = work_intervals(first, last, world)
    mine = []
    if rank < len(iv):
        a, b = iv[rank]
        mine = [search(i) for i in range(a, b)]
    if gather is None:
        return mine
    parts = gather(mine)
    return [x for part in parts for x in part]
