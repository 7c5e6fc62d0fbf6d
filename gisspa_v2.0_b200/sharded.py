"""One micrograph searched across ranks (norm_type=1): a contiguous range of the angle
sequence per rank and one exchange step that merges the per-window-pixel state.

The reference's GPUs only split the micrograph list (main.cu:51-90); its sweeps run every
(template, angle) pair of a micrograph on one device (SearchNorm::work, norm.cu:620-660).
Here the template-rotations of one micrograph are partitioned by angle.  Sweep 1 on each rank
accumulates partial sums S1 = sum c, S2 = sum c^2 (FP64, add_CCG_to_sum kernels.cu:681-695)
and, for top-K picking, the per-pixel max correlation with its (angle, template) index packed
in a signed 64-bit key.  One collective merges them (sum, sum, max); the normalisation
statistics (set_CCG_mean kernels.cu:697-706) then come from the complete sums on every rank:

* top-K: every rank picks from the merged state and returns the same list;
* chunk (reference picks): sweep 2 runs on each rank's angles again, and the ranks' lists
  concatenated in rank order are the single-GPU list, whose primary order is the angle
  (norm.cu:561-598).

Each rank owns a gisspa.Searcher on its own GPU with the same config and templates; the
collective is torch.distributed (NCCL between GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

from dataclasses import dataclass

import gisspa


def angle_ranges(n_angles: int, world: int) -> list[tuple[int, int]]:
    """Contiguous, balanced ranges covering [0, n_angles): sizes differ by at most one, the
    first n_angles % world ranks take the larger share; ranks beyond n_angles get (n, n)."""
    out, a = [], 0
    base, extra = divmod(n_angles, world)
    for r in range(world):
        b = a + base + (1 if r < extra else 0)
        out.append((a, b))
        a = b
    return out


@dataclass
class ShardState:
    """The state one rank exports and the collective merges (torch tensors on the rank's GPU)."""
    sum: object
    sum_sq: object
    key: object | None

    @staticmethod
    def empty(info: gisspa.ShardInfo, device):
        import torch
        n = int(info.n_pixels)
        key = torch.empty(n, dtype=torch.int64, device=device) if info.pick_mode == gisspa.PICK_TOPK else None
        return ShardState(torch.empty(n, dtype=torch.float64, device=device),
                          torch.empty(n, dtype=torch.float64, device=device), key)

    def pointers(self):
        return (self.sum.data_ptr(), self.sum_sq.data_ptr(), self.key.data_ptr() if self.key is not None else None)


def merge_state(st: ShardState, group=None):
    """The exchange step: sum the two FP64 sums, max the peak keys, over all ranks."""
    import torch.distributed as dist
    dist.all_reduce(st.sum, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(st.sum_sq, op=dist.ReduceOp.SUM, group=group)
    if st.key is not None:
        dist.all_reduce(st.key, op=dist.ReduceOp.MAX, group=group)


def shard_sweep1(searcher: gisspa.Searcher, image, ctf: gisspa.Ctf, rank: int, world: int, device):
    """Preparation and sweep 1 over this rank's angles; returns (info, angle range, exported state)."""
    info = searcher.shard_begin(image, ctf)
    rng = angle_ranges(info.n_angles, world)[rank]
    searcher.shard_sweep(1, *rng)
    st = ShardState.empty(info, device)
    searcher.shard_export(*st.pointers())
    return info, rng, st


def shard_finish(searcher: gisspa.Searcher, info: gisspa.ShardInfo, rng: tuple[int, int], st: ShardState):
    """After the merge: statistics from the complete sums, then this rank's picks."""
    searcher.shard_import(*st.pointers())
    if info.pick_mode != gisspa.PICK_TOPK:
        searcher.shard_sweep(2, *rng)
    return searcher.shard_picks()


def search_sharded(searcher: gisspa.Searcher, image, ctf: gisspa.Ctf, rank: int, world: int, device,
                   group=None):
    """The whole micrograph's picks on every rank (torch.distributed must be initialised)."""
    import numpy as np
    import torch.distributed as dist
    info, rng, st = shard_sweep1(searcher, image, ctf, rank, world, device)
    merge_state(st, group)
    picks = shard_finish(searcher, info, rng, st)
    if info.pick_mode == gisspa.PICK_TOPK:
        return picks
    parts = [None] * world
    dist.all_gather_object(parts, picks, group=group)
    return np.concatenate(parts) if parts else picks
