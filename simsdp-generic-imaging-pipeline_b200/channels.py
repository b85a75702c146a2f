"""Spectral sharding of the imaging pipeline over GPUs (one process per GPU).

The reference parallelises over frequency channels: each channel's gridding,
FFT and degridding are independent, and a joint continuum image is formed by
gathering the per-channel residuals on one rank, cleaning there and scattering
the model back (read_ms/joint_nnode_ms/main.c:118-145, MPI Gather / Scatter).

Here every rank owns whole channels, so the visibility pass needs no
collective at all; channels are dealt out by visibility count (the C3 case
has seeded per-channel flag fractions, so counts differ by up to 2.5x).  The
one exchange step is the continuum sum of per-rank residual grids or images
(``continuum_sum_``): an all-reduce, which over NVLink/NVSwitch replaces the
reference's gather-to-rank-0.  Time is reported as the maximum over ranks.

Everything here is host logic on ``torch.distributed``; it runs with the
``nccl`` backend on GPUs and with ``gloo`` on CPU (tests).
"""
from __future__ import annotations

import heapq
from typing import Sequence

import numpy as np


def flagged_counts(num_channels: int, vis_per_channel: int, seed: int, flag_lo: float = 0.0,
                   flag_hi: float = 0.6) -> list[int]:
    """Visibility count of each channel after a seeded per-channel flag
    fraction drawn uniformly in [flag_lo, flag_hi] (the batched multi-channel
    workload: 0-60 % flagged)."""
    rng = np.random.default_rng(seed)
    frac = rng.uniform(flag_lo, flag_hi, num_channels)
    return [int(round(vis_per_channel * (1.0 - f))) for f in frac]


def assign_channels(vis_counts: Sequence[int], world: int) -> list[list[int]]:
    """Deals channels to ``world`` ranks, largest first, each to the rank with
    the fewest visibilities so far (ties to the lower rank).  Deterministic,
    so every rank computes the same assignment without communicating.  Each
    rank's list is returned in increasing channel order."""
    if world < 1:
        raise ValueError(f"world size {world} < 1")
    if any(c < 0 for c in vis_counts):
        raise ValueError("negative visibility count")
    order = sorted(range(len(vis_counts)), key=lambda ch: (-vis_counts[ch], ch))
    heap = [(0, r) for r in range(world)]
    owned: list[list[int]] = [[] for _ in range(world)]
    for ch in order:
        load, r = heapq.heappop(heap)
        owned[r].append(ch)
        heapq.heappush(heap, (load + vis_counts[ch], r))
    return [sorted(o) for o in owned]


def rank_load(vis_counts: Sequence[int], channels: Sequence[int]) -> int:
    return int(sum(vis_counts[c] for c in channels))


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of ``value`` over all ranks (a single-process run returns
    it unchanged).  Used for step times: a sharded step ends when its slowest
    rank ends."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def continuum_sum_(tensor):
    """In-place sum over ranks of a per-rank residual grid or image (the joint
    continuum residual).  The tensor must live where the backend works: on
    the rank's GPU for nccl, on the host for gloo."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(tensor, op=dist.ReduceOp.SUM)
    return tensor
