"""DM-sharded replicas across GPUs (one process per GPU).

DM trials are independent (the reference hands them out from a mutex
counter, src/pipeline_multi.cu:38-86, and appends the workers' candidate
lists after joining them, :531-535).  Here each rank searches its own DM
trials with its own resident series; there is no collective on the data
path, only a host-side gather of the candidate lists at the end.
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np


def dm_schedule(ndm: int, rank: int, world: int, steps: int, per_step: int,
                offset: int = 0) -> List[List[int]]:
    """DM indices of each step of `rank`: rank-interleaved blocks of
    `per_step` consecutive DM trials, wrapping over the `ndm` trials."""
    out = []
    for s in range(steps):
        base = ((offset + s) * world + rank) * per_step
        out.append([(base + j) % ndm for j in range(per_step)])
    return out


def dm_partition(ndm: int, rank: int, world: int, per_step: int) -> List[int]:
    """Every DM trial exactly once: the blocks of this rank."""
    nblocks = (ndm + per_step - 1) // per_step
    mine = []
    for b in range(rank, nblocks, world):
        mine.extend(range(b * per_step, min(ndm, (b + 1) * per_step)))
    return mine


def gather_candidates(local: np.ndarray, group=None) -> np.ndarray:
    """Concatenate every rank's candidate array on every rank, ordered by
    (dm_idx, position in the rank's list) so the result does not depend on
    the number of ranks.  Host-side (object gather); no GPU collective."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        parts = [local]
    else:
        parts = [None] * dist.get_world_size(group)
        dist.all_gather_object(parts, local, group=group)
    parts = [p for p in parts if p is not None and len(p)]
    if not parts:
        return local[:0]
    allc = np.concatenate(parts)
    order = np.argsort(allc["dm_idx"], kind="stable")
    return allc[order]
