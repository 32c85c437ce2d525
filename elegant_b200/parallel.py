"""Multi-GPU plumbing for the tracking engine: one process per GPU.

Ring tracking has no exchange after the RFCA fiducial, so a
job is sharded by instance (or by particle) and every rank tracks its share
independently -- the role of Pelegant's scatter/gather (do_tracking.c:4736,
:4964) without any per-element communication.  The only collectives are
for reporting: max of the device times and sum of the work.
"""
from __future__ import annotations

import numpy as np


def shard_instances(offsets: np.ndarray, rank: int, world: int):
    """Contiguous block of instances for `rank`, balanced by particle count.

    Returns (first_instance, last_instance_exclusive, particle_offsets_local).
    """
    offsets = np.asarray(offsets, dtype=np.int64)
    n_inst = len(offsets) - 1
    total = offsets[-1]
    # instance boundaries closest to equal particle shares
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        cuts.append(int(np.searchsorted(offsets, target, side="left")))
    cuts.append(n_inst)
    cuts = np.maximum.accumulate(np.clip(cuts, 0, n_inst))
    i0, i1 = int(cuts[rank]), int(cuts[rank + 1])
    local = offsets[i0:i1 + 1] - offsets[i0]
    return i0, i1, local


def reduce_timing(seconds: float, work: float, dist=None, device=None):
    """(max seconds over ranks, total work) -- the job throughput is work / seconds."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return seconds, work
    import torch

    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    w = torch.tensor([work], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return float(t.item()), float(w.item())
