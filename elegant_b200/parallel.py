"""Multi-GPU plumbing for the tracking engine: one process per GPU.

Ring tracking has no exchange after the RFCA fiducial, so a job is sharded
by instance (or by particle) and every rank tracks its share independently --
the role of Pelegant's scatter/gather (do_tracking.c:4736, :4964) without any
per-element communication.  The only collectives are for reporting: max of
the device times and sum of the work.

A bunch whose CSR step is spread over several GPUs needs the reference's
per-kick exchange (findGlobalMinMax.c:20-21, csbend.c:2532-2550): the engine
calls a reducer at those points (b2e_set_csr_reducer), and
`torch_csr_reducer` implements it with torch.distributed all-reduces on the
engine's stream.
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


# reducer operations (include/elegant_b200.h)
REDUCE_MIN_U64, REDUCE_MAX_U64, REDUCE_SUM_U32, REDUCE_SUM_U64 = 0, 1, 2, 3
_SIGN = -(1 << 63)


def allreduce_keys_and_counts(t, op: int, dist, group=None):
    """All-reduce of one engine buffer viewed as a tensor: uint64 keys (as
    int64 bit patterns) by MIN/MAX, uint32 counts by SUM (as int32, counts per
    bin stay below 2^31), uint64 counts by SUM (as int64).  Order-preserving
    keys are compared unsigned; flipping the top bit maps that order onto
    int64's."""
    import torch
    if op in (REDUCE_MIN_U64, REDUCE_MAX_U64):
        v = torch.bitwise_xor(t, torch.tensor(_SIGN, dtype=torch.int64, device=t.device))
        dist.all_reduce(v, op=dist.ReduceOp.MIN if op == REDUCE_MIN_U64 else dist.ReduceOp.MAX, group=group)
        t.copy_(torch.bitwise_xor(v, torch.tensor(_SIGN, dtype=torch.int64, device=t.device)))
    elif op in (REDUCE_SUM_U32, REDUCE_SUM_U64):
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    else:
        raise ValueError(f"unknown reduction {op}")


class DeviceBuffer:
    """__cuda_array_interface__ view of an engine device buffer (the caller
    orders its use on the engine's stream)."""

    def __init__(self, ptr: int, count: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False), "version": 3,
                                         "stream": None}


def torch_csr_reducer(dist, group=None):
    """Reducer for Tracker.set_csr_reducer: NCCL (or any backend on device
    tensors) all-reduces issued on the engine's stream."""
    import torch

    def reduce(op: int, ptr: int, count: int, stream: int) -> int:
        typestr = "<i4" if op == REDUCE_SUM_U32 else "<i8"
        t = torch.as_tensor(DeviceBuffer(ptr, count, typestr), device="cuda")
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            allreduce_keys_and_counts(t, op, dist, group)
        return 0

    return reduce
