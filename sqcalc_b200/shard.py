"""Frames sharded over ranks: one process per GPU, one collective at the end.

The reference reads one trajectory in one process and accumulates frame after
frame (src/sqc_structure_factor.f90:457-470: num, the pair sums and gnum grow,
nframes counts).  Frames are independent, so here each rank takes a contiguous
block of them into its own plan (the same system on every rank), and the FP64
sums of all ranks are added once with a sum all-reduce -- in place on the
plan's device buffer over NCCL, or on host arrays over gloo -- before rank 0
normalises.  No data-path collective runs per frame.
"""
from __future__ import annotations

import numpy as np


def frame_block(nframes: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) of the frames of `rank`: contiguous blocks whose sizes differ by
    at most one, covering 0 .. nframes-1 exactly once over the ranks."""
    if world < 1 or not 0 <= rank < world or nframes < 0:
        raise ValueError("bad shard request")
    base, extra = divmod(nframes, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


class _DeviceArray:
    """__cuda_array_interface__ view of a plan's device buffer (no copy)."""

    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8",
                                         "data": (ptr, False), "version": 3}


def reduce_plan(plan, group=None) -> int:
    """Sum the plan's FP64 accumulators over the ranks of `group` in place
    (one NCCL all-reduce on the device buffer) and set the plan's frame count
    to the total; returns the total.  Every rank of the group must call it."""
    import torch
    import torch.distributed as dist

    ptr, count, nframes = plan.accumulator_view()
    buf = torch.as_tensor(_DeviceArray(ptr, count), device="cuda")
    frames = torch.tensor([float(nframes)], dtype=torch.float64, device=buf.device)
    dist.all_reduce(buf, group=group)
    dist.all_reduce(frames, group=group)
    torch.cuda.synchronize(buf.device)
    total = int(round(frames.item()))
    plan.set_frame_count(total)
    return total


def reduce_host(arrays: dict, group=None) -> dict:
    """Sum host accumulators (num, partial_num, gnum, nframes; any subset) over
    the ranks of `group` with one all-reduce of one packed FP64 buffer."""
    import torch
    import torch.distributed as dist

    keys = [k for k in ("num", "partial_num", "gnum", "nframes") if arrays.get(k) is not None]
    parts = [np.asarray(arrays[k], dtype=np.float64).reshape(-1) for k in keys]
    packed = torch.from_numpy(np.concatenate(parts))
    dist.all_reduce(packed, group=group)
    out, off = dict(arrays), 0
    flat = packed.numpy()
    for k, p in zip(keys, parts):
        v = flat[off:off + p.size].reshape(np.shape(arrays[k]))
        out[k] = int(round(float(v))) if k == "nframes" else v.copy()
        off += p.size
    return out
