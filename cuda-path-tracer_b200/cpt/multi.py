"""Multi-GPU plumbing for progressive rendering: one process per GPU.

The path shards by samples: every rank holds its own replica of the scene and its
BVH (the build is cheaper than moving it: 2 ms for 5.2 M triangles), renders a
disjoint range of the random stream into its own accumulator, and once per frame the
accumulators meet in one reduction into a display accumulator on rank 0 — the single
exchange step of the path (NCCL over NVLink between GPUs; gloo on CPU in the tests).
Each rank's accumulator stays its own (it keeps accumulating its later frames), so no
sample is counted twice. A Kahan accumulator is resolved on each rank before the sum:
the rank's compensated value (sum - compensation) goes into the reduction and the
display accumulator's compensation plane is zero, so the reduced image carries the
per-rank compensated sums, added in plain FP32 across ranks.

Batches of independent scenes shard by scene instead: `assign_by_cost` gives each
rank a set of whole scenes (its own BVHs, images and accumulators, no exchange).
"""
from __future__ import annotations

RANK_STREAM_STRIDE = 1 << 24  # sample indices reserved per rank: disjoint Philox streams
ACCUM_KAHAN, ACCUM_LERP, ACCUM_F64 = 0, 1, 2  # cpt_render_params.accum_mode


def rank_frame0(frame: int, rank: int) -> int:
    """Global sample index at which `rank` renders progressive sample `frame`."""
    if frame < 0 or frame >= RANK_STREAM_STRIDE:
        raise ValueError("frame outside the per-rank sample range")
    return rank * RANK_STREAM_STRIDE + frame


def reduce_accumulator(accum, out, dst: int = 0, mode: int = ACCUM_KAHAN, group=None) -> None:
    """Sum of the ranks' accumulators into `out` on rank `dst` (`out`: a buffer of the
    accumulator's size on every rank; `accum` is left as it is).

    Kahan (float4 sum plane, then float4 compensation plane): each rank contributes
    sum - compensation (sample counts in w add up) and `out`'s compensation plane is 0.
    FP64 (double4 sums): plain sum. Running mean (float4, the reference's lerp): the
    mean of the ranks' images (every rank renders the same number of samples)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    if mode == ACCUM_KAHAN:
        a = accum.view(torch.float32).view(2, -1)
        o = out.view(torch.float32).view(2, -1)
        torch.sub(a[0], a[1], out=o[0])
        o[1].zero_()
        t = o
    elif mode == ACCUM_F64:
        t = out.view(torch.float64)
        t.copy_(accum.view(torch.float64))
    elif mode == ACCUM_LERP:
        t = out.view(torch.float32)
        torch.div(accum.view(torch.float32), float(world), out=t)
    else:
        raise ValueError(f"unknown accumulator mode {mode}")
    dist.reduce(t, dst=dst, op=dist.ReduceOp.SUM, group=group)


def assign_by_cost(costs, world: int) -> list[list[int]]:
    """Scenes -> ranks, longest processing time first: scenes in decreasing cost
    (ties: lower index first) each go to the rank with the least total so far (ties:
    lower rank). Deterministic, so every rank computes the same assignment; the
    largest rank total is within one scene's cost of the best possible."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += float(costs[i])
    for lst in out:
        lst.sort()
    return out


def scene_cost(pixels: int, triangles: int, hairball: bool) -> float:
    """Relative render cost of one scene of a batch: rays (pixels) times the depth
    of its tree (log2 triangles), four times more for the long-triangle hairball
    scenes (their rays visit several times more nodes)."""
    import math

    return float(pixels) * max(1.0, math.log2(max(triangles, 2))) * (4.0 if hairball else 1.0)
