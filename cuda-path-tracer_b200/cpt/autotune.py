"""Wave-size and ray-sort autotuning for the wavefront renderer.

A render call traces its samples in waves, and a wave holds whole samples of every
view: clamp(wave_paths // pixels, 1, spp) samples per pixel are in flight at once
(`wave_samples` in csrc/render.cu), and the wave's queues, hits and path state take
scratch memory in proportion. Larger waves keep more rays in every launch and launch
less often; smaller waves keep the queues nearer the L2 and need less memory. Where
the balance lies depends on the mix of scenes and resolutions, so the tuner times
candidate settings on the real workload and keeps the fastest. The benchmark's
batched workload (64 scenes, one CUDA graph per frame) picks its wave this way.

    cands = candidates(pixels, spp, scratch_bytes, budget_bytes=8 << 30)
    result = tune(time_frame, cands)          # time_frame(wave_paths, ray_sort) -> ms
    cache = TuneCache(path); cache.put(key, result)

`time_frame` belongs to the caller (it renders on the GPU: one warm frame, one timed
frame, CUDA events on the launching stream); everything here is host logic.
"""
from __future__ import annotations

import json
import os
from dataclasses import asdict, dataclass, field
from typing import Callable, Iterable

MAX_WAVE_PATHS = (1 << 31) - 1  # the renderer's wave capacity limit (paths per wave)


@dataclass
class TuneResult:
    wave_paths: int
    ray_sort: int
    ms: float
    table: list = field(default_factory=list)  # every candidate: {"wave_paths", "ray_sort", "ms"}


def samples_per_wave(wave_paths: int, pixels: int, spp: int) -> int:
    """Samples per pixel one wave holds (the renderer's rule)."""
    return max(1, min(spp, wave_paths // pixels))


def candidates(pixels: int, spp: int, scratch_bytes: Callable[[int, int], int] | None = None,
               budget_bytes: int | None = None, try_sort: bool = True) -> list[tuple[int, int]]:
    """Distinct wave settings worth timing: samples per wave 1, 2, 4, ... and spp itself,
    each as wave_paths = samples x pixels, within the wave capacity and, when
    `scratch_bytes(wave_paths, ray_sort)` and a budget are given, within the budget; plus
    coherence sorting at the largest wave kept without it (when `try_sort`)."""
    if pixels <= 0 or spp <= 0:
        raise ValueError("pixels and spp must be positive")
    spws = sorted({1 << k for k in range(spp.bit_length()) if (1 << k) <= spp} | {spp})
    out = []
    for s in spws:
        wave = s * pixels
        if wave > MAX_WAVE_PATHS:
            break
        if scratch_bytes is not None and budget_bytes is not None:
            need = scratch_bytes(wave, 0)
            if not need or need > budget_bytes:
                break
        out.append((wave, 0))
    if not out:
        raise ValueError("no wave of whole samples fits the capacity or the memory budget")
    if try_sort:
        wave = out[-1][0]
        need = scratch_bytes(wave, 1) if scratch_bytes is not None else 0
        if scratch_bytes is None or budget_bytes is None or (need and need <= budget_bytes):
            out.append((wave, 1))
    return out


def tune(time_frame: Callable[[int, int], float], cands: Iterable[tuple[int, int]]) -> TuneResult:
    """Times every candidate once with `time_frame(wave_paths, ray_sort) -> ms` and returns
    the fastest (the first of equal times), with the whole table."""
    table = []
    for wave, sort in cands:
        ms = float(time_frame(int(wave), int(sort)))
        if not ms >= 0.0:
            raise ValueError(f"time_frame returned {ms} ms for wave {wave}, sort {sort}")
        table.append({"wave_paths": int(wave), "ray_sort": int(sort), "ms": round(ms, 3)})
    if not table:
        raise ValueError("no candidates to time")
    best = min(range(len(table)), key=lambda i: (table[i]["ms"], i))
    b = table[best]
    return TuneResult(b["wave_paths"], b["ray_sort"], b["ms"], table)


def workload_key(device: str, pixels: int, spp: int, bounces: int, triangles: int, nee: bool = False) -> str:
    """A cache key for one workload on one kind of GPU."""
    return f"{device}|px={pixels}|spp={spp}|b={bounces}|tri={triangles}|nee={int(nee)}"


class TuneCache:
    """Tuning results kept across runs in a JSON file, one entry per workload key.
    Writes go to a temporary name that is then renamed over the file."""

    def __init__(self, path: str):
        self.path = path
        self.entries: dict = {}
        if os.path.exists(path):
            with open(path) as f:
                self.entries = json.load(f)

    def get(self, key: str) -> TuneResult | None:
        e = self.entries.get(key)
        return None if e is None else TuneResult(**e)

    def put(self, key: str, result: TuneResult) -> None:
        self.entries[key] = asdict(result)
        tmp = f"{self.path}.tmp.{os.getpid()}"
        with open(tmp, "w") as f:
            json.dump(self.entries, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)
