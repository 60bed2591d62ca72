"""Wave-size, ray-sort and traversal launch-shape autotuning for the wavefront renderer.

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
    shape = tune(time_frame4, launch_candidates(result))  # time_frame4(wave, sort, refill, blocks)
    cache = TuneCache(path); cache.put(key, shape)

The second stage tunes the persistent traversal's launch shape at the chosen wave:
the refill threshold (a warp takes new rays once fewer than `refill_lanes` of its
lanes still trace: fewer idle lanes against more refill bookkeeping) and the resident
traversal blocks per SM (`traverse_blocks_per_sm`: fewer resident warps keep more of
each warp's nodes in L1 and L2, more hide more latency). Both are
cpt_render_params fields and leave the image unchanged.

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
    table: list = field(default_factory=list)  # every candidate: {"wave_paths", "ray_sort", ..., "ms"}
    refill_lanes: int = 0  # 0: the renderer's default
    blocks_per_sm: int = 0  # 0: the traversal's occupancy
    wave_lanes: int = 0  # 0: the renderer's default (one lane)


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


_FIELDS = ("wave_paths", "ray_sort", "refill_lanes", "blocks_per_sm", "wave_lanes")


def launch_candidates(base: TuneResult, refills: Iterable[int] = (0, 32, 28, 24, 16),
                      blocks: Iterable[int] = (0, 6, 4),
                      lanes: Iterable[int] = (2,)) -> list[tuple[int, int, int, int, int]]:
    """(wave_paths, ray_sort, refill_lanes, blocks_per_sm, wave_lanes) candidates at the
    wave and sort of `base`: every refill threshold at full occupancy, every smaller block
    count at the default threshold, then every other lane count at the default shape
    (0 = the renderer's default in each)."""
    out = [(base.wave_paths, base.ray_sort, int(r), 0, 0) for r in refills]
    out += [(base.wave_paths, base.ray_sort, 0, int(b), 0) for b in blocks if int(b)]
    out += [(base.wave_paths, base.ray_sort, 0, 0, int(n)) for n in lanes if int(n)]
    for r, b, n in ((c[2], c[3], c[4]) for c in out):
        if not (0 <= r <= 32 and 0 <= b and 0 <= n <= 2):
            raise ValueError(f"bad launch candidate: refill {r}, blocks {b}, lanes {n}")
    seen, uniq = set(), []
    for c in out:
        if c not in seen:
            seen.add(c)
            uniq.append(c)
    return uniq


def tune(time_frame: Callable[..., float], cands: Iterable[tuple]) -> TuneResult:
    """Times every candidate once and returns the fastest (the first of equal times),
    with the whole table. A candidate is (wave_paths, ray_sort), (wave_paths, ray_sort,
    refill_lanes, blocks_per_sm) or that and wave_lanes; `time_frame` is called with the
    candidate's values (two, four or five arguments) and returns milliseconds."""
    table = []
    for cand in cands:
        cand = tuple(int(x) for x in cand)
        if len(cand) not in (2, 4, 5):
            raise ValueError(f"a candidate has 2, 4 or 5 values, not {cand}")
        ms = float(time_frame(*cand))
        if not ms >= 0.0:
            raise ValueError(f"time_frame returned {ms} ms for candidate {cand}")
        row = dict(zip(_FIELDS, cand))
        row["ms"] = round(ms, 3)
        table.append(row)
    if not table:
        raise ValueError("no candidates to time")
    best = min(range(len(table)), key=lambda i: (table[i]["ms"], i))
    b = table[best]
    return TuneResult(b["wave_paths"], b["ray_sort"], b["ms"], table, b.get("refill_lanes", 0),
                      b.get("blocks_per_sm", 0), b.get("wave_lanes", 0))


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
