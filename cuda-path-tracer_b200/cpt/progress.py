"""Checkpoint and resume of progressive rendering.

The reference keeps its progressive state in the GL accumulation texture and the
frame counter m_localFrameNumber (cuda_path_tracer.h:39, advanced at
cuda_path_tracer.cu:461) and loses both when the application exits. Here that state
is the accumulator (the bytes `cpt_render` accumulates into, in one of the
CPT_ACCUM_* layouts, one per camera) plus the index of the next frame. The random
stream is counter-based (Philox keyed by the seed, counted by frame and pixel), so
saving after frames [0, k), loading and rendering frames [k, m) leaves the same
accumulator bytes as rendering [0, m) in one go — provided the parameters that pick
the samples and how they are summed are the same. `save` records those parameters
and `load` refuses a checkpoint whose parameters differ from the caller's.

File format: a NumPy .npz holding `accum` (uint8, the accumulator bytes) and `meta`
(a JSON string: format version, next frame, samples accumulated, and the parameter
fields in STREAM_FIELDS). Written to a temporary name and renamed, so a crash while
saving leaves the previous checkpoint intact.

The `cpt_tracer` object keeps its accumulator inside; `Tracer.get_progress` /
`Tracer.set_progress` (cpt_tracer_get_progress / cpt_tracer_set_progress) move it and
the frame counter, and `save` / `load` store them like any other accumulator.

What is not covered: a radiance cache's optimizer state (its weights can be read and
set with cpt_rc_get_weights / cpt_rc_set_weights, its Adam moments cannot), so a
cached render resumes with the same weights but not bit-identically.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass

import numpy as np

from . import ACCUM_F64, ACCUM_KAHAN, ACCUM_LERP, RenderParams, accum_bytes

FORMAT_VERSION = 1

# Parameters that decide which samples land in the accumulator and how they are summed.
# wave_paths, ray_sort and trace_stats are absent: they do not change the image.
STREAM_FIELDS = ("width", "height", "cameras", "accum_mode", "bounces", "indirect_intensity", "stratified",
                 "seed_lo", "seed_hi", "ref_grid", "nee")


@dataclass
class Progress:
    accum: np.ndarray   # uint8 accumulator bytes, all cameras
    next_frame: int     # frame0 of the next render call
    samples: int        # samples per pixel accumulated so far
    meta: dict


def _fields(params: RenderParams) -> dict:
    out = {}
    for f in STREAM_FIELDS:
        v = getattr(params, f)
        out[f] = float(np.float32(v)) if f == "indirect_intensity" else int(v)
    out["cameras"] = max(1, out["cameras"])
    return out


def _host_bytes(accum) -> np.ndarray:
    if hasattr(accum, "detach"):  # a torch tensor, on any device
        accum = accum.detach().contiguous().cpu().numpy()
    return np.ascontiguousarray(accum).reshape(-1).view(np.uint8)


def _expected_bytes(fields: dict) -> int:
    return accum_bytes(fields["width"], fields["height"], fields["accum_mode"]) * fields["cameras"]


def counted_samples(accum: np.ndarray, fields: dict) -> int | None:
    """Samples per pixel the accumulator itself records (the largest per-pixel count:
    pixels outside the reference grid hold none), or None for the running mean, which
    keeps no count."""
    w, h, ncam, mode = fields["width"], fields["height"], fields["cameras"], fields["accum_mode"]
    if mode == ACCUM_KAHAN:
        planes = accum.view(np.float32).reshape(ncam, 2, h * w, 4)
        return int(planes[:, 0, :, 3].max())
    if mode == ACCUM_F64:
        return int(accum.view(np.float64).reshape(ncam, h * w, 4)[:, :, 3].max())
    if mode == ACCUM_LERP:
        return None
    raise ValueError(f"unknown accumulator mode {mode}")


def save(path: str, accum, params: RenderParams, next_frame: int, samples: int | None = None) -> None:
    """Writes the progressive state after a render call: `accum` (torch tensor or NumPy
    array) as accumulated with `params`, and the frame0 the next call would use. For the
    summing accumulators the sample count is read from the accumulator and, when
    `samples` is given, must agree with it. Synchronizes (reads device memory)."""
    fields = _fields(params)
    raw = _host_bytes(accum)
    if raw.size != _expected_bytes(fields):
        raise ValueError(f"accumulator holds {raw.size} B; {fields['cameras']} camera(s) of "
                         f"{fields['width']}x{fields['height']} in mode {fields['accum_mode']} hold "
                         f"{_expected_bytes(fields)} B")
    if next_frame < 0 or next_frame >= 1 << 32:
        raise ValueError(f"next_frame {next_frame} outside [0, 2^32)")
    counted = counted_samples(raw, fields)
    if counted is not None and samples is not None and counted != samples:
        raise ValueError(f"accumulator counts {counted} samples per pixel, caller says {samples}")
    n = counted if counted is not None else samples
    if n is None:
        raise ValueError("a running-mean accumulator keeps no count: pass samples")
    meta = {"format": FORMAT_VERSION, "next_frame": int(next_frame), "samples": int(n), **fields}
    tmp = f"{path}.tmp.{os.getpid()}"
    with open(tmp, "wb") as f:
        np.savez(f, accum=raw, meta=np.array(json.dumps(meta, sort_keys=True)))
    os.replace(tmp, path)


def load(path: str, params: RenderParams | None = None) -> Progress:
    """Reads a checkpoint. With `params`, refuses (ValueError naming the field) one taken
    with different stream parameters, since resuming it would mix two renders."""
    with np.load(path, allow_pickle=False) as z:
        raw = np.array(z["accum"], np.uint8)
        meta = json.loads(str(z["meta"]))
    if meta.get("format") != FORMAT_VERSION:
        raise ValueError(f"checkpoint format {meta.get('format')}, this library reads {FORMAT_VERSION}")
    fields = {f: meta[f] for f in STREAM_FIELDS}
    if raw.size != _expected_bytes(fields):
        raise ValueError(f"checkpoint accumulator has {raw.size} B, its parameters need {_expected_bytes(fields)}")
    counted = counted_samples(raw, fields)
    if counted is not None and counted != meta["samples"]:
        raise ValueError(f"checkpoint accumulator counts {counted} samples per pixel, its record says "
                         f"{meta['samples']}")
    if params is not None:
        want = _fields(params)
        for f in STREAM_FIELDS:
            if want[f] != fields[f]:
                raise ValueError(f"checkpoint was rendered with {f} = {fields[f]}, the caller renders with {want[f]}")
    return Progress(raw, int(meta["next_frame"]), int(meta["samples"]), meta)


def resume(renderer, path: str) -> int:
    """Loads a checkpoint into a DeviceRenderer's accumulator (after checking it against
    the renderer's parameters) and returns the frame0 for its next render call."""
    import torch

    p = load(path, renderer.params)
    src = torch.from_numpy(p.accum)
    if renderer.accum.numel() != src.numel():
        raise ValueError("renderer accumulator size differs from the checkpoint's")
    renderer.accum.copy_(src.to(renderer.accum.device).view(renderer.accum.dtype).view(renderer.accum.shape))
    return p.next_frame


__all__ = ["FORMAT_VERSION", "STREAM_FIELDS", "Progress", "counted_samples", "save", "load", "resume",
           "ACCUM_KAHAN", "ACCUM_LERP", "ACCUM_F64"]
