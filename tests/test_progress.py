"""Checkpoint / resume of progressive rendering (cpt/progress.py), on the CPU.

The resume property is checked on the oracle's integrator, which the device renderer
matches bit for bit: frames [0, 2) accumulated, saved, loaded, then frames [2, 4)
rendered by a second call and accumulated onto the loaded state give the bytes of
frames [0, 4) in one go, for the Kahan and the running-mean accumulators. The rest
checks the file: round trips, and the refusals (other stream parameters, a wrong
size, a count that disagrees, an unknown format)."""
import json
import os

import numpy as np
import pytest

import cpt
from cpt import progress
from cpt.device import make_params
from oracle import cpu

W, H = 16, 12


@pytest.fixture(scope="module")
def scene():
    tris, infos = cpt.scene_random(2000, seed=21)
    b = cpu.build(tris, 30)
    cam = cpt.camera_look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.0), aspect=W / H)
    return b, infos, cpu.ocam_from(cam.eye, cam.as_array()[3:])


def samples(scene, spp, frame0, seed=5):
    b, infos, ocam = scene
    rad, _ = cpu.render(b, infos, None, W, H, spp, frame0, 3, 3.0, True, seed, ocam)
    return rad


def kahan_bytes(s, c, n):
    """The device's Kahan layout: a plane of float4 sums (w = samples), then a plane of
    float4 compensations (w = 0)."""
    out = np.zeros((2, H, W, 4), np.float32)
    out[0, ..., :3], out[0, ..., 3] = s, n
    out[1, ..., :3] = c
    return out.view(np.uint8).reshape(-1)


def from_kahan_bytes(raw):
    a = raw.view(np.float32).reshape(2, H, W, 4)
    return a[0, ..., :3], a[1, ..., :3], a[0, 0, 0, 3]


def test_counter_based_stream_splits_by_frame(scene):
    # the property resume rests on: samples of frames [2, 4) do not depend on the call
    assert samples(scene, 2, 2).tobytes() == samples(scene, 4, 0)[2:].tobytes()


def test_kahan_resume_is_bit_identical(scene, tmp_path):
    p = make_params(W, H, 2, 0, 3, 3.0, True, 5, cpt.ACCUM_KAHAN)
    first = cpu.accumulate_kahan(samples(scene, 2, 0))
    path = str(tmp_path / "progress.npz")
    progress.save(path, kahan_bytes(*first), p, next_frame=2)
    assert os.listdir(tmp_path) == ["progress.npz"]  # written whole, no temporary left
    loaded = progress.load(path, p)
    assert (loaded.next_frame, loaded.samples) == (2, 2)
    resumed = cpu.accumulate_kahan(samples(scene, 2, loaded.next_frame), init=from_kahan_bytes(loaded.accum))
    straight = cpu.accumulate_kahan(samples(scene, 4, 0))
    assert kahan_bytes(*resumed).tobytes() == kahan_bytes(*straight).tobytes()


def test_running_mean_resume_is_bit_identical(scene, tmp_path):
    p = make_params(W, H, 2, 0, 3, 3.0, True, 5, cpt.ACCUM_LERP)
    img = cpu.accumulate_lerp(samples(scene, 2, 0), 0)
    acc = np.zeros((H, W, 4), np.float32)
    acc[..., :3], acc[..., 3] = img, 1.0
    path = str(tmp_path / "lerp.npz")
    with pytest.raises(ValueError, match="keeps no count"):
        progress.save(path, acc, p, next_frame=2)
    progress.save(path, acc, p, next_frame=2, samples=2)
    loaded = progress.load(path, p)
    prev = loaded.accum.view(np.float32).reshape(H, W, 4)[..., :3]
    resumed = cpu.accumulate_lerp(samples(scene, 2, loaded.next_frame), loaded.next_frame, prev=prev)
    straight = cpu.accumulate_lerp(samples(scene, 4, 0), 0)
    assert resumed.tobytes() == straight.tobytes()


def test_f64_count_and_cameras(tmp_path):
    p = make_params(W, H, 1, 0, 3, 3.0, True, 5, cpt.ACCUM_F64, cameras=3)
    acc = np.zeros((3, H * W, 4), np.float64)
    acc[..., 3] = 7.0
    acc[1, :5, 3] = 0.0  # pixels outside the reference grid hold no samples
    path = str(tmp_path / "f64.npz")
    progress.save(path, acc, p, next_frame=7, samples=7)
    assert progress.load(path, p).samples == 7
    with pytest.raises(ValueError, match="counts 7"):
        progress.save(path, acc, p, next_frame=7, samples=6)


def test_refusals(tmp_path):
    p = make_params(W, H, 2, 0, 3, 3.0, True, 5, cpt.ACCUM_KAHAN)
    acc = np.zeros((2, H, W, 4), np.float32)
    acc[0, ..., 3] = 2.0
    path = str(tmp_path / "k.npz")
    progress.save(path, acc, p, next_frame=2)
    for changed, field in ((make_params(W, H, 2, 0, 3, 3.0, True, 6, cpt.ACCUM_KAHAN), "seed_lo"),
                           (make_params(W, H, 2, 0, 3, 3.0, True, 5 + (1 << 32), cpt.ACCUM_KAHAN), "seed_hi"),
                           (make_params(W + 8, H, 2, 0, 3, 3.0, True, 5, cpt.ACCUM_KAHAN), "width"),
                           (make_params(W, H, 2, 0, 4, 3.0, True, 5, cpt.ACCUM_KAHAN), "bounces"),
                           (make_params(W, H, 2, 0, 3, 2.5, True, 5, cpt.ACCUM_KAHAN), "indirect_intensity"),
                           (make_params(W, H, 2, 0, 3, 3.0, False, 5, cpt.ACCUM_KAHAN), "stratified"),
                           (make_params(W, H, 2, 0, 3, 3.0, True, 5, cpt.ACCUM_KAHAN, nee=True), "nee")):
        with pytest.raises(ValueError, match=field):
            progress.load(path, changed)
    # parameters that leave the image unchanged do not block a resume
    assert progress.load(path, make_params(W, H, 8, 0, 3, 3.0, True, 5, cpt.ACCUM_KAHAN, wave_paths=4096,
                                           ray_sort=True)).next_frame == 2
    with pytest.raises(ValueError, match="holds"):
        progress.save(path, acc[:, :-1], p, next_frame=2)
    with pytest.raises(ValueError, match="next_frame"):
        progress.save(path, acc, p, next_frame=-1)
    # a record that disagrees with its accumulator, and an unknown format
    with np.load(path) as z:
        raw, meta = np.array(z["accum"]), json.loads(str(z["meta"]))
    for key, value, message in (("samples", 3, "counts 2"), ("format", 99, "format")):
        bad = dict(meta, **{key: value})
        np.savez(str(tmp_path / "bad.npz"), accum=raw, meta=np.array(json.dumps(bad)))
        with pytest.raises(ValueError, match=message):
            progress.load(str(tmp_path / "bad.npz"))


def test_resume_fills_a_renderer_accumulator(tmp_path):
    # resume() on anything with `params` and a uint8 `accum` tensor: a CPU tensor here
    import types

    import torch

    p = make_params(W, H, 2, 0, 3, 3.0, True, 5, cpt.ACCUM_KAHAN)
    acc = np.zeros((2, H, W, 4), np.float32)
    acc[0, ..., :3] = np.random.default_rng(0).random((H, W, 3), np.float32)
    acc[0, ..., 3] = 2.0
    path = str(tmp_path / "k.npz")
    progress.save(path, torch.from_numpy(acc.view(np.uint8).reshape(-1).copy()), p, next_frame=2)
    r = types.SimpleNamespace(params=p, accum=torch.zeros(acc.nbytes, dtype=torch.uint8))
    assert progress.resume(r, path) == 2
    assert r.accum.numpy().tobytes() == acc.tobytes()
    small = types.SimpleNamespace(params=make_params(W, H - 1, 2, 0, 3, 3.0, True, 5, cpt.ACCUM_KAHAN),
                                  accum=torch.zeros(8, dtype=torch.uint8))
    with pytest.raises(ValueError, match="height"):
        progress.resume(small, path)
