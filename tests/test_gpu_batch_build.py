"""cpt_lbvh_build_batch: many scenes built by one launch sequence (one Morton launch,
one sort over all scenes with a scene-id digit, one topology launch, one refit
launch). Every scene's arrays must equal the oracle's single build of that scene bit
for bit — keys, sorted triangles, children, both parent arrays, boxes — and the
single GPU build's traversal records; in-place scenes, tie-heavy keys, two-triangle
scenes, both key widths, a second build over the same objects, and a CUDA-graph
replay are covered."""
import numpy as np
import pytest
import torch

import cpt
from conftest import quantized
from cpt.device import DeviceLbvh, LbvhBatch, to_device
from oracle import cpu
from test_gpu_build import assert_same_as

pytestmark = pytest.mark.gpu


def scenes(seed):
    g = np.random.default_rng(seed)
    out = [cpt.scene_random(2, seed=1)[0][:2].copy(),              # the smallest scene
           quantized(cpt.scene_random(40_000, seed=2)[0], 1.0 / 32),  # tie-heavy keys
           cpt.scene_sphere_hairball(128, 64, 9_000, seed=3)[0]]
    for k in range(9):
        out.append(cpt.scene_random(int(g.integers(500, 60_000)), seed=10 + k)[0])
    return out


@pytest.mark.parametrize("bits", [30, 63])
def test_batch_equals_oracle_per_scene(cuda, bits):
    soups = scenes(5)
    lbs = [DeviceLbvh(len(t), bits) for t in soups]
    batch = LbvhBatch(lbs)
    boxes = np.stack([cpu.enclosing_box(t) for t in soups])
    src = [to_device(t) for t in soups]
    # scene 3 in place: its input is its own output array
    torch.cuda.synchronize()
    lbs[3].mem[: src[3].numel()].copy_(src[3])
    ins = list(src)
    ins[3] = lbs[3].bvh.tris
    for rep in range(2):  # a second build over the same objects gives the same arrays
        if rep:
            torch.cuda.synchronize()
            lbs[3].mem[: src[3].numel()].copy_(src[3])
        batch.build(ins, boxes, check_root=True)
        torch.cuda.synchronize()
        for t, lb, box in zip(soups, lbs, boxes):
            out = lb.download()
            assert_same_as(out, cpu.build(t, bits, box=box))
            single = DeviceLbvh(len(t), bits)
            single.build(to_device(t), box=box, check_root=True)
            assert out["nodes"].tobytes() == single.download()["nodes"].tobytes()


def test_batch_replays_in_a_cuda_graph(cuda):
    soups = scenes(6)[:6]
    lbs = [DeviceLbvh(len(t), 63) for t in soups]
    batch = LbvhBatch(lbs)
    boxes = np.stack([cpu.enclosing_box(t) for t in soups])
    src = [to_device(t) for t in soups]
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        batch.build(src, boxes)
    torch.cuda.synchronize()
    for lb in lbs:  # clear the outputs, then rebuild them by replaying the captured call
        lb.mem.zero_()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        batch.build(src, boxes)
    for lb in lbs:
        lb.mem.zero_()
    g.replay()
    torch.cuda.synchronize()
    for t, lb, box in zip(soups, lbs, boxes):
        lb.status()
        assert_same_as(lb.download(), cpu.build(t, 63, box=box))


def test_batch_argument_checks(cuda):
    soups = scenes(7)[:3]
    lbs = [DeviceLbvh(len(t), 30) for t in soups]
    with pytest.raises(ValueError):
        LbvhBatch([DeviceLbvh(10, 30), DeviceLbvh(10, 63)])
    n = (cpt.ctypes.c_uint32 * 1)(1)
    assert cpt.lib.cpt_lbvh_batch_scratch_bytes(n, 1, 30) == 0  # a scene of one triangle
    assert cpt.lib.cpt_lbvh_batch_scratch_bytes(n, 0, 30) == 0
    batch = LbvhBatch(lbs)
    with pytest.raises(cpt.CptError) as e:  # no boxes
        cpt.check(cpt.lib.cpt_lbvh_build_batch(None, batch.n, 3, None, 30, batch.bvh_ptrs, batch.scratch.data_ptr(),
                                               batch.scratch_bytes, 0, None), "batch")
    assert e.value.code == cpt.ERR_INVALID_ARGUMENT
