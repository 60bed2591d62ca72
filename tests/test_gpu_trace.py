"""Closest-hit and any-hit traversal on the GPU against the oracle and the
reference's golden hits: triangle index, t and barycentrics bit-exact."""
import numpy as np
import pytest
import torch

import cpt
from conftest import GOLDEN_CASES, load_golden, rays_at
from cpt.device import DeviceLbvh, to_device
from oracle import cpu

pytestmark = pytest.mark.gpu


def rays8(rays6):
    r = np.zeros((len(rays6), 8), np.float32)
    r[:, 0:3] = rays6[:, 0:3]
    r[:, 4:7] = rays6[:, 3:6]
    return torch.from_numpy(r).cuda()


def gpu_hits(lb, rays6, any_hit=False, stats=False):
    h, st = lb.trace(rays8(rays6), any_hit=any_hit, stats=stats)
    torch.cuda.synchronize()
    lb.status()
    h = h.cpu().numpy()
    return h[:, 0].copy(), h[:, 3].copy().view(np.uint32), h[:, 1:3].copy(), (None if st is None else st.cpu().numpy())


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_trace_matches_golden(cuda, name):
    g = load_golden(name)
    lb = DeviceLbvh(len(g["tris_in"]), int(g["bits"]))
    lb.build(to_device(g["tris_in"]), box=g["box"], check_root=True)
    t, idx, uv, _ = gpu_hits(lb, g["rays"])
    assert np.array_equal(idx, g["idx"])
    assert t.tobytes() == g["t"].tobytes()
    hit = g["idx"] != cpu.INVALID
    assert uv[hit].tobytes() == g["uv"][hit].tobytes()


@pytest.mark.parametrize("bits", [30, 63])
def test_trace_matches_oracle_large(cuda, bits):
    tris = cpt.scene_sphere_hairball(256, 128, 60_000, seed=9)[0]
    lb = DeviceLbvh(len(tris), bits)
    lb.build(to_device(tris), check_root=True)
    ob = cpu.build(tris, bits)
    rays = rays_at(tris, 200_000, seed=1, spread=(-2.5, 2.5))
    t, idx, uv, st = gpu_hits(lb, rays, stats=True)
    ot, oidx, ouv, ost = cpu.trace(ob, rays, stats=True)
    assert np.array_equal(idx, oidx)
    assert t.tobytes() == ot.tobytes()
    hit = oidx != cpu.INVALID
    assert hit.sum() > 50_000
    assert uv[hit].tobytes() == ouv[hit].tobytes()
    # the traversal visits the same nodes and tests the same triangles as the reference's
    assert np.array_equal(st[:, 0].astype(np.uint64), ost[:, 0])
    assert np.array_equal(st[:, 1].astype(np.uint64), ost[:, 2])


def test_any_hit_matches_closest_hit_occlusion(cuda):
    tris = cpt.scene_random(100_000, seed=3)[0]
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris), check_root=True)
    rays = rays_at(tris, 100_000, seed=2)
    t_any, _, _, _ = gpu_hits(lb, rays, any_hit=True)
    t_cl, _, _, _ = gpu_hits(lb, rays, any_hit=False)
    assert np.array_equal(t_any < cpu.FLT_MAX, t_cl < cpu.FLT_MAX)
    ot, _, _ = cpu.trace(cpu.build(tris, 30), rays, any_hit=True)
    assert np.array_equal(t_any < cpu.FLT_MAX, ot < cpu.FLT_MAX)


def test_trace_zero_rays_is_a_no_op(cuda):
    tris = cpt.scene_random(100, seed=3)[0]
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris))
    cpt.trace(lb.bvh, 0, 0, False, 0)
