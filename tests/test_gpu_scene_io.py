"""Ingested OBJ scenes and the BVH heat map on the GPU, against the oracle."""
import numpy as np
import pytest
import torch

import cpt
from cpt.device import DeviceLbvh, DeviceRenderer, DeviceScene, make_params, to_device
from oracle import cpu
from scene_files import write_box

pytestmark = pytest.mark.gpu


def heat(tris, cam, w, h, bits, base=(0.02, 0.01, 0.005)):
    lb = DeviceLbvh(len(tris), bits)
    lb.build(to_device(tris), check_root=True)
    rgba = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    counts = torch.zeros((h, w), dtype=torch.int32, device="cuda")
    cpt.bvh_heatmap(lb.bvh, cam, w, h, base, rgba.data_ptr(), counts.data_ptr(),
                    torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    b = cpu.build(tris, bits)
    o_rgba, o_counts = cpu.heatmap(b, cpu.ocam_from(cam.eye, cam.as_array()[3:]), w, h, base)
    return rgba.cpu().numpy(), counts.cpu().numpy().view(np.uint32), o_rgba, o_counts


@pytest.mark.parametrize("bits", [30, 63])
def test_heatmap_matches_oracle(cuda, bits):
    tris = cpt.scene_sphere_hairball(128, 64, 20_000, seed=4)[0]
    cam = cpt.camera_look_at((0.0, 0.3, -3.6), (0, 0, 0), aspect=1.5)
    g, gc, o, oc = heat(tris, cam, 96, 64, bits)
    assert np.array_equal(gc, oc) and gc.max() > 50
    assert g.tobytes() == o.tobytes()


def test_obj_box_render_matches_oracle(cuda, tmp_path):
    tris, infos = cpt.load_obj(write_box(str(tmp_path)))
    w, h = 64, 48
    cam = cpt.camera_look_at((0.0, 0.0, -3.4), (0, 0, 0), aspect=w / h)
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris), check_root=True)
    r = DeviceRenderer(make_params(w, h, 4, 0, 4, 3.0, True, 9))
    r.render(lb, DeviceScene(infos), cam)
    torch.cuda.synchronize()
    r.check_status()
    acc = r.accum.cpu().numpy().view(np.float32).reshape(2, h, w, 4)[0]
    b = cpu.build(tris, 30)
    rad, _ = cpu.render(b, infos, None, w, h, 4, 0, 4, 3.0, True, 9, cpu.ocam_from(cam.eye, cam.as_array()[3:]))
    s, _, _ = cpu.accumulate_kahan(rad)
    assert s.max() > 1.0, "the lamp must light the box"
    assert acc[..., :3].tobytes() == s.tobytes()
    g, gc, o, oc = heat(tris, cam, w, h, 30)
    assert np.array_equal(gc, oc) and g.tobytes() == o.tobytes()
