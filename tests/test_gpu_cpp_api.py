"""The C++ mirror classes (include/cpt.hpp: BVHBuilder, CUDAPathTracer and the
scene descriptions, named as the reference's) driven by a C++ program the way the
reference application drives its classes: the build equals the oracle's bit for
bit, the image equals the C ABI / Python path's, and a bad call is reported (or
thrown) without breaking the tracer."""
import os
import subprocess

import numpy as np
import pytest

import cpt
from oracle import cpu

pytestmark = pytest.mark.gpu

EXE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "cuda-path-tracer_b200", "_build",
                   "cpp_api_test")


def test_cpp_classes_build_and_render(cuda, tmp_path):
    assert os.path.exists(EXE), "build the library first (make -C cuda-path-tracer_b200)"
    r = subprocess.run([EXE, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "cpp api ok" in r.stdout and "frames 2" in r.stdout
    # the same scene as the program: cpt_scene_random(20000, seed 4), reference bounds
    tris, infos = cpt.scene_random(20000, seed=4)
    box = cpt.scene_bounds(tris)
    b = cpu.build(tris, 30, box=np.asarray(box, np.float32))
    got = {k: np.fromfile(tmp_path / f"{k}.bin", dtype) for k, dtype in
           (("tris", cpt.TRIANGLE_DTYPE), ("children", np.uint32), ("parents_leaf", np.uint32),
            ("parents_internal", np.uint32), ("boxes", cpt.BBOX_DTYPE))}
    assert got["tris"].tobytes() == b.tris.tobytes()
    assert got["children"].tobytes() == b.children.tobytes()
    assert got["parents_leaf"].tobytes() == b.parents_leaf.tobytes()
    assert got["parents_internal"].tobytes() == b.parents_internal.tobytes()
    assert got["boxes"].tobytes() == b.node_boxes.tobytes()
    # the image through the C ABI tracer object with the same calls
    t = cpt.Tracer(30)
    t.set_settings(bounces=3, intensity=3.0, stratified=True, seed=7)
    t.upload(tris, infos, None, box)
    cam = cpt.camera_look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.0), aspect=48 / 32)
    t.set_primary_rays(cam.as_array()[3:])
    t.set_eye(cam.eye)
    t.raytrace(48, 32)
    t.raytrace(48, 32)
    ref = t.read_image(48, 32)
    img = np.fromfile(tmp_path / "image.bin", np.float32).reshape(32, 48, 4)
    assert img.tobytes() == ref.tobytes()
    assert np.isfinite(img).all() and img[..., :3].max() > 0
    t.close()
    # setSplit / setWide / setNextEventEstimation against the same calls through the C ABI
    t = cpt.Tracer(30)
    t.set_settings(bounces=3, intensity=3.0, stratified=True, seed=7)
    t.set_split(2.0)
    t.set_wide(True)
    t.set_nee(True)
    t.upload(tris, infos, None, box)
    t.set_primary_rays(cam.as_array()[3:])
    t.set_eye(cam.eye)
    t.raytrace(48, 32)
    ref = t.read_image(48, 32)
    img = np.fromfile(tmp_path / "image_ext.bin", np.float32).reshape(32, 48, 4)
    assert img.tobytes() == ref.tobytes()
    assert t.bvh().wide_capacity == t.bvh().split_capacity > 0
    t.close()
