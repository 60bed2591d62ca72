"""Device-side image output and resume of progressive renders, on the GPU: the tracer
object's image written to device memory (cpt_tracer_resolve), its accumulator and frame
counter moved out and back (cpt_tracer_get_progress / cpt_tracer_set_progress), and a
renderer's accumulator saved to a file and loaded into another (cpt/progress.py). Each
resumed or device-side result must equal, byte for byte, the uninterrupted or host-side
one."""
import pytest
import torch

import cpt
from cpt.device import DeviceLbvh, DeviceRenderer, DeviceScene, make_params, to_device

pytestmark = pytest.mark.gpu

W, H = 64, 48


def scene(n=8000, seed=5):
    tris, infos = cpt.scene_random(n, seed=seed)
    infos["material"]["specularity"][: len(infos) - 2] = 0.0
    cam = cpt.camera_look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.0), aspect=W / H)
    return tris, infos, None, cam


def test_tracer_resolve_writes_the_image_on_the_device(cuda):
    """cpt_tracer_resolve (the device-side image the C++ mirror's setScreenTexture copies
    into its array) gives the bytes cpt_tracer_read_image gives."""
    tris, infos, _, cam = scene(n=8000)
    t = cpt.Tracer(63)
    t.upload(tris, infos)
    t.set_settings(bounces=2, intensity=3.0, stratified=True, seed=123, accum_mode=cpt.ACCUM_KAHAN)
    t.set_primary_rays(cam.as_array()[3:])
    t.set_eye(cam.as_array()[:3])
    t.raytrace(W, H, 2)
    img = t.read_image(W, H)
    out = torch.full((H, W, 4), -1.0, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    t.resolve(out.data_ptr())
    torch.cuda.synchronize()
    assert out.cpu().numpy().tobytes() == img.tobytes()
    t.close()


def test_tracer_progress_resume_matches_one_run(cuda):
    """cpt_tracer_get_progress / cpt_tracer_set_progress: frames [0, 2) by one tracer,
    restored into a second tracer with the same scene, camera and settings that renders
    frame 2, give the image of one tracer rendering frames [0, 3)."""
    tris, infos, _, cam = scene(n=8000)

    def tracer():
        t = cpt.Tracer(63)
        t.upload(tris, infos)
        t.set_settings(bounces=2, intensity=3.0, stratified=True, seed=123, accum_mode=cpt.ACCUM_KAHAN)
        t.set_primary_rays(cam.as_array()[3:])
        t.set_eye(cam.as_array()[:3])
        return t

    straight = tracer()
    straight.raytrace(W, H, 3)
    want = straight.read_image(W, H)
    first = tracer()
    first.raytrace(W, H, 2)
    acc, frame = first.get_progress(W, H, cpt.ACCUM_KAHAN)
    assert frame == 2 and acc.nbytes == cpt.accum_bytes(W, H, cpt.ACCUM_KAHAN)
    second = tracer()
    # the checkpoint's accumulator mode is checked: the FP64 layout has the same size
    with pytest.raises(cpt.CptError) as e:
        second.set_progress(acc, W, H, frame, cpt.ACCUM_F64)
    assert e.value.code == cpt.ERR_INVALID_ARGUMENT
    second.set_progress(acc, W, H, frame, cpt.ACCUM_KAHAN)
    second.raytrace(W, H, 1)
    assert second.frame == 3
    assert second.read_image(W, H).tobytes() == want.tobytes()
    for t in (straight, first, second):
        t.close()


def test_checkpoint_resume_matches_one_accumulation(cuda, tmp_path):
    """Frames [0, 2) rendered, saved to a file (cpt/progress.py), loaded into a fresh
    renderer's accumulator and frames [2, 4) rendered there: the same accumulator bytes
    as both calls on one accumulator."""
    from cpt import progress

    tris, infos, _, cam = scene(n=8000)
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris), check_root=True)
    sc = DeviceScene(infos)
    p = make_params(W, H, 2, 0, 3, 3.0, True, 3, cpt.ACCUM_KAHAN)
    direct = DeviceRenderer(p)
    direct.render(lb, sc, cam, frame0=0)
    direct.render(lb, sc, cam, frame0=2)
    first = DeviceRenderer(p)
    first.render(lb, sc, cam, frame0=0)
    torch.cuda.synchronize()
    path = str(tmp_path / "progress.npz")
    progress.save(path, first.accum, p, next_frame=2)
    second = DeviceRenderer(p)
    frame0 = progress.resume(second, path)
    assert frame0 == 2
    second.render(lb, sc, cam, frame0=frame0)
    torch.cuda.synchronize()
    direct.check_status()
    second.check_status()
    assert second.accum.cpu().numpy().tobytes() == direct.accum.cpu().numpy().tobytes()
