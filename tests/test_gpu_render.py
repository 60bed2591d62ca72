"""Wavefront path tracer on the GPU against the oracle's restatement of the
reference estimator (same Philox stream): per-pixel accumulators bit-exact for
the Kahan, running-lerp and FP64 modes; ray counts exact; the tracer object
(host buffers in, image out) equal to the device path."""
import numpy as np
import pytest
import torch

import cpt
from cpt.device import DeviceLbvh, DeviceRenderer, DeviceScene, make_params, to_device
from oracle import cpu

pytestmark = pytest.mark.gpu

W, H = 64, 48


def scene(n=20_000, seed=5, lights=None, spec=0.0):
    tris, infos = cpt.scene_random(n, seed=seed)
    infos["material"]["specularity"][: len(infos) - 2] = spec
    cam = cpt.camera_look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.0), aspect=W / H)
    return tris, infos, lights, cam


def dir_lights():
    l = np.zeros(2, cpt.DIR_LIGHT_DTYPE)
    l[0] = ((1.0, 0.9, 0.8), (0.3, -1.0, 0.2), 1.5)
    l[1] = ((0.2, 0.3, 1.0), (-0.5, -0.7, 0.4), 0.7)
    l["direction"] /= np.linalg.norm(l["direction"], axis=1, keepdims=True)
    return l.astype(cpt.DIR_LIGHT_DTYPE)


def ocam(cam, jitter=False):
    return cpu.ocam_from(cam.eye, cam.as_array()[3:], np.ctypeslib.as_array(cam.inv_view_proj), jitter=int(jitter),
                         jitter_x=2.0 / W, jitter_y=2.0 / H)


def gpu_render(tris, infos, lights, cam, mode, spp=4, frame0=5, bounces=3, seed=77, bits=30, jitter=False,
               wave_paths=0, ref_grid=False, w=W, h=H, stratified=True, ray_sort=False, wave_lanes=0):
    lb = DeviceLbvh(len(tris), bits)
    lb.build(to_device(tris), check_root=True)
    sc = DeviceScene(infos, lights)
    c = cpt.Camera.from_buffer_copy(cam)
    c.jitter, c.jitter_x, c.jitter_y = int(jitter), 2.0 / w, 2.0 / h
    r = DeviceRenderer(make_params(w, h, spp, frame0, bounces, 3.0, stratified, seed, mode, ref_grid, wave_paths,
                                   ray_sort=ray_sort, wave_lanes=wave_lanes))
    r.render(lb, sc, c)
    torch.cuda.synchronize()
    r.check_status()
    return r, lb


def oracle_samples(tris, infos, lights, cam, spp=4, frame0=5, bounces=3, seed=77, bits=30, jitter=False, w=W, h=H,
                   stratified=True):
    b = cpu.build(tris, bits)
    return cpu.render(b, infos, lights, w, h, spp, frame0, bounces, 3.0, stratified, seed, ocam(cam, jitter))


def accum_arrays(r, mode):
    a = r.accum.cpu().numpy().view(np.uint8)
    if mode == cpt.ACCUM_KAHAN:
        f = a.view(np.float32).reshape(2, H, W, 4)
        return f[0], f[1]
    if mode == cpt.ACCUM_LERP:
        return a.view(np.float32).reshape(H, W, 4), None
    return a.view(np.float64).reshape(H, W, 4), None


@pytest.mark.parametrize("bits", [30, 63])
def test_kahan_accumulator_bit_exact(cuda, bits):
    tris, infos, lights, cam = scene()
    r, _ = gpu_render(tris, infos, lights, cam, cpt.ACCUM_KAHAN, bits=bits)
    rad, counts = oracle_samples(tris, infos, lights, cam, bits=bits)
    s, c, n = cpu.accumulate_kahan(rad)
    gs, gc = accum_arrays(r, cpt.ACCUM_KAHAN)
    assert (rad.sum(axis=(0, 1, 2)) > 0).all(), "scene should receive light"
    assert gs[..., :3].tobytes() == s.tobytes()
    assert gc[..., :3].tobytes() == c.tobytes()
    assert np.all(gs[..., 3] == n)
    assert np.array_equal(r.counts.cpu().numpy()[:3].astype(np.uint64), counts)
    img = r.resolve().cpu().numpy()
    assert img[..., :3].tobytes() == (s / n).astype(np.float32).tobytes()


def test_lerp_accumulator_matches_reference_running_mean(cuda):
    tris, infos, lights, cam = scene()
    r, _ = gpu_render(tris, infos, lights, cam, cpt.ACCUM_LERP, frame0=0)
    rad, _ = oracle_samples(tris, infos, lights, cam, frame0=0)
    img, _ = accum_arrays(r, cpt.ACCUM_LERP)
    assert img[..., :3].tobytes() == cpu.accumulate_lerp(rad, 0).tobytes()
    assert np.all(img[..., 3] == 1.0)


def test_f64_accumulator(cuda):
    tris, infos, lights, cam = scene()
    r, _ = gpu_render(tris, infos, lights, cam, cpt.ACCUM_F64)
    rad, _ = oracle_samples(tris, infos, lights, cam)
    acc, _ = accum_arrays(r, cpt.ACCUM_F64)
    want = np.zeros((H, W, 3), np.float64)
    for x in rad:
        want += x.astype(np.float64)
    assert acc[..., :3].tobytes() == want.tobytes()


def test_camera_jitter_per_sample(cuda):
    tris, infos, lights, cam = scene()
    r, _ = gpu_render(tris, infos, lights, cam, cpt.ACCUM_KAHAN, jitter=True)
    rad, _ = oracle_samples(tris, infos, lights, cam, jitter=True)
    s, c, _ = cpu.accumulate_kahan(rad)
    gs, _ = accum_arrays(r, cpt.ACCUM_KAHAN)
    assert gs[..., :3].tobytes() == s.tobytes()


def test_wave_size_does_not_change_the_image(cuda):
    tris, infos, lights, cam = scene()
    a, _ = gpu_render(tris, infos, lights, cam, cpt.ACCUM_KAHAN, spp=6, wave_paths=W * H)
    b, _ = gpu_render(tris, infos, lights, cam, cpt.ACCUM_KAHAN, spp=6, wave_paths=4 * W * H)
    c, _ = gpu_render(tris, infos, lights, cam, cpt.ACCUM_KAHAN, spp=6)
    assert a.accum.cpu().numpy().tobytes() == b.accum.cpu().numpy().tobytes() == c.accum.cpu().numpy().tobytes()


@pytest.mark.parametrize("mode", [cpt.ACCUM_KAHAN, cpt.ACCUM_LERP])
def test_wave_lanes_do_not_change_the_image(cuda, mode):
    """Two lanes (each wave's paths in halves on two streams) against one: the same
    accumulator bytes and ray counts, with one wave and with several."""
    tris, infos, _, cam = scene()
    lights = dir_lights()
    for wave_paths in (0, 2 * W * H):
        one, _ = gpu_render(tris, infos, lights, cam, mode, spp=6, bounces=4, wave_paths=wave_paths, wave_lanes=1)
        two, _ = gpu_render(tris, infos, lights, cam, mode, spp=6, bounces=4, wave_paths=wave_paths, wave_lanes=2)
        assert one.accum.cpu().numpy().tobytes() == two.accum.cpu().numpy().tobytes()
        assert np.array_equal(one.counts.cpu().numpy()[:16], two.counts.cpu().numpy()[:16])
        assert int(two.counts[0]) > 0


def test_coherence_sort_does_not_change_the_image(cuda):
    tris, infos, _, cam = scene()
    lights = dir_lights()
    a, _ = gpu_render(tris, infos, lights, cam, cpt.ACCUM_KAHAN, spp=3, bounces=5, ray_sort=False)
    b, _ = gpu_render(tris, infos, lights, cam, cpt.ACCUM_KAHAN, spp=3, bounces=5, ray_sort=True)
    assert a.accum.cpu().numpy().tobytes() == b.accum.cpu().numpy().tobytes()
    assert np.array_equal(a.counts.cpu().numpy(), b.counts.cpu().numpy())
    rad, _ = oracle_samples(tris, infos, lights, cam, spp=3, bounces=5)
    s, _, _ = cpu.accumulate_kahan(rad)
    gs, _ = accum_arrays(b, cpt.ACCUM_KAHAN)
    assert gs[..., :3].tobytes() == s.tobytes()


def test_several_cameras_in_one_call(cuda):
    tris, infos, _, _ = scene()
    cams = [cpt.camera_look_at(eye, (0.5, 0.5, 0.5), aspect=W / H)
            for eye in ((0.5, 0.5, -1.2), (-0.8, 0.7, 0.4), (1.9, 0.3, 0.6))]
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris), check_root=True)
    r = DeviceRenderer(make_params(W, H, 2, 3, 3, 3.0, True, 21, cpt.ACCUM_KAHAN, cameras=3, wave_paths=2 * W * H))
    r.render(lb, DeviceScene(infos), cams)
    torch.cuda.synchronize()
    r.check_status()
    acc = r.accum.cpu().numpy().view(np.float32).reshape(3, 2, H, W, 4)
    b = cpu.build(tris, 30)
    for c, cam in enumerate(cams):
        rad, _ = cpu.render(b, infos, None, W, H, 2, 3, 3, 3.0, True, 21, cpu.ocam_from(cam.eye, cam.as_array()[3:]),
                            camera_index=c)
        s, _, n = cpu.accumulate_kahan(rad)
        assert acc[c, 0, ..., :3].tobytes() == s.tobytes()
        assert np.all(acc[c, 0, ..., 3] == n)


def test_batched_scenes_in_one_call(cuda):
    """Three different scenes at three resolutions in the same waves: each view's
    accumulator equals the oracle's render of that scene alone (view i = stream word i)."""
    from cpt.device import BatchRenderer

    cube = ((0.5, 0.5, -1.2), (0.5, 0.5, 0.0))
    specs = [(cpt.scene_random(9000, seed=3), (40, 24), cube), (cpt.scene_random(15000, seed=4), (64, 48), cube),
             (cpt.scene_sphere_hairball(64, 32, 3000, seed=5), (32, 32), ((0.0, 0.3, -3.6), (0.0, 0.0, 0.0)))]
    views, keep = [], []
    for (tris, infos), (w, h), (eye, tgt) in specs:
        lb = DeviceLbvh(len(tris), 30)
        lb.build(to_device(tris), check_root=True)
        sc = DeviceScene(infos)
        cam = cpt.camera_look_at(eye, tgt, aspect=w / h)
        views.append((lb, sc, cam, w, h))
        keep.append((tris, infos, cam, w, h))
    br = BatchRenderer(views, make_params(0, 0, 3, 1, 4, 3.0, True, 13, cpt.ACCUM_KAHAN, wave_paths=3000))
    br.render()
    torch.cuda.synchronize()
    br.check_status()
    for i, (tris, infos, cam, w, h) in enumerate(keep):
        acc = br.accums[i].cpu().numpy().view(np.float32).reshape(2, h, w, 4)[0]
        b = cpu.build(tris, 30)
        rad, _ = cpu.render(b, infos, None, w, h, 3, 1, 4, 3.0, True, 13, cpu.ocam_from(cam.eye, cam.as_array()[3:]),
                            camera_index=i)
        s, _, n = cpu.accumulate_kahan(rad)
        assert acc[..., :3].tobytes() == s.tobytes(), i
        assert np.all(acc[..., 3] == n)


def test_batched_scenes_with_two_lanes(cuda):
    """Views of different scenes split between two wave lanes (the halves of the path
    range cut through a view): every accumulator equals the one-lane call's."""
    from cpt.device import BatchRenderer

    views = []
    for k, (n, (w, h)) in enumerate([(9000, (40, 24)), (15000, (64, 48)), (6000, (48, 40))]):
        tris, infos = cpt.scene_random(n, seed=20 + k)
        lb = DeviceLbvh(len(tris), 30)
        lb.build(to_device(tris), check_root=True)
        views.append((lb, DeviceScene(infos), cpt.camera_look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.0), aspect=w / h), w, h))
    out = []
    for lanes in (1, 2):
        br = BatchRenderer(views, make_params(0, 0, 3, 1, 4, 3.0, True, 13, cpt.ACCUM_KAHAN, wave_lanes=lanes))
        br.render()
        torch.cuda.synchronize()
        br.check_status()
        out.append(([a.cpu().numpy().tobytes() for a in br.accums], br.counts.cpu().numpy()[:16].copy()))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])


def test_directional_lights_shadow_rays(cuda):
    tris, infos, _, cam = scene()
    lights = dir_lights()
    r, _ = gpu_render(tris, infos, lights, cam, cpt.ACCUM_KAHAN)
    rad, counts = oracle_samples(tris, infos, lights, cam)
    s, _, _ = cpu.accumulate_kahan(rad)
    gs, _ = accum_arrays(r, cpt.ACCUM_KAHAN)
    assert counts[2] > 0
    assert gs[..., :3].tobytes() == s.tobytes()  # shininess 0: no pow() in play, bit-exact
    assert np.array_equal(r.counts.cpu().numpy()[:3].astype(np.uint64), counts)


def test_specular_term_within_tolerance(cuda):
    # powf differs between CUDA and the host libm by at most a few ulp; the
    # specular term is a colour, it does not steer rays: relative 1e-5.
    tris, infos, _, cam = scene(spec=32.0)
    lights = dir_lights()
    r, _ = gpu_render(tris, infos, lights, cam, cpt.ACCUM_KAHAN)
    rad, _ = oracle_samples(tris, infos, lights, cam)
    s, _, _ = cpu.accumulate_kahan(rad)
    gs, _ = accum_arrays(r, cpt.ACCUM_KAHAN)
    np.testing.assert_allclose(gs[..., :3], s, rtol=1e-5, atol=1e-6)


def test_reference_grid_truncation(cuda):
    w, h = 70, 50
    tris, infos, lights, _ = scene()
    cam = cpt.camera_look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.0), aspect=w / h)
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris))
    sc = DeviceScene(infos, None)
    r = DeviceRenderer(make_params(w, h, 2, 0, 2, 3.0, True, 1, cpt.ACCUM_KAHAN, True, 0))
    r.render(lb, sc, cam)
    torch.cuda.synchronize()
    acc = r.accum.cpu().numpy().view(np.float32).reshape(2, h, w, 4)[0]
    assert np.all(acc[:48, :64, 3] == 2) and np.all(acc[48:, :, 3] == 0) and np.all(acc[:, 64:, 3] == 0)
    b = cpu.build(tris, 30)
    rad, _ = cpu.render(b, infos, None, w, h, 2, 0, 2, 3.0, True, 1, cpu.ocam_from(cam.eye, cam.as_array()[3:]))
    s, _, _ = cpu.accumulate_kahan(rad)
    assert acc[:48, :64, :3].tobytes() == np.ascontiguousarray(s[:48, :64]).tobytes()


def test_tracer_object_host_buffers(cuda):
    """cpt_tracer (CUDAPathTracer): upload host soup, set rays and eye, raytrace
    frame by frame, read the image — equals the oracle."""
    tris, infos, _, cam = scene(n=8000)
    t = cpt.Tracer(63)
    t.upload(tris, infos)
    t.set_settings(bounces=2, intensity=3.0, stratified=True, seed=123, accum_mode=cpt.ACCUM_KAHAN)
    t.set_primary_rays(cam.as_array()[3:])
    t.set_eye(cam.as_array()[:3])
    t.raytrace(W, H, 1)
    t.raytrace(W, H, 2)
    assert t.frame == 3
    img = t.read_image(W, H)
    b = cpu.build(tris, 63)
    rad, counts = cpu.render(b, infos, None, W, H, 3, 0, 2, 3.0, True, 123, cpu.ocam_from(cam.eye, cam.as_array()[3:]))
    s, _, n = cpu.accumulate_kahan(rad)
    assert img[..., :3].tobytes() == (s / n).astype(np.float32).tobytes()
    assert np.array_equal(t.ray_counts(), counts)
    t.reset_frames()
    t.raytrace(W, H, 1)
    img1 = t.read_image(W, H)
    s1, _, _ = cpu.accumulate_kahan(rad[:1])
    assert img1[..., :3].tobytes() == s1.tobytes()
    t.close()


def test_tracer_uploads_overlap_frames(cuda):
    """The tracer keeps two scenes: an upload issued while the previous scene's frame is
    still in flight (before its read-back) builds into the other scene, and every image
    equals the image of a tracer given that scene alone."""
    (ta, ia, _, cam), (tb, ib) = scene(n=8000), cpt.scene_random(6000, seed=17)

    def alone(tris, infos):
        t = cpt.Tracer(63)
        t.set_camera(cam)
        t.set_settings(bounces=2, intensity=3.0, stratified=True, seed=5)
        t.upload(tris, infos)
        t.raytrace(W, H, 2)
        img = t.read_image(W, H)
        t.close()
        return img

    want = [alone(ta, ia), alone(tb, ib)]
    t = cpt.Tracer(63)
    t.set_camera(cam)
    t.set_settings(bounces=2, intensity=3.0, stratified=True, seed=5)
    order = [0, 1, 0, 1, 1]
    t.upload(*((ta, ia), (tb, ib))[order[0]])
    t.raytrace(W, H, 2)
    for i, k in enumerate(order):
        if i + 1 < len(order):
            t.upload(*((ta, ia), (tb, ib))[order[i + 1]])  # before this frame's read-back
        img = t.read_image(W, H)
        assert img.tobytes() == want[k].tobytes(), (i, k)
        if i + 1 < len(order):
            t.raytrace(W, H, 2)
    assert t.bvh().n == len(tb)
    t.close()


def test_graph_replay_advances_the_sample_stream(cuda):
    """One render call captured in a CUDA graph, replayed twice, equals two direct
    calls with frame0 = 0 and spp (the device frame counter advances per replay)."""
    tris, infos, _, cam = scene(n=8000)
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris), check_root=True)
    sc = DeviceScene(infos)
    direct = DeviceRenderer(make_params(W, H, 2, 0, 3, 3.0, True, 3, cpt.ACCUM_KAHAN))
    direct.render(lb, sc, cam, frame0=0)
    direct.render(lb, sc, cam, frame0=2)
    counter = torch.zeros(1, dtype=torch.int32, device="cuda")
    p = make_params(W, H, 2, 0, 3, 3.0, True, 3, cpt.ACCUM_KAHAN)
    p.frame_counter = counter.data_ptr()
    graphed = DeviceRenderer(p)
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        graphed.render(lb, sc, cam)  # warm-up outside the graph (frame 0..1)
    torch.cuda.synchronize()
    graphed.reset()
    counter.zero_()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        graphed.render(lb, sc, cam)
    torch.cuda.synchronize()
    graphed.reset()
    counter.zero_()
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    assert int(counter.item()) == 4
    assert graphed.accum.cpu().numpy().tobytes() == direct.accum.cpu().numpy().tobytes()
