"""Next-event estimation on the GPU against the oracle.

The emitter table (cpt_emitters_build) must equal the oracle's byte for byte; a
render with params.nee = 1 must give the oracle's per-sample radiance bit for bit
(Kahan accumulators) with the same primary / extension / shadow ray counts; and,
since it only changes how emission is sampled, its converged image must agree
with the reference estimator's within the noise of both."""
import numpy as np
import pytest
import torch

import cpt
from cpt.device import DeviceLbvh, DeviceRenderer, DeviceScene, make_params, to_device
from oracle import cpu

pytestmark = pytest.mark.gpu

W, H = 64, 48


def scene(n=20_000, seed=5, emissive_frac=0.0):
    tris, infos = cpt.scene_random(n, seed=seed)
    if emissive_frac:
        rng = np.random.default_rng(seed)
        pick = rng.random(len(infos) - 2) < emissive_frac
        infos["material"]["emission"][: len(infos) - 2][pick] = rng.uniform(0.05, 0.5, (pick.sum(), 3))
    cam = cpt.camera_look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.0), aspect=W / H)
    return tris, infos, cam


def ocam(cam):
    return cpu.ocam_from(cam.eye, cam.as_array()[3:], np.ctypeslib.as_array(cam.inv_view_proj))


def device_table(sc, lb, cap):
    found = sc.build_emitters(lb, cap)
    nbytes = 16 + 48 * cap
    return sc.emitters[:nbytes].cpu().numpy().view(np.float32).copy(), found


@pytest.mark.parametrize("frac", [0.0, 0.3])
def test_emitter_table_bit_exact(cuda, frac):
    tris, infos, _ = scene(emissive_frac=frac)
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris), check_root=True)
    sc = DeviceScene(infos)
    cap = 8192
    got, found = device_table(sc, lb, cap)
    want, want_found = cpu.emitters(cpu.build(tris, 30), infos, cap)
    assert found == want_found
    if frac == 0.0:
        assert found == 2  # the light quad
    else:
        assert found > 2 * 256  # several chunks and cdf segments
    count = int(got[:1].view(np.uint32)[0])
    assert count == found
    # header and the listed emitters (the rest of the capacity is not written)
    assert got[:4 + 12 * count].tobytes() == want[:4 + 12 * count].tobytes()
    cdf = got[4:].reshape(-1, 12)[:count, 3]
    assert np.all(np.diff(cdf) >= 0) and cdf[-1] == np.float32(1.0)


def test_emitter_table_overflow(cuda):
    tris, infos, _ = scene(emissive_frac=0.3)
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris))
    sc = DeviceScene(infos)
    with pytest.raises(cpt.CptError) as e:
        sc.build_emitters(lb, 64)
    assert e.value.code == cpt.ERR_SCRATCH_TOO_SMALL
    hdr = sc.emitters[:16].cpu().numpy().view(np.uint32)
    assert hdr[0] == 0 and hdr[2] > 64 and hdr[3] == 1


def nee_render(tris, infos, cam, bits=30, spp=4, frame0=5, bounces=3, seed=77, nee=True, mode=cpt.ACCUM_KAHAN,
               wave_paths=0, stratified=True):
    lb = DeviceLbvh(len(tris), bits)
    lb.build(to_device(tris), check_root=True)
    sc = DeviceScene(infos)
    if nee:
        sc.build_emitters(lb, 1 << 14)
    r = DeviceRenderer(make_params(W, H, spp, frame0, bounces, 3.0, stratified, seed, mode, wave_paths=wave_paths,
                                   nee=nee))
    r.render(lb, sc, cam)
    torch.cuda.synchronize()
    r.check_status()
    return r, lb, sc


@pytest.mark.parametrize("bits,frac", [(30, 0.0), (63, 0.0), (30, 0.3)])
def test_nee_render_bit_exact(cuda, bits, frac):
    tris, infos, cam = scene(emissive_frac=frac)
    r, _, _ = nee_render(tris, infos, cam, bits=bits)
    b = cpu.build(tris, bits)
    table, _ = cpu.emitters(b, infos, 1 << 14)
    rad, counts = cpu.render(b, infos, None, W, H, 4, 5, 3, 3.0, True, 77, ocam(cam), nee_table=table)
    s, c, n = cpu.accumulate_kahan(rad)
    a = r.accum.cpu().numpy().view(np.float32).reshape(2, H, W, 4)
    assert counts[2] > 0, "shadow rays expected"
    assert (rad.sum(axis=(0, 1, 2)) > 0).all()
    assert a[0][..., :3].tobytes() == s.tobytes()
    assert a[1][..., :3].tobytes() == c.tobytes()
    assert np.array_equal(r.counts.cpu().numpy()[:3].astype(np.uint64), counts)


def test_nee_wave_size_does_not_change_the_image(cuda):
    tris, infos, cam = scene()
    a, _, _ = nee_render(tris, infos, cam, spp=6, wave_paths=W * H)
    b, _, _ = nee_render(tris, infos, cam, spp=6)
    assert a.accum.cpu().numpy().tobytes() == b.accum.cpu().numpy().tobytes()


def test_nee_needs_a_table(cuda):
    tris, infos, cam = scene()
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris))
    sc = DeviceScene(infos)
    r = DeviceRenderer(make_params(W, H, 1, nee=True))
    with pytest.raises(cpt.CptError) as e:
        r.render(lb, sc, cam)
    assert e.value.code == cpt.ERR_INVALID_ARGUMENT


def test_nee_converges_to_the_reference_estimator(cuda):
    """Same expectation: FP64 means of 2048 samples per pixel, reference estimator
    vs next-event estimation, agree within the standard error of their difference."""
    tris, infos, cam = scene(n=5000, seed=9)
    spp = 2048
    imgs, var = [], []
    for nee in (False, True):
        r, _, _ = nee_render(tris, infos, cam, spp=spp, frame0=0, nee=nee, mode=cpt.ACCUM_F64, stratified=False)
        acc = r.accum.cpu().numpy().view(np.float64).reshape(H, W, 4)
        imgs.append(acc[..., :3] / acc[..., 3:4])
    # per-pixel spread from two independent halves of each estimator
    for nee in (False, True):
        halves = []
        for f0 in (0, spp):
            r, _, _ = nee_render(tris, infos, cam, spp=spp // 2, frame0=f0 + 10 * spp, nee=nee,
                                 mode=cpt.ACCUM_F64, stratified=False)
            acc = r.accum.cpu().numpy().view(np.float64).reshape(H, W, 4)
            halves.append(acc[..., :3] / acc[..., 3:4])
        var.append(((halves[0] - halves[1]) ** 2) / 4.0)  # variance of a 2048-sample mean
    d = imgs[1] - imgs[0]
    se_mean = np.sqrt((var[0] + var[1]).mean() / d.size)  # standard error of the image-wide mean difference
    assert imgs[0].mean() > 0.01
    assert abs(d.mean()) < 5 * se_mean + 1e-5
    # next-event estimation lowers the per-pixel variance on this small light
    assert var[1].mean() < 0.5 * var[0].mean()


def test_tracer_object_with_nee(cuda):
    """cpt_tracer with cpt_tracer_set_nee(1): the emitter table is built from the
    upload (more emitters than the first sizing pass holds) and the image equals the
    oracle's next-event render; switching the estimator restarts the accumulation."""
    tris, infos, cam = scene(n=8000, emissive_frac=0.5)
    t = cpt.Tracer(63)
    t.upload(tris, infos)
    t.set_settings(bounces=2, intensity=3.0, stratified=True, seed=123, accum_mode=cpt.ACCUM_KAHAN)
    t.set_primary_rays(cam.as_array()[3:])
    t.set_eye(cam.as_array()[:3])
    t.raytrace(W, H, 1)
    t.set_nee(True)
    assert t.frame == 0
    t.raytrace(W, H, 2)
    img = t.read_image(W, H)
    b = cpu.build(tris, 63)
    table, found = cpu.emitters(b, infos, 1 << 14)
    assert found > 1024
    rad, _ = cpu.render(b, infos, None, W, H, 2, 0, 2, 3.0, True, 123, cpu.ocam_from(cam.eye, cam.as_array()[3:]),
                        nee_table=table)
    s, _, n = cpu.accumulate_kahan(rad)
    assert img[..., :3].tobytes() == (s / n).astype(np.float32).tobytes()
    t.close()
