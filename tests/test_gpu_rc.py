"""Radiance cache on the GPU: the fused BF16 tensor-core MLP against a PyTorch
float64 reference with the same BF16 rounding points (inference within 1%,
gradients within 2% in norm), training that reduces the loss, and cached
rendering: a network that predicts zero reproduces the plain depth-2 render bit
for bit (the image's first bounce is the plain tracer's), and a trained cache
agrees with the plain full-depth image in the mean."""
import numpy as np
import pytest
import torch

import cpt
from cpt.device import (CachedRenderer, BatchRenderer, DeviceLbvh, DeviceScene, RadianceCache, make_params,
                        rc_default_params, to_device)

import rc_reference as ref

pytestmark = pytest.mark.gpu

BOX = np.array([-1.0, -0.5, 0.0, 2.0, 1.5, 1.0], np.float32)


def random_samples(n, seed=0, smooth_target=False):
    g = np.random.default_rng(seed)
    s = np.zeros((n, 16), np.float32)
    s[:, 0:3] = g.uniform(BOX[:3], BOX[3:], (n, 3))
    d = g.normal(size=(n, 3))
    s[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    nn = g.normal(size=(n, 3))
    s[:, 8:11] = nn / np.linalg.norm(nn, axis=1, keepdims=True)
    s[:, 12:15] = g.uniform(0.2, 0.9, (n, 3))
    if smooth_target:
        p = (s[:, 0:3] - BOX[:3]) / (BOX[3:] - BOX[:3])
        t = 0.5 + 0.3 * np.sin(2 * np.pi * p[:, 0]) * np.cos(np.pi * p[:, 1]) + 0.2 * p[:, 2]
        s[:, 3], s[:, 7], s[:, 11] = t, 0.8 * t, 0.6 * t
    else:
        s[:, [3, 7, 11]] = g.uniform(0.0, 2.0, (n, 3))
    return s


def random_weights(seed=1, scale=1.0):
    g = np.random.default_rng(seed)
    return [(g.uniform(-1, 1, (fi, fo)) * np.sqrt(6.0 / fi) * scale).astype(np.float32) for fi, fo in ref.LAYERS]


def test_inference_matches_torch(cuda):
    rc = RadianceCache()
    w = random_weights()
    rc.set_weights(w)
    s = random_samples(5000, seed=2)
    got = rc.infer(torch.from_numpy(s).cuda(), BOX).cpu().numpy().astype(np.float64)
    y, _ = ref.forward(w, torch.from_numpy(s), BOX)
    want = y[:, :3].numpy()
    scale = np.abs(want).max()
    err = np.abs(got - want)
    # BF16 activations: a value on a rounding boundary may round the other way
    assert err.max() <= 0.02 * scale
    assert err.mean() <= 1e-3 * scale
    assert rc.get_weights()[2].tobytes() == w[2].tobytes()


def test_inference_ragged_counts(cuda):
    rc = RadianceCache()
    rc.set_weights(random_weights(seed=3))
    s = torch.from_numpy(random_samples(1000, seed=4)).cuda()
    full = rc.infer(s, BOX).cpu().numpy()
    for n in (1, 15, 16, 17, 129, 999):
        part = rc.infer(s[:n], BOX).cpu().numpy()
        assert part.tobytes() == full[:n].tobytes()


def test_gradient_matches_torch(cuda):
    # Adam's first step is lr * g / (|g| + eps); with lr = eps = 1e6 it is g to 1e-6
    rc = RadianceCache(rc_default_params(learning_rate=1e6, epsilon=1e6))
    w = random_weights(seed=5)
    rc.set_weights(w)
    s = random_samples(3000, seed=6)
    loss = rc.train(torch.from_numpy(s).cuda(), BOX, steps=1)
    new = rc.get_weights()
    grads, want_loss = ref.gradients(w, torch.from_numpy(s), BOX)
    assert abs(loss - want_loss) <= 1e-3 * want_loss
    for l, (w0, w1, g) in enumerate(zip(w, new, grads)):
        got = (w0.astype(np.float64) - w1.astype(np.float64))
        g = g.numpy()
        rel = np.linalg.norm(got - g) / np.linalg.norm(g)
        assert rel < 0.02, (l, rel)


def test_training_reduces_loss(cuda):
    rc = RadianceCache(rc_default_params(learning_rate=1e-2))
    s = torch.from_numpy(random_samples(1 << 14, seed=7, smooth_target=True)).cuda()
    first = rc.train(s, BOX, steps=1)
    for _ in range(300):
        last = rc.train(s, BOX, steps=4)
    assert last < 0.1 * first
    pred = rc.infer(s, BOX).cpu().numpy()
    t = s.cpu().numpy()[:, [3, 7, 11]]
    assert np.abs(pred - t).mean() < 0.05


def cornell_like(n=30_000, seed=3):
    tris, infos = cpt.scene_random(n, seed=seed)
    cam = cpt.camera_look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.0), aspect=96 / 64)
    return tris, infos, cam


def views_of(tris, infos, cam, w=96, h=64):
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris), check_root=True)
    sc = DeviceScene(infos)
    return [(lb, sc, cam, w, h)], (lb, sc)


def training_path(pixel, frame, stride):
    """Host restatement of the renderer's training-path choice (render.cu training_path)."""
    m = 0xFFFFFFFF
    h = ((pixel * 0x9E3779B1) & m) ^ (((frame + 0x7F4A7C15) & m) * 0x85EBCA77 & m)
    h ^= h >> 16
    h = (h * 0x7FEB352D) & m
    h ^= h >> 15
    h = (h * 0x846CA68B) & m
    h ^= h >> 16
    return h % stride == 0


def test_zero_network_image_is_cut_paths_plus_training_paths(cuda):
    """With a zero network, a cached 1-sample frame is, pixel by pixel, the plain
    depth-2 estimate (paths cut at vertex 1, remainder 0) or — for the training paths
    picked by the (pixel, sample) hash — the plain full-depth estimate."""
    tris, infos, cam = cornell_like()
    views, keep = views_of(tris, infos, cam)
    rc = RadianceCache(rc_default_params(learning_rate=0.0, train_samples=512))
    rc.set_weights([np.zeros((fi, fo), np.float32) for fi, fo in ref.LAYERS])
    frame, bounces = 7, 5
    cr = CachedRenderer(rc, views, make_params(96, 64, 1, frame, bounces, 3.0, True, 11, cpt.ACCUM_KAHAN))
    cr.render()
    torch.cuda.synchronize()
    cr.check_status()

    def plain(b):
        r = BatchRenderer(views, make_params(96, 64, 1, frame, b, 3.0, True, 11, cpt.ACCUM_KAHAN))
        r.render()
        torch.cuda.synchronize()
        return r.accums[0].cpu().numpy().view(np.float32).reshape(2, 64, 96, 4)[0]

    cut, full = plain(1), plain(bounces)
    stride = (96 * 64) // 512
    sel = np.array([[training_path(y * 96 + x, frame, stride) for x in range(96)] for y in range(64)])
    assert 300 < sel.sum() < 800
    want = np.where(sel[..., None], full, cut)
    got = cr.accums[0].cpu().numpy().view(np.float32).reshape(2, 64, 96, 4)[0]
    assert got.tobytes() == want.tobytes()
    # the training paths that reached vertex 1 gave this frame's training samples
    assert 0 < rc.sample_count() <= sel.sum()


def test_training_targets_are_path_suffixes(cuda):
    # with bounces = 2 the suffix is a single term a2 L2 >= 0; its mean over the
    # training paths equals the plain depth-3 minus depth-2 radiance per unit weight
    tris, infos, cam = cornell_like()
    views, keep = views_of(tris, infos, cam)
    rc = RadianceCache(rc_default_params(learning_rate=0.0))
    cr = CachedRenderer(rc, views, make_params(96, 64, 1, 0, 2, 3.0, True, 5, cpt.ACCUM_KAHAN))
    cr.render()
    torch.cuda.synchronize()
    s = rc.samples()
    assert len(s) > 500  # every path of this small frame is a training path; those reaching vertex 1
    t = s[:, [3, 7, 11]]
    assert np.all(t >= 0) and np.isfinite(t).all()
    assert (t > 0).any()
    # positions lie in the scene box, directions and normals are unit vectors
    lo, hi = cpt.scene_bounds(tris)[:3] - 1e-3, cpt.scene_bounds(tris)[3:] + 1e-3
    assert np.all((s[:, 0:3] >= lo) & (s[:, 0:3] <= hi))
    np.testing.assert_allclose(np.linalg.norm(s[:, 4:7], axis=1), 1.0, atol=1e-3)


def test_bounces_below_two_render_plain(cuda):
    tris, infos, cam = cornell_like()
    views, keep = views_of(tris, infos, cam)
    rc = RadianceCache()
    p = make_params(96, 64, 2, 3, 1, 3.0, True, 9, cpt.ACCUM_KAHAN)
    cr = CachedRenderer(rc, views, p)
    cr.render()
    plain = BatchRenderer(views, p)
    plain.render()
    torch.cuda.synchronize()
    assert cr.accums[0].cpu().numpy().tobytes() == plain.accums[0].cpu().numpy().tobytes()


def test_trained_cache_agrees_with_plain_in_the_mean(cuda):
    tris, infos, cam = cornell_like()
    views, keep = views_of(tris, infos, cam)
    # 4 samples per frame, one path in six a training path
    rc = RadianceCache(rc_default_params(train_samples=4096))
    bounces = 4
    cr = CachedRenderer(rc, views, make_params(96, 64, 4, 0, bounces, 3.0, True, 21, cpt.ACCUM_KAHAN))
    for f in range(60):          # train on 60 frames, then start a fresh image
        cr.render(frame0=4 * f)
    cr.accums[0].zero_()
    for f in range(60, 124):
        cr.render(frame0=4 * f)
    plain = BatchRenderer(views, make_params(96, 64, 256, 0, bounces, 3.0, True, 33, cpt.ACCUM_KAHAN))
    plain.render()
    torch.cuda.synchronize()
    cr.check_status()

    def mean_image(acc):
        a = acc.cpu().numpy().view(np.float32).reshape(2, 64, 96, 4)[0]
        return a[..., :3] / np.maximum(a[..., 3:4], 1)

    mc, mp = mean_image(cr.accums[0]).mean(), mean_image(plain.accums[0]).mean()
    assert abs(mc - mp) <= 0.05 * mp, (mc, mp)
