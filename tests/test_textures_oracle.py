"""The oracle's restatement of the reference's texture sampler (normalized
coordinates, wrap addressing, bilinear filtering of RGBA8 read as [0, 1] floats;
Scene.cu:57-81) on the CPU: texel centres return the texel, the pattern repeats
with period 1 in u and v, a corner averages the four wrapped corner texels, and
the filter weights sit on the 1/256 grid of the hardware's fixed-point weights."""
import numpy as np

from oracle import cpu


def image(h=4, w=8, seed=0):
    return np.random.default_rng(seed).integers(0, 256, (h, w, 4), dtype=np.uint8)


def test_texel_centres_return_the_texel():
    im = image()
    h, w = im.shape[:2]
    uv = np.array([[(i + 0.5) / w, (j + 0.5) / h] for j in range(h) for i in range(w)], np.float32)
    np.testing.assert_array_equal(np.rint(cpu.tex_sample(im, uv) * 255), im.reshape(-1, 4))


def test_wrap_is_periodic():
    im = image(5, 7, seed=1)
    uv = np.random.default_rng(2).random((500, 2)).astype(np.float32) * 0.9 + 0.05
    base = cpu.tex_sample(im, uv)
    for shift in (1.0, -1.0, 3.0):
        np.testing.assert_allclose(cpu.tex_sample(im, uv + np.float32(shift)), base, atol=2e-6)


def test_corner_averages_wrapped_corners():
    im = image(6, 10, seed=3)
    got = cpu.tex_sample(im, np.zeros((1, 2), np.float32))[0]
    want = im[[0, 0, -1, -1], [0, -1, 0, -1]].astype(np.float64).mean(0) / 255
    np.testing.assert_allclose(got, want, atol=1e-7)


def test_weights_on_the_fixed_point_grid():
    # two texels 0 and 255 in u: the filtered value is the weight itself, a
    # multiple of 1/256 (9-bit weight, 8 fraction bits)
    im = np.zeros((1, 2, 4), np.uint8)
    im[0, 1] = 255
    u = np.linspace(0.25, 0.75, 301, dtype=np.float32)
    uv = np.stack([u, np.full_like(u, 0.5)], 1)
    a = cpu.tex_sample(im, uv)[:, 0].astype(np.float64)
    np.testing.assert_allclose(a * 256, np.rint(a * 256), atol=1e-4)
    assert np.all(np.diff(a) >= 0) and a[0] == 0.0 and a[-1] == 1.0
