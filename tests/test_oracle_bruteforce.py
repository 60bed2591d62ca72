"""The oracle's traversal against an exhaustive scan of every triangle.

The golden fixtures pin the oracle to the reference's own output; this file checks
the property that output is meant to have: the closest-hit traversal of
trace.h:73-169 returns the nearest Moller-Trumbore hit (intersection.h:28-59) over
the whole soup. The scan restates that triangle test in numpy float32 with the
oracle's operation order (products first, sums left to right, glm's cross), so a
hit distance reached by both is the same float bit for bit.

Where they may differ is fixed by the reference, not by the oracle: the slab test
(intersection.h:106-117) is rounded too, so a ray that grazes a box's face can miss
the box while its triangle's own test hits. The test bounds the share of such rays,
requires that each of them hits its nearest triangle on a face of that triangle's
box, and requires for every ray that the oracle's hit is a real hit of the triangle
it names at the distance it reports, never nearer than the scan's minimum.
"""
import numpy as np
import pytest

import cpt
from conftest import GOLDEN_CASES, load_golden, rays_at
from oracle import cpu

F32 = np.float32
EPS = np.finfo(np.float32).eps


def _dot(a, b):
    x, y, z = a[..., 0] * b[..., 0], a[..., 1] * b[..., 1], a[..., 2] * b[..., 2]
    return (x + y) + z


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - b[..., 1] * a[..., 2],
                     a[..., 2] * b[..., 0] - b[..., 2] * a[..., 0],
                     a[..., 0] * b[..., 1] - b[..., 0] * a[..., 1]], -1)


def mt_all(tris, rays, block=128):
    """(m, n) float32 hit distances of every ray against every triangle, +inf where
    the triangle test misses; same steps and rejections as intersection.h:28-59."""
    p0 = tris["v0"].astype(F32)[None]
    e1 = (tris["v1"].astype(F32) - tris["v0"].astype(F32))[None]
    e2 = (tris["v2"].astype(F32) - tris["v0"].astype(F32))[None]
    out = np.empty((len(rays), len(tris)), F32)
    with np.errstate(all="ignore"):
        for s in range(0, len(rays), block):
            o = rays[s:s + block, None, :3].astype(F32)
            d = rays[s:s + block, None, 3:6].astype(F32)
            q = _cross(d, e2)
            det = _dot(e1, q)
            culled = (det > -EPS) & (det < EPS)
            inv = F32(1.0) / det
            sv = o - p0
            u = inv * _dot(sv, q)
            r = _cross(sv, e1)
            v = inv * _dot(d, r)
            t = inv * _dot(e2, r)
            hit = ~culled & ~(u < 0) & ~((v < 0) | ((u + v) > 1)) & (t >= 0)
            out[s:s + block] = np.where(hit, t, F32(np.inf))
    return out


def _check(tris, rays, max_graze, bits=30):
    b = cpu.build(tris, bits)
    t, idx, _ = cpu.trace(b, rays)
    all_t = mt_all(b.tris, rays)              # b.tris: the Morton-sorted soup that idx indexes
    best = all_t.min(1)
    hit = idx != cpu.INVALID
    # a reported hit is a real hit of the named triangle at exactly the reported distance
    assert np.array_equal(all_t[np.flatnonzero(hit), idx[hit]], t[hit])
    # never nearer than the nearest hit of the whole soup, and a miss reports FLT_MAX
    assert (t[hit] >= best[hit]).all()
    assert (t[~hit] == cpu.FLT_MAX).all()
    # equal to it except on grazing rays the rounded slab test drops: there the nearest
    # hit point lies on a face of its triangle's box (a flat box, for an axis-aligned
    # triangle, is all face), within a few ulps
    agree = np.where(hit, t == best, ~np.isfinite(best))
    bad = np.flatnonzero(~agree)
    assert len(bad) <= max_graze * len(rays), (len(bad), len(rays))
    for i in bad:
        j = int(np.argmin(all_t[i]))
        tri = b.tris[j]
        v = np.stack([tri["v0"], tri["v1"], tri["v2"]]).astype(np.float64)
        p = rays[i, :3].astype(np.float64) + float(best[i]) * rays[i, 3:6].astype(np.float64)
        face = np.minimum(np.abs(p - v.min(0)), np.abs(p - v.max(0)))
        assert face.min() <= 1e-6 * max(1.0, np.abs(p).max()), (i, j, p, v)
    return agree, hit


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_golden_rays_find_the_nearest_hit(name):
    g = load_golden(name)
    # ties1k_30 sits on a coarse grid: many axis-aligned triangles with flat boxes
    agree, hit = _check(g["tris_in"], g["rays"], 2e-2 if name == "ties1k_30" else 2e-3, int(g["bits"]))
    if name != "tiny2_30":
        assert hit.mean() > 0.1  # the scenes are hit often enough for the check to mean something


@pytest.mark.parametrize("bits", [30, 63])
def test_random_scene_finds_the_nearest_hit(bits):
    tris, _ = cpt.scene_random(3000, seed=11)
    rays = rays_at(tris, 4000, seed=12)
    agree, hit = _check(tris, rays, 2e-3, bits)
    assert hit.sum() > 1500


def test_duplicate_and_coplanar_triangles():
    # every triangle three times (identical vertices, so identical distances) plus a
    # coplanar copy shifted in its plane: ties everywhere; the oracle still names a
    # triangle whose own distance is the nearest
    tris, _ = cpt.scene_random(500, seed=3)
    shifted = tris.copy()
    for f in ("v0", "v1", "v2"):
        shifted[f] = (tris[f] + np.float32(0.002) * (tris["v1"] - tris["v0"])).astype(np.float32)
    soup = np.concatenate([tris, tris, shifted, tris])
    rays = rays_at(soup, 2000, seed=4)
    agree, hit = _check(soup, rays, 2e-3)
    assert hit.sum() > 500
