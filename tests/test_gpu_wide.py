"""Compressed 8-wide traversal BVH (cpt_lbvh_wide) on the GPU: the closest hits of
the binary tree it collapses (the LBVH — the oracle's restatement of the reference
traversal — or the split tree), identical (t, u, v, triangle) except where two
triangles are hit at exactly the same t; the same occlusion for any-hit and far-limited
rays; images equal to the binary tree's up to such ties; counts of the tree written
to the status words; a rebuild or split drops the stale wide tree."""
import numpy as np
import pytest
import torch

import cpt
from cpt.device import BatchRenderer, DeviceLbvh, DeviceScene, make_params, to_device
from oracle import cpu
from test_gpu_split import hairball, random_rays, tie_or_equal

pytestmark = pytest.mark.gpu


def trace_pair(lb, d_rays):
    h, st = lb.trace(d_rays, stats=True)
    a, _ = lb.trace(d_rays, any_hit=True)
    torch.cuda.synchronize()
    lb.status()
    return h.cpu().numpy(), st.cpu().numpy(), a.cpu().numpy()


@pytest.mark.parametrize("sah", [False, True])
@pytest.mark.parametrize("bits", [30, 63])
@pytest.mark.parametrize("split,flags", [(0.0, 0), (1.25, 0), (1.25, cpt.SPLIT_TREELET)])
def test_wide_hits_match_binary(cuda, bits, split, flags, sah):
    """Both collapses (largest child first; surface-area cost, CPT_WIDE_SAH) over the LBVH
    and over split trees, whose node arrays hold more records than the tree uses."""
    tris, _ = hairball()
    lb = DeviceLbvh(len(tris), bits)
    lb.build(to_device(tris), check_root=True)
    if split:
        lb.split(split, flags=flags)
    rays = np.concatenate([random_rays(20_000, 1), random_rays(10_000, 2, inside=True)])
    d_rays = torch.from_numpy(rays).cuda()
    hb, sb, ab = trace_pair(lb, d_rays)
    lb.wide(sah=sah)
    hw, sw, aw = trace_pair(lb, d_rays)
    ok, exact = tie_or_equal(hw, hb)
    assert ok.all()
    assert exact.mean() > 0.999
    assert np.array_equal(aw[:, 0] < 3e38, ab[:, 0] < 3e38)
    # against the oracle's reference traversal as well
    b = cpu.build(tris, bits)
    t, idx, uv = cpu.trace(b, rays[:, [0, 1, 2, 4, 5, 6]])
    ok2, _ = tie_or_equal(hw, np.stack([t, uv[:, 0], uv[:, 1], idx.view(np.float32)], 1))
    assert ok2.all()
    # fewer node fetches than the binary tree; the counts in the status words
    assert sw[:, 0].mean() < 0.6 * sb[:, 0].mean(), (sw[:, 0].mean(), sb[:, 0].mean())
    leaves = lb.bvh.split_capacity if split else lb.n
    assert lb.bvh.wide_capacity == leaves
    counts = lb.status_words()
    assert 1 <= counts[2] <= leaves - 1 and counts[3] >= 1


def test_wide_far_limit_and_zero_direction(cuda):
    """Rays along the axes (zero direction components) and occlusion tests with a far
    limit (the renderer's shadow rays) agree with the binary tree."""
    tris, _ = cpt.scene_random(20_000, seed=4)
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris))
    g = np.random.default_rng(8)
    m = 6000
    rays = np.zeros((m, 8), np.float32)
    rays[:, 0:3] = g.uniform(-0.2, 1.2, (m, 3))
    axis = g.integers(0, 3, m)
    sign = np.where(g.random(m) < 0.5, -1.0, 1.0)
    rays[np.arange(m), 4 + axis] = sign
    d_rays = torch.from_numpy(rays).cuda()
    hb, _, ab = trace_pair(lb, d_rays)
    lb.wide()
    hw, _, aw = trace_pair(lb, d_rays)
    ok, _ = tie_or_equal(hw, hb)
    assert ok.all()
    assert np.array_equal(aw[:, 0] < 3e38, ab[:, 0] < 3e38)
    assert (hb[:, 0] < 3e38).mean() > 0.1


@pytest.mark.parametrize("nee,sah", [(False, False), (True, False), (False, True)])
def test_wide_render_matches_binary(cuda, nee, sah):
    tris, infos = hairball(n_hair=30_000)
    cam = cpt.camera_look_at((0.0, 0.35, -3.6), (0.0, 0.0, 0.0), aspect=64 / 48)
    lb = DeviceLbvh(len(tris), 63)
    lb.build(to_device(tris), check_root=True)
    lb.split(1.25)
    sc = DeviceScene(infos)
    if nee:
        sc.build_emitters(lb)
    p = make_params(64, 48, 8, 3, 5, 3.0, True, 17, cpt.ACCUM_KAHAN, nee=nee)
    r0 = BatchRenderer([(lb, sc, cam, 64, 48)], p)
    r0.render()
    lb.wide(sah=sah)
    r1 = BatchRenderer([(lb, sc, cam, 64, 48)], p)
    r1.render()
    torch.cuda.synchronize()
    r1.check_status()
    a0 = r0.accums[0].cpu().numpy().view(np.uint32).reshape(2, 48, 64, 4)[0]
    a1 = r1.accums[0].cpu().numpy().view(np.uint32).reshape(2, 48, 64, 4)[0]
    differ = (a0 != a1).any(-1)
    assert differ.mean() < 0.002  # only pixels whose path met an exact tie may differ
    assert np.array_equal(r0.counts.cpu().numpy()[:3], r1.counts.cpu().numpy()[:3]) or differ.any()
    # a new split or build drops the wide tree of the old binary tree
    lb.split(1.25)
    assert not lb.bvh.wide_nodes and lb.bvh.wide_capacity == 0
    lb.wide()
    lb.build(to_device(tris))
    assert not lb.bvh.wide_nodes and not lb.bvh.split_nodes


def test_tracer_object_with_wide_tree(cuda):
    """cpt_tracer_set_wide: the tracer builds the wide tree on upload (after the split
    tree; 2: with the surface-area collapse) and its image equals the binary tree's up
    to exact ties."""
    tris, infos = hairball(n_hair=10_000)
    cam = cpt.camera_look_at((0.0, 0.35, -3.6), (0.0, 0.0, 0.0), aspect=64 / 48)
    imgs = []
    for wide in (0, 1, 2):
        t = cpt.Tracer(63)
        t.set_split(2.0)
        t.set_wide(wide)
        t.upload(tris, infos)
        t.set_settings(bounces=3, intensity=3.0, stratified=True, seed=5, accum_mode=cpt.ACCUM_KAHAN)
        t.set_camera(cam)
        t.raytrace(64, 48, 4)
        imgs.append(t.read_image(64, 48))
        b = t.bvh()
        assert b.wide_capacity == (b.split_capacity if wide else 0)
        t.close()
    for img in imgs[1:]:
        differ = (imgs[0].view(np.uint32) != img.view(np.uint32)).any(-1)
        assert differ.mean() < 0.002


def _closest_brute(tris, rays):
    """Closest Moller-Trumbore hit distance of every ray over every triangle, with the
    product's float32 operation order (each operation rounded); inf on a miss."""
    v0 = tris["v0"].astype(np.float32)
    e1 = (tris["v1"] - tris["v0"]).astype(np.float32)
    e2 = (tris["v2"] - tris["v0"]).astype(np.float32)

    def cross(a, b):
        return np.stack([a[..., 1] * b[..., 2] - b[..., 1] * a[..., 2], a[..., 2] * b[..., 0] - b[..., 2] * a[..., 0],
                         a[..., 0] * b[..., 1] - b[..., 0] * a[..., 1]], -1)

    def dot(a, b):
        return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]

    out = np.full(len(rays), np.inf, np.float32)
    eps = np.float32(np.finfo(np.float32).eps)
    with np.errstate(all="ignore"):
        for k in range(len(rays)):
            o, d = rays[k, 0:3], rays[k, 4:7]
            q = cross(np.broadcast_to(d, e2.shape), e2)
            det = dot(e1, q)
            inv = np.float32(1.0) / det
            sv = o - v0
            u = inv * dot(sv, q)
            r = cross(sv, e1)
            v = inv * dot(np.broadcast_to(d, r.shape), r)
            t = inv * dot(e2, r)
            hit = ~((det > -eps) & (det < eps)) & ~(u < 0) & ~(v < 0) & ~((u + v) > 1) & (t >= 0)
            if hit.any():
                out[k] = t[hit].min()
    return out


@pytest.mark.parametrize("distance", [3.0, 1000.0])
def test_wide_far_camera_finds_every_closest_hit(cuda, distance):
    """Rays from far away (the plane distances (p - o) / d round at the scale of the
    distance, not of the scene): the wide tree still returns the brute-force closest
    hit of every ray."""
    tris, _ = cpt.scene_random(20_000, seed=12)
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris))
    lb.wide()
    g = np.random.default_rng(21)
    m = 1000
    d0 = g.normal(size=(m, 3))
    o = 0.5 + distance * d0 / np.linalg.norm(d0, axis=1, keepdims=True)
    tgt = g.uniform(0.0, 1.0, (m, 3))
    dirs = tgt - o
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    rays = np.zeros((m, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 4:7] = dirs
    h, _ = lb.trace(torch.from_numpy(rays).cuda())
    torch.cuda.synchronize()
    lb.status()
    got = h.cpu().numpy()[:, 0]
    want = _closest_brute(tris, rays)
    assert (want < np.inf).mean() > 0.2
    got = np.where(got >= 3e38, np.inf, got)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("distance", [3.0, 1000.0])
@pytest.mark.parametrize("flags", [0, cpt.SPLIT_TREELET])
def test_split_far_camera_finds_every_closest_hit(cuda, distance, flags):
    """The same far-camera check for the binary split tree (pieces of long triangles,
    fused slab test), with the Karras and the treelet-restructured topology."""
    tris, _ = hairball(n_hair=8000, nu=32, nv=16, seed=6)
    lb = DeviceLbvh(len(tris), 63)
    lb.build(to_device(tris))
    lb.split(2.0, flags=flags)
    g = np.random.default_rng(22)
    m = 1000
    d0 = g.normal(size=(m, 3))
    o = distance * d0 / np.linalg.norm(d0, axis=1, keepdims=True)
    tgt = g.uniform(-1.0, 1.0, (m, 3))
    dirs = tgt - o
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    rays = np.zeros((m, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 4:7] = dirs
    h, _ = lb.trace(torch.from_numpy(rays).cuda())
    torch.cuda.synchronize()
    lb.status()
    got = np.where(h.cpu().numpy()[:, 0] >= 3e38, np.inf, h.cpu().numpy()[:, 0])
    want = _closest_brute(tris, rays)
    assert (want < np.inf).mean() > 0.2
    assert np.array_equal(got, want)


def test_wide_batched_views_match_binary(cuda):
    """Several scenes in one call (the per-ray view lookup of the wide kernels): each
    view's image equals its binary-tree image up to exact ties, with and without
    next-event estimation; a call mixing wide and binary views traverses the binary
    trees of all."""
    specs = [(hairball(n_hair=6000, nu=32, nv=16, seed=s), s) for s in (1, 2)]
    views, lbs, scs = [], [], []
    cam = cpt.camera_look_at((0.0, 0.35, -3.6), (0.0, 0.0, 0.0), aspect=1.0)
    for (tris, infos), s in specs:
        lb = DeviceLbvh(len(tris), 63)
        lb.build(to_device(tris))
        lb.split(1.0)
        sc = DeviceScene(infos)
        sc.build_emitters(lb)
        lbs.append(lb)
        scs.append(sc)
        views.append((lb, sc, cam, 40, 40))
    for nee in (False, True):
        p = make_params(0, 0, 4, 0, 4, 3.0, True, 9, cpt.ACCUM_KAHAN, nee=nee)
        for lb in lbs:
            lb.unwide()
        r0 = BatchRenderer(views, p)
        r0.render()
        lbs[0].wide()
        rm = BatchRenderer(views, p)  # mixed: every view traverses its binary tree
        rm.render()
        lbs[1].wide()
        r1 = BatchRenderer(views, p)
        r1.render()
        torch.cuda.synchronize()
        r1.check_status()
        for k in range(2):
            a0 = r0.accums[k].cpu().numpy().view(np.uint32)
            assert a0.tobytes() == rm.accums[k].cpu().numpy().tobytes()
            a1 = r1.accums[k].cpu().numpy().view(np.uint32)
            differ = (a0.reshape(2, 40, 40, 4)[0] != a1.reshape(2, 40, 40, 4)[0]).any(-1)
            assert differ.mean() < 0.003


def test_wide_build_rejects_bad_arguments(cuda):
    """Buffers below cpt_lbvh_wide_bytes, misaligned or missing pointers: an error code
    and no wide tree attached."""
    import ctypes

    tris, _ = cpt.scene_random(3000, seed=2)
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris))
    nb, tb = ctypes.c_size_t(), ctypes.c_size_t()
    sb = int(cpt.lib.cpt_lbvh_wide_bytes(lb.n, 0, ctypes.byref(nb), ctypes.byref(tb)))
    assert sb > 0 and nb.value >= (lb.n - 1) * 80 and tb.value >= lb.n * 48
    assert cpt.lib.cpt_lbvh_wide_bytes(1, 0, None, None) == 0
    assert cpt.lib.cpt_lbvh_wide_bytes(lb.n, 2, None, None) == 0  # an unknown flag
    assert cpt.lib.cpt_lbvh_wide_bytes(lb.n, cpt.WIDE_SAH, None, None) > sb  # the cost tables
    nodes = torch.empty(nb.value, dtype=torch.uint8, device="cuda")
    trs = torch.empty(tb.value, dtype=torch.uint8, device="cuda")
    scr = torch.empty(sb, dtype=torch.uint8, device="cuda")
    b = ctypes.byref(lb.bvh)
    assert cpt.lib.cpt_lbvh_wide(b, 0, nodes.data_ptr(), nb.value - 16, trs.data_ptr(), tb.value, scr.data_ptr(), sb,
                                 0) == cpt.ERR_SCRATCH_TOO_SMALL
    assert cpt.lib.cpt_lbvh_wide(b, 0, nodes.data_ptr(), nb.value, trs.data_ptr(), tb.value, scr.data_ptr(), sb - 1,
                                 0) == cpt.ERR_SCRATCH_TOO_SMALL
    assert cpt.lib.cpt_lbvh_wide(b, 0, nodes.data_ptr() + 4, nb.value, trs.data_ptr(), tb.value, scr.data_ptr(), sb,
                                 0) == cpt.ERR_INVALID_ARGUMENT
    assert cpt.lib.cpt_lbvh_wide(b, 0, None, nb.value, trs.data_ptr(), tb.value, scr.data_ptr(), sb,
                                 0) == cpt.ERR_INVALID_ARGUMENT
    assert cpt.lib.cpt_lbvh_wide(b, cpt.WIDE_SAH, nodes.data_ptr(), nb.value, trs.data_ptr(), tb.value, scr.data_ptr(),
                                 sb, 0) == cpt.ERR_SCRATCH_TOO_SMALL  # the surface-area collapse needs more
    assert not lb.bvh.wide_nodes
    assert cpt.lib.cpt_lbvh_wide(b, 0, nodes.data_ptr(), nb.value, trs.data_ptr(), tb.value, scr.data_ptr(), sb,
                                 0) == 0
    torch.cuda.synchronize()
    lb.status()
    assert lb.bvh.wide_nodes == nodes.data_ptr() and lb.bvh.wide_capacity == lb.n


def test_wide_batch_matches_single_builds(cuda):
    """cpt_lbvh_wide_batch over trees of different kinds and sizes (an LBVH at 30 bits,
    split trees at 63 bits, a five-triangle LBVH): each tree's wide tree has the node and
    record counts of its cpt_lbvh_wide build and gives the binary tree's hits; a second
    batch call after a rebuild gives them again."""
    from cpt.device import WideBatch

    scenes = [(cpt.scene_random(3000, seed=2)[0], 30, 0.0), (hairball(n_hair=20_000)[0], 63, 1.25),
              (cpt.scene_random(20_000, seed=6)[0], 63, 1.25), (cpt.scene_random(5, seed=1)[0], 30, 0.0)]
    lbs, singles = [], []
    for tris, bits, split in scenes:
        lb = DeviceLbvh(len(tris), bits)
        lb.build(to_device(tris), check_root=True)
        if split:
            lb.split(split)
        lb.wide()
        torch.cuda.synchronize()
        singles.append(lb.status_words()[2:4].copy())
        lbs.append(lb)
    for lb in lbs:
        lb.unwide()
    wb = WideBatch(lbs)
    for _ in range(2):
        wb.build()
        torch.cuda.synchronize()
        for (tris, bits, split), lb, counts in zip(scenes, lbs, singles):
            lb.status()
            assert np.array_equal(lb.status_words()[2:4], counts)
            assert lb.bvh.wide_nodes and lb.bvh.wide_capacity == (lb.bvh.split_capacity if split else lb.n)
            rays = random_rays(4000, 3, inside=True)
            d_rays = torch.from_numpy(rays).cuda()
            hw, _, aw = trace_pair(lb, d_rays)
            wide_nodes, wide_tris = lb.bvh.wide_nodes, lb.bvh.wide_tris
            lb.unwide()
            hb, _, ab = trace_pair(lb, d_rays)
            ok, _ = tie_or_equal(hw, hb)
            assert ok.all()
            assert np.array_equal(aw[:, 0] < 3e38, ab[:, 0] < 3e38)
            lb.bvh.wide_nodes, lb.bvh.wide_tris = wide_nodes, wide_tris
            lb.bvh.wide_capacity = lb.bvh.split_capacity if split else lb.n
        for (tris, bits, split), lb in zip(scenes, lbs):  # rebuilt trees drop their wide trees
            lb.build(to_device(tris))
            if split:
                lb.split(split)


def test_wide_sah_collapse_does_not_cost_node_fetches(cuda):
    """The surface-area collapse fetches no more wide nodes per ray than the largest-child
    collapse, within a tenth, on a split hairball (a guard against a cost model that
    lets subtrees too large for one leaf slot compete as leaf slots)."""
    tris, _ = hairball(n_hair=30_000)
    lb = DeviceLbvh(len(tris), 63)
    lb.build(to_device(tris), check_root=True)
    lb.split(1.25)
    d_rays = torch.from_numpy(random_rays(20_000, 5, inside=True)).cuda()
    lb.wide()
    hg, sg, _ = trace_pair(lb, d_rays)
    lb.wide(sah=True)
    hs, ss, _ = trace_pair(lb, d_rays)
    ok, _ = tie_or_equal(hs, hg)
    assert ok.all()
    assert ss[:, 0].mean() <= 1.1 * sg[:, 0].mean(), (ss[:, 0].mean(), sg[:, 0].mean())
