"""Split traversal BVH (cpt_lbvh_split) on the GPU: the same closest hits as the
LBVH it is built from (the oracle's restatement of the reference traversal) —
identical (t, u, v, triangle) except where two triangles are hit at exactly the
same t — fewer node visits on long thin triangles, bit-identical images on the
test scenes, and the reference-format outputs left untouched."""
import numpy as np
import pytest
import torch

import cpt
from cpt.device import BatchRenderer, DeviceLbvh, DeviceScene, make_params, to_device
from oracle import cpu

pytestmark = pytest.mark.gpu


def hairball(n_hair=20_000, nu=64, nv=32, seed=3):
    return cpt.scene_sphere_hairball(nu, nv, n_hair, seed=seed, hair_radius=1.3)


def random_rays(m, seed=1, inside=False):
    g = np.random.default_rng(seed)
    if inside:
        o = g.uniform(-1.2, 1.2, (m, 3))
    else:
        d0 = g.normal(size=(m, 3))
        o = 3.0 * d0 / np.linalg.norm(d0, axis=1, keepdims=True)
    tgt = g.uniform(-1.0, 1.0, (m, 3))
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((m, 8), np.float32)
    r[:, 0:3] = o
    r[:, 4:7] = d
    return r


def tie_or_equal(h_split, h_ref, ulps=1):
    """Same hit, or hits whose t agree within `ulps` units in the last place: the
    closest of two triangles whose distances are that close depends on the order in
    which the trees visit them (the box entry distance and a triangle's computed t
    differ by rounding)."""
    same = h_split.view(np.uint32) == h_ref.view(np.uint32)
    all_same = same.all(axis=1)
    tr = h_ref[:, 0].astype(np.float64)
    with np.errstate(over="ignore"):  # misses carry FLT_MAX, whose spacing overflows
        ulp = np.spacing(np.abs(h_ref[:, 0])).astype(np.float64)
    near = np.abs(h_split[:, 0].astype(np.float64) - tr) <= ulps * ulp
    return all_same | near, all_same


@pytest.mark.parametrize("bits", [30, 63])
@pytest.mark.parametrize("ratio", [0.5, 2.0])
@pytest.mark.parametrize("flags", [0, cpt.SPLIT_TREELET])
def test_split_hits_match_oracle(cuda, bits, ratio, flags):
    tris, _ = hairball()
    lb = DeviceLbvh(len(tris), bits)
    lb.build(to_device(tris), check_root=True)
    before = lb.download()
    rays = np.concatenate([random_rays(20_000, 1), random_rays(10_000, 2, inside=True)])
    d_rays = torch.from_numpy(rays).cuda()
    base_hits, base_stats = lb.trace(d_rays, stats=True)
    lb.split(ratio, flags=flags)
    split_hits, split_stats = lb.trace(d_rays, stats=True)
    torch.cuda.synchronize()
    lb.status()
    hs, hb = split_hits.cpu().numpy(), base_hits.cpu().numpy()
    ok, exact = tie_or_equal(hs, hb)
    assert ok.all()
    assert exact.mean() > 0.999
    # the oracle's restatement of the reference traversal agrees with the LBVH path
    b = cpu.build(tris, bits)
    t, idx, uv = cpu.trace(b, rays[:, [0, 1, 2, 4, 5, 6]])
    ok2, _ = tie_or_equal(hs, np.stack([t, uv[:, 0], uv[:, 1], idx.view(np.float32)], 1))
    assert ok2.all()
    # any-hit agrees on occlusion
    a_split, _ = lb.trace(d_rays, any_hit=True)
    lb.unsplit()
    a_base, _ = lb.trace(d_rays, any_hit=True)
    assert np.array_equal(a_split.cpu().numpy()[:, 0] < 3e38, a_base.cpu().numpy()[:, 0] < 3e38)
    # fewer visits on the hairball; reference-format outputs untouched
    v_split, v_base = split_stats.cpu().numpy()[:, 0].mean(), base_stats.cpu().numpy()[:, 0].mean()
    assert v_split < (0.95 if ratio >= 2.0 else 1.0) * v_base, (v_split, v_base)
    after = lb.download()
    for k in ("tris", "keys", "children", "parents_leaf", "parents_internal", "node_boxes", "nodes"):
        assert after[k].tobytes() == before[k].tobytes(), k


@pytest.mark.parametrize("flags", [0, cpt.SPLIT_TREELET])
def test_split_render_matches_plain(cuda, flags):
    tris, infos = hairball(n_hair=30_000)
    cam = cpt.camera_look_at((0.0, 0.35, -3.6), (0.0, 0.0, 0.0), aspect=64 / 48)
    lb = DeviceLbvh(len(tris), 63)
    lb.build(to_device(tris), check_root=True)
    sc = DeviceScene(infos)
    p = make_params(64, 48, 8, 3, 5, 3.0, True, 17, cpt.ACCUM_KAHAN)
    r0 = BatchRenderer([(lb, sc, cam, 64, 48)], p)
    r0.render()
    lb.split(1.0, flags=flags)
    r1 = BatchRenderer([(lb, sc, cam, 64, 48)], p)
    r1.render()
    torch.cuda.synchronize()
    r1.check_status()
    a0 = r0.accums[0].cpu().numpy().view(np.float32)
    a1 = r1.accums[0].cpu().numpy().view(np.float32)
    differ = (a0.view(np.uint32) != a1.view(np.uint32)).reshape(2, 48, 64, 4)[0].any(-1)
    assert differ.mean() < 0.002   # only pixels whose path met an exact tie may differ
    assert np.array_equal(r0.counts.cpu().numpy()[:3] > 0, r1.counts.cpu().numpy()[:3] > 0)
    # a new build drops the split tree of the old triangles
    lb.build(to_device(tris))
    assert not lb.bvh.split_nodes and lb.bvh.split_capacity == 0


@pytest.mark.parametrize("flags", [0, cpt.SPLIT_TREELET])
def test_split_degenerate_and_zero_budget(cuda, flags):
    # ratio 0: one piece per triangle; a flat scene (zero extent on an axis) where every
    # hit is a near-tie between coplanar triangles
    tris, _ = cpt.scene_random(5000, seed=9)
    tris["v0"][:, 2] = tris["v1"][:, 2] = tris["v2"][:, 2] = 0.5
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris))
    rays = random_rays(5000, 4)
    rays[:, 4:7] = np.array([0.1, 0.2, 1.0]) / np.linalg.norm([0.1, 0.2, 1.0])
    rays[:, 0:3] = np.random.default_rng(5).uniform(0, 1, (5000, 3)) - np.array([0, 0, 1.0])
    d_rays = torch.from_numpy(rays.astype(np.float32)).cuda()
    h0, _ = lb.trace(d_rays)
    lb.split(0.0, flags=flags)
    h1, _ = lb.trace(d_rays)
    torch.cuda.synchronize()
    lb.status()
    a, b = h1.cpu().numpy(), h0.cpu().numpy()
    ok, _ = tie_or_equal(a, b, ulps=4)
    assert ok.all()
    assert np.array_equal(a[:, 0] < 3e38, b[:, 0] < 3e38)


@pytest.mark.parametrize("flags", [0, cpt.SPLIT_TREELET])
def test_split_on_identical_boxes(cuda, flags):
    # every piece the same box (all Morton keys equal, every treelet cost a tie): the
    # split tree's hits are those of the LBVH
    tri = np.zeros(1, cpt.TRIANGLE_DTYPE)
    tri["v0"], tri["v1"], tri["v2"] = (0.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0)
    tris = np.repeat(tri, 3000)
    tris["info_idx"] = np.arange(3000, dtype=np.uint32)
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris))
    rays = np.zeros((1000, 8), np.float32)
    rays[:, 0:2] = np.random.default_rng(2).uniform(-0.2, 0.8, (1000, 2))
    rays[:, 2] = -1.0
    rays[:, 6] = 1.0
    d_rays = torch.from_numpy(rays).cuda()
    h0, _ = lb.trace(d_rays)
    lb.split(0.0, flags=flags)
    h1, _ = lb.trace(d_rays)
    torch.cuda.synchronize()
    lb.status()
    a, b = h1.cpu().numpy(), h0.cpu().numpy()
    assert np.array_equal(a[:, 0], b[:, 0])  # same t; any of the identical triangles may be reported


def split_tree(lb):
    """Walks the split tree's 96-B records from the root, level by level: returns the
    reached internal node indices, the leaf triangles (with multiplicity), the height,
    the summed half surface area of the internal child boxes, and whether every
    internal child's box lies inside its parent's and every leaf triangle's box meets
    its parent's."""
    raw = lb.split_nodes.cpu().numpy()
    rec = raw[: (raw.size // 96) * 96].view(np.float32).reshape(-1, 24)
    words = rec[:, 20].view(np.uint32)
    right = rec[:, 21].view(np.uint32)
    frontier = np.array([0], np.int64)
    pbox = np.array([[-np.inf] * 3 + [np.inf] * 3], np.float32)
    reached, leaves, height, area, contained = [], [], 0, 0.0, True
    while frontier.size:
        reached.append(frontier)
        height += 1
        w = words[frontier]
        nxt, nbox = [], []
        for side in (0, 1):
            internal = ((w >> side) & 1).astype(bool)
            idx = (w >> 2) if side == 0 else right[frontier]
            slot = rec[frontier, 10 * side:10 * side + 10]
            b = slot[internal, :6]
            pb = pbox[internal]
            contained &= bool(np.all(b[:, :3] >= pb[:, :3]) and np.all(b[:, 3:] <= pb[:, 3:]))
            ext = b[:, 3:].astype(np.float64) - b[:, :3]
            area += float((ext[:, 0] * ext[:, 1] + ext[:, 1] * ext[:, 2] + ext[:, 2] * ext[:, 0]).sum())
            nxt.append(idx[internal].astype(np.int64))
            nbox.append(b)
            lf = slot[~internal]
            v0 = lf[:, 0:3]
            tri = np.stack([v0, v0 + lf[:, 4:7], v0 + lf[:, 7:10]], 1)
            lo, hi, pl = tri.min(1), tri.max(1), pbox[~internal]
            contained &= bool(np.all(lo <= pl[:, 3:] + 1e-6) and np.all(hi >= pl[:, :3] - 1e-6))
            leaves.append(lf[:, 3].view(np.uint32))
        frontier = np.concatenate(nxt)
        pbox = np.concatenate(nbox) if frontier.size else pbox[:0]
    return np.concatenate(reached), np.sort(np.concatenate(leaves)), height, area, contained


@pytest.mark.parametrize("bits,ratio", [(63, 1.0), (30, 0.0)])
def test_treelet_tree_structure(cuda, bits, ratio):
    # restructuring keeps every piece exactly once, every node reachable once, boxes
    # nested, never a taller tree, and lowers the summed node surface area; and its
    # result does not depend on timing (two builds are byte-identical)
    tris, _ = hairball(n_hair=20_000)
    lb = DeviceLbvh(len(tris), bits)
    lb.build(to_device(tris), check_root=True)
    lb.split(ratio)
    torch.cuda.synchronize()
    lb.status()
    r0, l0, h0, a0, c0 = split_tree(lb)
    lb.split(ratio, flags=cpt.SPLIT_TREELET)
    torch.cuda.synchronize()
    lb.status()
    raw1 = lb.split_nodes.cpu().numpy().copy()
    r1, l1, h1, a1, c1 = split_tree(lb)
    assert c0 and c1
    assert np.array_equal(l0, l1)
    assert r1.size == l1.size - 1 and np.unique(r1).size == r1.size
    assert np.array_equal(np.sort(r1), np.arange(r1.size))
    assert h1 <= h0
    assert a1 < 0.99 * a0, (a1, a0)
    lb.split(ratio, flags=cpt.SPLIT_TREELET)
    torch.cuda.synchronize()
    raw2 = lb.split_nodes.cpu().numpy()
    used = r1.size * 96
    assert raw2[:used].tobytes() == raw1[:used].tobytes()


def test_treelet_flag_checks(cuda):
    tris, _ = hairball(n_hair=2_000, nu=16, nv=8)
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris))
    with pytest.raises(ValueError):
        lb.split(1.0, flags=cpt.SPLIT_TREELET | 1)
    with pytest.raises(ValueError):
        lb.split(1.0, flags=8)
    # two and three triangles: no treelet of 3 leaves or fewer to improve; hits still match
    for count in (2, 3):
        small = tris[:count].copy()
        lb2 = DeviceLbvh(count, 30)
        lb2.build(to_device(small))
        rays = random_rays(2000, 7)
        d_rays = torch.from_numpy(rays).cuda()
        h0, _ = lb2.trace(d_rays)
        lb2.split(2.0, flags=cpt.SPLIT_TREELET)
        h1, _ = lb2.trace(d_rays)
        torch.cuda.synchronize()
        lb2.status()
        ok, _ = tie_or_equal(h1.cpu().numpy(), h0.cpu().numpy())
        assert ok.all()


@pytest.mark.parametrize("bits", [30, 63])
def test_treelet_matches_oracle(cuda, bits):
    # one piece per triangle (ratio 0): the leaves' boxes are their triangles' boxes, so
    # the oracle's restatement (oracle/cpt_treelet.c) can restructure the GPU's Karras
    # split tree and must reproduce the GPU's restructured records: the same words, and
    # the same box and triangle floats (as values: the sign of a zero may differ)
    tris, _ = hairball(n_hair=20_000)
    n = len(tris)
    lb = DeviceLbvh(n, bits)
    lb.build(to_device(tris), check_root=True)
    lb.split(0.0)
    torch.cuda.synchronize()
    lb.status()
    rec0 = lb.split_nodes.cpu().numpy()[: (n - 1) * 96].view(np.float32).reshape(n - 1, 24).copy()
    lb.split(0.0, flags=cpt.SPLIT_TREELET)
    torch.cuda.synchronize()
    lb.status()
    rec1 = lb.split_nodes.cpu().numpy()[: (n - 1) * 96].view(np.float32).reshape(n - 1, 24).copy()
    srt = lb.download()["tris"]
    lo = np.minimum(np.minimum(srt["v0"], srt["v1"]), srt["v2"])
    hi = np.maximum(np.maximum(srt["v0"], srt["v1"]), srt["v2"])
    words, right = rec0[:, 20].view(np.uint32), rec0[:, 21].view(np.uint32)
    leaf_boxes = np.full((n, 6), np.nan, np.float32)
    for side in (0, 1):
        leaf = ((words >> side) & 1) == 0
        ids = ((words >> 2) if side == 0 else right)[leaf]
        tri = rec0[leaf, 10 * side + 3].view(np.uint32)
        leaf_boxes[ids] = np.concatenate([lo[tri], hi[tri]], 1)
    assert not np.isnan(leaf_boxes).any()
    want = cpu.treelet(rec0, n, leaf_boxes, 4)
    assert (want.view(np.uint32) != rec0.view(np.uint32)).any()  # the restructuring changed something
    assert np.array_equal(rec1[:, 20:24].view(np.uint32), want[:, 20:24].view(np.uint32))
    assert np.array_equal(rec1[:, :20], want[:, :20])
