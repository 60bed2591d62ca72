"""LBVH build on the GPU against the oracle and the reference's golden outputs.
Bit-exact: keys, sorted triangles, children, parents, boxes. The compact
traversal records are checked against the reference-format arrays."""
import numpy as np
import pytest
import torch

import cpt
from conftest import GOLDEN_CASES, load_golden, quantized
from cpt.device import DeviceLbvh, to_device
from oracle import cpu

pytestmark = pytest.mark.gpu


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def gpu_build(tris, bits, box=None, check=True, in_place=False):
    lb = DeviceLbvh(len(tris), bits)
    src = to_device(tris)
    if in_place:
        torch.cuda.synchronize()
        lb.mem[: src.numel()].copy_(src)  # bvh.tris is the first array of the allocation
        assert lb.bvh.tris == lb.mem.data_ptr()
        lb.build(lb.bvh.tris, box=box, check_root=check)
    else:
        lb.build(src, box=box, check_root=check)
    torch.cuda.synchronize()
    return lb, lb.download()


def assert_same_as(out, ref):
    for k in ("keys", "tris", "children", "parents_leaf", "parents_internal", "node_boxes"):
        want = ref[k] if isinstance(ref, dict) else getattr(ref, k)
        assert same_bits(out[k], want), k


def leaf_boxes(tris):
    v = np.stack([tris["v0"], tris["v1"], tris["v2"]], 1)  # (n, 3, 3)
    mn = np.full((len(tris), 3), np.finfo(np.float32).max, np.float32)
    mx = np.full((len(tris), 3), -np.finfo(np.float32).max, np.float32)
    for k in range(3):  # glm::min(x, y) = x < y ? x : y, applied v0, v1, v2 in order
        mn = np.where(mn < v[:, k], mn, v[:, k])
        mx = np.where(mx > v[:, k], mx, v[:, k])
    return mn, mx


def assert_records_consistent(out):
    """96-B node = [left slot | right slot | Node word | right index | pad]; a slot is
    the child's box padded with zeros (internal child) or the child triangle as v0,
    its index, v1 - v0, v2 - v0 (leaf child)."""
    n = len(out["tris"])
    nodes, ch = out["nodes"], out["children"]
    assert nodes.shape == (n - 1, 24)
    assert same_bits(nodes[:, 20].view(np.uint32), ch)
    assert same_bits(nodes[:, 21].view(np.uint32), (ch >> 2) + 1)
    t = out["tris"]
    tri_slot = np.zeros((n, 10), np.float32)
    tri_slot[:, 0:3] = t["v0"]
    tri_slot[:, 3] = np.arange(len(t), dtype=np.uint32).view(np.float32)
    tri_slot[:, 4:7] = (t["v1"] - t["v0"]).astype(np.float32)
    tri_slot[:, 7:10] = (t["v2"] - t["v0"]).astype(np.float32)
    box_slot = np.zeros((n - 1, 10), np.float32)
    box_slot[:, 0:3] = out["node_boxes"]["min"]
    box_slot[:, 3:6] = out["node_boxes"]["max"]
    li = ch >> 2
    for side, col in ((0, slice(0, 10)), (1, slice(10, 20))):
        idx = li + side
        internal = ((ch >> side) & 1) == 1
        want = np.where(internal[:, None], box_slot[np.minimum(idx, n - 2)], tri_slot[idx])
        assert same_bits(nodes[:, col], want)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_build_matches_golden(cuda, name):
    g = load_golden(name)
    _, out = gpu_build(g["tris_in"], int(g["bits"]), box=g["box"])
    assert_same_as(out, g)
    assert_records_consistent(out)


@pytest.mark.parametrize("bits", [30, 63])
@pytest.mark.parametrize("n", [2, 3, 17, 4095, 4096, 4097, 100_000])
def test_build_matches_oracle_sizes(cuda, bits, n):
    tris = cpt.scene_random(max(n - 2, 0), seed=n)[0] if n >= 2 else None
    tris = tris[:n]
    _, out = gpu_build(tris, bits)
    assert_same_as(out, cpu.build(tris, bits))
    assert_records_consistent(out)


@pytest.mark.parametrize("bits", [30, 63])
def test_build_tie_heavy_is_stable(cuda, bits):
    # 200k triangles drawn (with repetition) from 2k distinct ones: at most 2k
    # distinct keys; equal keys must keep their input order (stable sort).
    base = cpt.scene_random(2000, seed=4)[0]
    pick = np.random.default_rng(4).integers(0, len(base), 200_000)
    tris = base[pick].copy()
    tris["info_idx"] = np.arange(len(tris), dtype=np.uint32)
    _, out = gpu_build(tris, bits)
    ref = cpu.build(tris, bits)
    assert len(np.unique(ref.keys)) <= 2002
    assert_same_as(out, ref)
    assert_records_consistent(out)


@pytest.mark.parametrize("bits", [30, 63])
def test_build_large_sphere_hairball(cuda, bits):
    tris = cpt.scene_sphere_hairball(512, 256, 200_000, seed=8)[0]
    _, out = gpu_build(tris, bits)
    assert_same_as(out, cpu.build(tris, bits))
    assert_records_consistent(out)


def test_build_device_box_equals_host_box(cuda):
    tris = cpt.scene_random(50_000, seed=5)[0]
    _, a = gpu_build(tris, 63, box=None)
    _, b = gpu_build(tris, 63, box=cpu.enclosing_box(tris))
    for k in ("keys", "tris", "children", "node_boxes"):
        assert same_bits(a[k], b[k])


def test_build_in_place_like_the_reference(cuda):
    tris = cpt.scene_random(30_000, seed=6)[0]
    _, out = gpu_build(tris, 30, in_place=True)
    assert_same_as(out, cpu.build(tris, 30))


def test_build_repeat_is_deterministic(cuda):
    tris = cpt.scene_sphere_hairball(256, 128, 50_000, seed=2)[0]
    lb = DeviceLbvh(len(tris), 63)
    src = to_device(tris)
    outs = []
    for _ in range(3):
        lb.build(src, check_root=True)
        outs.append(lb.download())
    for k in outs[0]:
        assert same_bits(outs[0][k], outs[1][k]) and same_bits(outs[0][k], outs[2][k])


def test_nonfinite_vertex_is_reported(cuda):
    tris = cpt.scene_random(5000, seed=1)[0]
    tris[1234]["v1"][2] = np.nan
    lb = DeviceLbvh(len(tris), 30)
    with pytest.raises(cpt.CptError) as e:
        lb.build(to_device(tris), box=np.array([0, 0, 0, 1, 1, 1], np.float32), check_root=True)
    assert e.value.code == cpt.ERR_NONFINITE_INPUT


def test_wrong_enclosing_box_fails_the_root_check(cuda):
    tris = cpt.scene_random(5000, seed=1)[0]
    lb = DeviceLbvh(len(tris), 30)
    box = cpu.enclosing_box(tris)
    box[3] += 0.5
    with pytest.raises(cpt.CptError) as e:
        lb.build(to_device(tris), box=box, check_root=True)
    assert e.value.code == cpt.ERR_CHECK_FAILED


def test_flat_scene_zero_extent_axis(cuda):
    """All vertices at z = 0.1: scale.z = 0, 1/scale = inf; the GPU quantizer
    saturates (cvt.rzi), which the oracle follows."""
    tris = cpt.scene_random(3000, seed=2)[0]
    for f in ("v0", "v1", "v2"):
        tris[f][:, 2] = np.float32(0.1)
    _, out = gpu_build(tris, 30, check=False)
    assert_same_as(out, cpu.build(tris, 30))
