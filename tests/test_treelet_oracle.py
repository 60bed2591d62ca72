"""The treelet restructuring's CPU restatement (oracle/cpt_treelet.c), the checker of
the split tree's k_treelet, on LBVHs built by the oracle: it keeps every leaf once and
every node reachable once, keeps boxes the exact unions of their children's, never makes
the tree taller, lowers the summed node area, and gives the same bytes on every run."""
import numpy as np
import pytest

import cpt
from oracle import cpu


def walk(rec, leaf_boxes):
    """(reached internal nodes, leaf indices, height, summed half area of the internal
    nodes below the root, whether every internal child's box is the union of its
    children's boxes)."""
    words = rec[:, 20].view(np.uint32)
    right = rec[:, 21].view(np.uint32)

    def child_box(node, side):
        w = words[node]
        if (w >> side) & 1:
            return rec[node, 10 * side:10 * side + 6]
        idx = (w >> 2) if side == 0 else right[node]
        return leaf_boxes[idx]

    reached, leaves, exact = [], [], True
    height, area = 0, 0.0
    frontier = [0]
    while frontier:
        height += 1
        nxt = []
        for node in frontier:
            reached.append(node)
            w = words[node]
            for side in (0, 1):
                idx = int((w >> 2) if side == 0 else right[node])
                if (w >> side) & 1:
                    b = rec[node, 10 * side:10 * side + 6].astype(np.float64)
                    e = b[3:] - b[:3]
                    area += e[0] * e[1] + e[1] * e[2] + e[2] * e[0]
                    kids = np.stack([child_box(idx, 0), child_box(idx, 1)])
                    union = np.concatenate([kids[:, :3].min(0), kids[:, 3:].max(0)])
                    exact &= bool(np.array_equal(union, rec[node, 10 * side:10 * side + 6]))
                    nxt.append(idx)
                else:
                    leaves.append(idx)
        frontier = nxt
    return np.array(reached), np.sort(np.array(leaves)), height, area, exact


@pytest.mark.parametrize("gamma", [3, 4, 7])
@pytest.mark.parametrize("bits", [30, 63])
def test_treelet_restatement_properties(bits, gamma):
    tris, _ = cpt.scene_sphere_hairball(32, 16, 1500, seed=5, hair_radius=1.3)
    b = cpu.build(tris, bits)
    rec, leaf_boxes = cpu.records_of(b)
    n = len(tris)
    r0, l0, h0, a0, x0 = walk(rec, leaf_boxes)
    out = cpu.treelet(rec, n, leaf_boxes, gamma)
    r1, l1, h1, a1, x1 = walk(out, leaf_boxes)
    assert x0 and x1
    assert np.array_equal(l0, np.arange(n)) and np.array_equal(l1, l0)
    assert np.array_equal(np.sort(r1), np.arange(n - 1))
    assert h1 <= h0
    assert a1 < 0.97 * a0, (a1, a0)
    changed = (out.view(np.uint32) != rec.view(np.uint32)).any(1)
    assert changed.any()
    assert (out[changed, 22:24] == 0).all()  # rewritten records: last two words cleared
    assert out.tobytes() == cpu.treelet(rec, n, leaf_boxes, gamma).tobytes()


def test_treelet_restatement_small_and_malformed():
    tris, _ = cpt.scene_random(3, seed=2)
    b = cpu.build(tris[:3], 30)
    rec, leaf_boxes = cpu.records_of(b)
    assert cpu.treelet(rec, 3, leaf_boxes, 4).tobytes() == rec.tobytes()  # 3 leaves: below gamma
    bad = rec.copy()
    bad[0, 20] = np.uint32(0xFFFF0001).view(np.float32)  # an internal child index far out of range
    with pytest.raises(ValueError):
        cpu.treelet(bad, 3, leaf_boxes, 2)
