"""The reference's own GPU LBVH build — CUDA::BVHBuilder::build with its thrust sort
and kernels (BVHBuilder.cu:207-269), compiled from its sources for sm_100a into
oracle/_ref/librefgpu.so — against this library's build of the same triangles at
the same 30-bit key width, on the same B200: sorted triangles, Node words, both
parent arrays and the internal-node boxes."""
import numpy as np
import pytest

import cpt
from conftest import quantized
from cpt.device import DeviceLbvh, to_device
from oracle import cpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["random", "ties", "sphere"])
def test_reference_gpu_build_equals_ours(cuda, case):
    if not cpu.refgpu_available():
        pytest.fail("oracle/_ref/librefgpu.so was not built (make -C oracle ref)")
    if case == "random":
        tris = cpt.scene_random(200_000, seed=3)[0]
    elif case == "ties":  # many equal Morton keys: the sort's tie order matters
        tris = quantized(cpt.scene_random(100_000, seed=4)[0], 1.0 / 64)
    else:
        tris = cpt.scene_sphere_hairball(256, 128, 30_000, seed=5)[0]
    box = cpu.enclosing_box(tris)
    stats, ref = cpu.refgpu_build(tris, box=box, reps=1, outputs=True)
    assert stats["ms_mean"] > 0
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris), box=box, check_root=True)
    out = lb.download()
    for k in ("tris", "children", "parents_leaf", "parents_internal"):
        assert np.ascontiguousarray(out[k]).tobytes() == np.ascontiguousarray(getattr(ref, k)).tobytes(), k
    # boxes: the reference's refit reads its sibling's box with no fence after the
    # counter (BVHBuilder.cu:63-86); a stale read would show here as a differing box
    differ = (out["node_boxes"].view(np.uint32).reshape(-1, 6) != ref.node_boxes.view(np.uint32).reshape(-1, 6))
    assert not differ.any(), f"{int(differ.any(1).sum())} internal boxes differ"
