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
from oracle import cpu, refgpu_child

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
    r = refgpu_child.run("build", tris, box, reps=1, outputs=True)  # in a process of its own
    assert float(r["ms_mean"]) > 0
    ref = cpu.BuildResult(len(tris), 30)
    ref.tris = r["tris_out"].view(cpu.TRIANGLE_DTYPE)
    ref.children, ref.parents_leaf, ref.parents_internal = r["children"], r["parents_leaf"], r["parents_internal"]
    ref.node_boxes = r["node_boxes"].view(cpu.BBOX_DTYPE)
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris), box=box, check_root=True)
    out = lb.download()
    for k in ("tris", "children", "parents_leaf", "parents_internal"):
        assert np.ascontiguousarray(out[k]).tobytes() == np.ascontiguousarray(getattr(ref, k)).tobytes(), k
    # boxes: this library's equal the oracle's bit for bit. The reference's refit reads a
    # sibling's box with no fence after the counter (BVHBuilder.cu:63-86), so on the GPU
    # an occasional stale read leaves a box off (3 of 200,001 in one run, none in the
    # others); its boxes may differ from the fenced result at a few nodes, never more.
    mine = out["node_boxes"].view(np.uint32).reshape(-1, 6)
    ob = cpu.build(tris, 30, box=box)
    assert mine.tobytes() == ob.node_boxes.view(np.uint32).reshape(-1, 6).tobytes()
    differ = (mine != ref.node_boxes.view(np.uint32).reshape(-1, 6)).any(1)
    assert differ.sum() <= max(16, len(tris) // 10_000), f"{int(differ.sum())} of the reference's boxes differ"


def test_reference_gpu_render_estimates_the_same_image(cuda):
    """The reference's raytrace_kernel (cuda_path_tracer.cu:385-421, its own curand
    stream) and this library's renderer (the Philox stream) estimate the same image,
    512 one-sample frames each. The image means agree within 2 % (or 4 standard
    deviations of their difference as the seed pairs estimate it). Block by block
    (8x8 pixels, 3 channels), the squared differences between a reference image and one
    of this library's (averaged over the four pairs) sum to about the two renderers' own
    noise, measured by two independent renders of each (seeds 3, 4 and 9, 10): without a
    bias the ratio is near 1 whatever each renderer's variance; a bias of a few percent
    in the lit blocks would push it far above. It must stay below 2 (with about 50-150
    lit block values the ratio's spread is a few tenths).

    The reference's own render is not repeatable: its LBVH refit reads a sibling's box
    with no fence after the counter (BVHBuilder.cu:63-86), and two runs with the same
    seed gave images 34 pixels apart, some runs' means 2-3 % apart. So the reference
    side is rendered again, up to three times, until one pair of its renders meets both
    criteria; this library's side is rendered once (it repeats bit for bit)."""
    if not cpu.refgpu_available():
        pytest.fail("oracle/_ref/librefgpu.so was not built (make -C oracle ref)")
    import torch

    from cpt.device import DeviceRenderer, DeviceScene, make_params

    tris, infos = cpt.scene_random(20_000, seed=5)
    w, h, bounces, spp = 64, 48, 3, 512
    cam = cpt.camera_look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.0), aspect=w / h)
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris), check_root=True)
    scene = DeviceScene(infos)
    ours = []
    for seed in (9, 10):
        r = DeviceRenderer(make_params(w, h, spp, 0, bounces, 3.0, True, seed, cpt.ACCUM_KAHAN))
        r.render(lb, scene, cam)
        torch.cuda.synchronize()
        r.check_status()
        ours.append(r.resolve().cpu().numpy()[..., :3].astype(np.float64))
    assert ours[0].mean() > 0.01

    def blocks(img):
        return img.reshape(h // 8, 8, w // 8, 8, 3).mean(axis=(1, 3))

    def judge(theirs):
        """(means agree, block ratio below 2, figures)"""
        # image means, each renderer's two seeds averaged; one image mean's variance from
        # the two pairs (E[(a - b)^2] = 2 var); the difference of two averages of two
        # images each has the same variance
        mo, mt = 0.5 * (ours[0].mean() + ours[1].mean()), 0.5 * (theirs[0].mean() + theirs[1].mean())
        var_one = 0.25 * ((ours[0].mean() - ours[1].mean()) ** 2 + (theirs[0].mean() - theirs[1].mean()) ** 2)
        sd_diff = var_one ** 0.5
        means_ok = abs(mt - mo) <= max(0.02 * mo, 4 * sd_diff)
        o1, o2, t1, t2 = (blocks(x) for x in (ours[0], ours[1], theirs[0], theirs[1]))
        lit = o1 > 0.05 * o1.max()
        assert lit.sum() >= 40
        own_noise = 0.5 * (((o2 - o1)[lit] ** 2).sum() + ((t2 - t1)[lit] ** 2).sum())
        # every reference image against every one of ours (four pairs)
        cross = 0.25 * sum(((t - o)[lit] ** 2).sum() for t in (t1, t2) for o in (o1, o2))
        ratio = cross / own_noise
        return means_ok and ratio < 2.0, (mt, mo, sd_diff, ratio)

    tries = []
    for _ in range(3):
        theirs = []
        for seed in (3, 4):
            rr = refgpu_child.run("render", tris, cpu.enclosing_box(tris), infos=infos, width=w, height=h,
                                  cam15=cam.as_array(), bounces=bounces, intensity=3.0, stratified=1, warmup=0,
                                  frames=spp, seed=seed)
            assert float(rr["ms_per_frame"]) > 0 and np.isfinite(rr["image"]).all()
            theirs.append(rr["image"][..., :3].astype(np.float64))
        ok, figures = judge(theirs)
        tries.append(figures)
        if ok:
            return
    pytest.fail(f"reference renders (mean theirs, mean ours, sd of the difference, block ratio): {tries}")
