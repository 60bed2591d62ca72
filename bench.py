"""Benchmark: LBVH build + progressive path tracing on one B200 (or N, one process each).

Workload (default, "c2"): 4,194,304-triangle fBm-displaced lat-long sphere
(2048 x 1024 quads) + 1,048,576 thin "hairball" triangles + a 2-triangle quad
emitter = 5,242,882 triangles, 63-bit Morton LBVH, 1920 x 1080, 16 samples per
pixel per frame, depth 8 (7 indirect bounces), Philox random stream. Synthetic
scene, generated on the host from a fixed seed.

One step = one progressive frame (16 spp) rendered with the BVH resident in HBM.
`value` is rays traced (primary + extension + shadow, counted on the device) per
second over the K timed frames, max over ranks. The LBVH build of the same scene
is timed separately (`lbvh`). `e2e` is the same metric through the
reference-facing tracer object with host buffers: every step uploads the scene
(triangles + shading records, pinned host memory), rebuilds the LBVH, renders the
frame and reads the image back.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c2|c1]
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "cuda-path-tracer_b200"))

WORKLOADS = {
    "c2": dict(kind="sphere_hairball", nu=2048, nv=1024, n_hair=1 << 20, bits=63, width=1920, height=1080, spp=16,
               bounces=7, eye=(0.0, 0.35, -3.6), target=(0.0, 0.0, 0.0), seed=0, split=8.0, wide=1, treelet=1,
               wide_sah=1,
               # every e2e step rebuilds the trees inside its timed region: there the cheaper build wins
               e2e_split=4.0, e2e_treelet=0),
    "c1": dict(kind="random", n=65536, bits=30, width=512, height=512, spp=1, bounces=3, eye=(0.5, 0.5, -1.2),
               target=(0.5, 0.5, 0.0), seed=0, wide=1, wide_sah=1),
    # 64 scenes, 10k-2M triangles (log-uniform, alternating generators), 256^2-1024^2, one graph launch per frame
    "c3": dict(kind="batch", scenes=64, tri_min=10_000, tri_max=2_000_000, res_min=256, res_max=1024, spp=4,
               bounces=5, bits=63, seed=0, width=0, height=0, split=1.25, wide=1, wide_sah=1),
    # radiance cache on the C2 scene: 1 spp frames through the cache vs plain 16 spp, RMSE vs an FP64 image
    "c4": dict(kind="sphere_hairball", nu=2048, nv=1024, n_hair=1 << 20, bits=63, width=1920, height=1080, spp=1,
               bounces=7, eye=(0.0, 0.35, -3.6), target=(0.0, 0.0, 0.0), seed=0, plain_spp=64, ref_spp=4096,
               ref_div=4, warm_updates=1, max_spp=256, split=8.0, wide=1, treelet=1, wide_sah=1),
    # deforming 16.8 M-triangle displaced sphere, full rebuild every frame, 8 cameras
    "c5": dict(kind="deform", nu=4096, nv=2048, n_hair=0, bits=63, width=1280, height=720, spp=1, bounces=7,
               eye=(0.0, 0.35, -3.6), target=(0.0, 0.0, 0.0), seed=0, cameras=8, amp=0.01, omega=40.0, cache=True),
}
METRIC = "Mrays/s"


def make_scene(w):
    import cpt

    if w["kind"] == "random":
        return cpt.scene_random(w["n"], seed=w["seed"])
    return cpt.scene_sphere_hairball(w["nu"], w["nv"], w["n_hair"], seed=w["seed"])


def make_cameras(w):
    """The workload's camera(s): one, or `cameras` orbiting the target at the eye's distance."""
    import math

    import cpt

    aspect = w["width"] / w["height"]
    k = w.get("cameras", 1)
    if k == 1:
        return [cpt.camera_look_at(w["eye"], w["target"], fov_deg=45.0, aspect=aspect)]
    r = math.hypot(w["eye"][0], w["eye"][2])
    return [cpt.camera_look_at((r * math.sin(2 * math.pi * i / k), w["eye"][1], -r * math.cos(2 * math.pi * i / k)),
                               w["target"], fov_deg=45.0, aspect=aspect) for i in range(k)]


def workload_config(name, w, n_tris, l2_note):
    hair = f'{w["n_hair"] >> 20}M' if w.get("n_hair", 0) and w["n_hair"] % (1 << 20) == 0 else str(w.get("n_hair"))
    desc = {"c2": f'fBm sphere {w.get("nu")}x{w.get("nv")}x2 + {hair} hairball + quad light',
            "c4": "fBm sphere 2048x1024x2 + 1M hairball + quad light, radiance cache (96-64x4-16 BF16 MLP, 2^16 "
                  "training paths per frame, Adam 1e-2) vs plain path tracing",
            "c1": "65,536 random triangles + quad light",
            "c5": "deforming fBm sphere 4096x2048x2 + quad light, rebuild every frame, 8 cameras, radiance cache "
                  "(trained across the deforming frames)",
            "c3": "64 scenes 10k-2M triangles (random / sphere+hairball alternating; split BVH for the hairball scenes), 256^2-1024^2, 4 spp, "
                  "depth 6, one CUDA-graph launch per frame, autotuned wave"}[name]
    c = {"workload": f"{name}: {desc}",
         "triangles": int(n_tris), "morton_bits": w["bits"], "resolution": f'{w["width"]}x{w["height"]}',
         "spp_per_step": w["spp"], "depth": w["bounces"] + 1, "cameras": w.get("cameras", 1), "l2": l2_note}
    return c


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


def dist_setup(n_gpus):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# --------------------------------------------------------------------------- CPU baseline
def sample_rows(height, stride):
    """Every stride-th row of the frame, starting half a stride in: a sample spread
    evenly over the whole image (sky, sphere and hairball rows in their proportions)."""
    return np.arange(stride // 2, height, stride, dtype=np.uint32)


def cpu_reference_run(w, tris, infos, cam, bits, target_s=12.0, stride=None):
    """The reference's own builder (oracle/_ref, OpenMP over all host threads) on the
    full scene, then the restated integrator over the reference's trace functions on
    every `stride`-th row of frame 0 (samples 0 .. spp-1 of the workload's seed), with
    the stride chosen for ~target_s seconds of CPU work. The frame's rate is taken to
    be the sampled rows' rate (the rows are spread over the whole frame). Per-pixel
    float64 sums of the rows come back for the parity check against the GPU's frame 0.
    Falls back to the oracle port when the reference library was not built."""
    from oracle import cpu

    threads = os.cpu_count() or 1
    kind = "reference" if cpu.ref_available(bits) else "port"
    t0 = time.perf_counter()
    b = cpu.build(tris, bits, use_ref=(kind == "reference"))
    build_s = time.perf_counter() - t0
    width, height, spp = w["width"], w["height"], w["spp"]
    cam15 = cam.as_array()

    def run(rows):
        t1 = time.perf_counter()
        if kind == "reference":
            sums, cnt = cpu.ref_render_rows(b, infos, None, width, height, rows, spp, 0, w["bounces"], 3.0, True,
                                            w["seed"], cam15, threads)
        else:
            sums, cnt = cpu.render_rows(b, infos, width, height, rows, spp, 0, w["bounces"], 3.0, True, w["seed"],
                                        cpu.ocam_from(cam.eye, cam15[3:]))
        return time.perf_counter() - t1, int(cnt.sum()), sums

    if stride is None:  # probe 8 rows spread over the frame, then size the sample
        probe = sample_rows(height, max(1, height // 8))
        dt, _, _ = run(probe)
        rows_needed = max(1.0, target_s / max(dt / len(probe), 1e-4))
        stride = int(min(height, max(1, round(height / rows_needed))))
    rows = sample_rows(height, stride)
    dt, rays, sums = run(rows)
    return {"kind": kind, "threads": threads, "build_s": build_s, "build_mtris_s": len(tris) / build_s / 1e6,
            "render_s": dt, "rays": rays, "rows": rows, "stride": stride, "sums": sums,
            "mrays_s": rays / dt / 1e6,
            "sample": f"one row in {stride} of frame 0 ({len(rows)} of {height} rows, from row {stride // 2}) x "
                      f"{width} px x {spp} spp, depth {w['bounces'] + 1}; the frame's rate is taken as the sampled "
                      f"rows' rate; build of all {len(tris)} triangles"}


def reference_gpu(w, tris, infos, cam, dev, ours_ms_per_spp, rays_per_spp, reps=5, frames=8):
    """The reference's own GPU code on this GPU (oracle/_ref/librefgpu.so: its sources
    compiled for sm_100a, 30-bit keys as shipped), beside this library on the same
    triangles: BVHBuilder::build against cpt_lbvh_build at the same key width, and
    raytrace_kernel (one sample per pixel per launch, its own curand stream) against this
    library's time per sample of the timed frames. The reference counts no rays: its
    Mrays/s uses this library's rays per sample of the same scene and estimator (the
    expected count is the estimator's). None when that library was not built."""
    import torch

    import cpt
    from oracle import cpu, refgpu_child
    from cpt.device import DeviceLbvh, to_device

    if not cpu.refgpu_available():
        return None
    n = len(tris)
    box = cpt.scene_bounds(tris)
    try:  # in a child process: the reference's thrust and CUDA runtime stay out of this one
        r = refgpu_child.run("build", tris, box, reps=reps, outputs=False)
    except Exception as e:
        return {"unavailable": str(e)[-300:]}
    ref = {k: float(r[k]) for k in ("ms_mean", "ms_min", "wall_ms_mean")}
    lb = DeviceLbvh(n, 30, dev)
    d = to_device(tris, dev)
    lb.build(d, check_root=True)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        lb.build(d)
    e1.record(stream)
    torch.cuda.synchronize()
    lb.status()
    ours = e0.elapsed_time(e1) / reps
    del lb, d
    out = {"what": "the reference's own CUDA code compiled from its sources for sm_100a, on this GPU",
           "lbvh": {"reference": "BVHBuilder::build (thrust sort + its kernels, BVHBuilder.cu:207-269)",
                    "ours": "cpt_lbvh_build at the same 30-bit key width", "triangles": n, "morton_bits": 30,
                    "builds": reps, "reference_ms": round(ref["ms_mean"], 3),
                    "reference_ms_min": round(ref["ms_min"], 3), "reference_wall_ms": round(ref["wall_ms_mean"], 3),
                    "reference_mtris_s": round(n / ref["ms_mean"] / 1e3, 2), "ours_ms": round(ours, 4),
                    "ours_mtris_s": round(n / ours / 1e3, 2), "speedup": round(ref["ms_mean"] / ours, 2)}}
    if w["width"] % 8 == 0 and w["height"] % 8 == 0:
        try:
            rr = refgpu_child.run("render", tris, box, infos=infos, width=w["width"], height=w["height"],
                                  cam15=cam.as_array(), bounces=w["bounces"], intensity=3.0, stratified=1, warmup=2,
                                  frames=frames, seed=w["seed"] + 1)
        except Exception as e:
            out["render"] = {"unavailable": str(e)[-300:]}
            return out
        r = {"ms_per_frame": float(rr["ms_per_frame"]), "build_ms": float(rr["build_ms"])}
        img = rr["image"]
        ref_mrays = rays_per_spp / r["ms_per_frame"] / 1e3
        out["render"] = {"reference": "raytrace_kernel (cuda_path_tracer.cu:385-421), 8x8 blocks, one sample per "
                                      "pixel per launch, over its own 30-bit LBVH",
                         "ours": "the timed frames (the benchmark's traversal tree), per sample",
                         "frames": frames, "reference_ms_per_spp": round(r["ms_per_frame"], 3),
                         "ours_ms_per_spp": round(ours_ms_per_spp, 4),
                         "speedup": round(r["ms_per_frame"] / ours_ms_per_spp, 2),
                         "reference_mrays_s_est": round(ref_mrays, 3),
                         "rays_per_spp_used": int(rays_per_spp),
                         "reference_image_mean": round(float(img[..., :3].mean()), 6)}
    return out


def extra_builds(dev, reps=5):
    """Two build measurements the driver's default run carries beside C2: a full rebuild
    of the 16.8 M-triangle displaced sphere of C5 after a deformation step (63-bit keys),
    and C3's 64 scenes as one batched build against 64 single builds. Scenes generated on
    the host (seeded), resident on the device; CUDA events."""
    import torch

    import cpt
    from cpt.device import DeviceLbvh, LbvhBatch, stream_handle, to_device

    stream = torch.cuda.current_stream()

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {}
    w5 = WORKLOADS["c5"]
    rest, _ = cpt.scene_sphere_hairball(w5["nu"], w5["nv"], 0, seed=w5["seed"])
    n5 = len(rest)
    d_rest, d_tris = to_device(rest, dev), to_device(rest, dev)
    cpt.check(cpt.lib.cpt_scene_deform(d_rest.data_ptr(), d_tris.data_ptr(), n5, w5["amp"], w5["omega"], 0.1,
                                       stream_handle()), "cpt_scene_deform")
    lb = DeviceLbvh(n5, 63, dev)
    lb.build(d_tris, check_root=True)
    ms = timed(lambda: lb.build(d_tris))
    lb.status()
    out["c5_rebuild"] = {"triangles": n5, "morton_bits": 63, "ms": round(ms, 3), "mtris_s": round(n5 / ms / 1e3, 2),
                         "what": "cpt_lbvh_build of the deformed 4096x2048x2 displaced sphere, box computed on the "
                                 "device"}
    del lb, d_rest, d_tris
    torch.cuda.empty_cache()
    w3 = WORKLOADS["c3"]
    lbs, srcs, boxes = [], [], []
    for i, (kind, ntri, _side) in enumerate(batch_specs(w3)):
        tris, _ = batch_scene(kind, ntri, w3["seed"] + i)
        lbs.append(DeviceLbvh(len(tris), w3["bits"], dev))
        srcs.append(to_device(tris, dev))
        boxes.append(cpt.scene_bounds(tris))
    batch = LbvhBatch(lbs, dev)
    batch.build(srcs, boxes, check_root=True)
    n3 = sum(lb.n for lb in lbs)
    t_batch = timed(lambda: batch.build(srcs, boxes))
    t_single = timed(lambda: [lb.build(d) for lb, d in zip(lbs, srcs)])
    for lb in lbs:
        lb.status()
    out["c3_batch_build"] = {"scenes": len(lbs), "triangles": n3, "morton_bits": w3["bits"],
                             "batched_ms": round(t_batch, 3), "batched_mtris_s": round(n3 / t_batch / 1e3, 2),
                             "single_calls_ms": round(t_single, 3),
                             "single_calls_mtris_s": round(n3 / t_single / 1e3, 2)}
    return out


def frame_parity(gpu_sums, cpu_sums, spp):
    """GPU frame-0 rows (FP64 accumulator) against the reference's rows (float64 sums
    of the same float samples in the same order): pixels whose three sums differ in
    any bit, and the largest difference of the per-pixel mean."""
    differ = (gpu_sums != cpu_sums).any(axis=-1)
    diff = np.abs(gpu_sums - cpu_sums).max() / spp if gpu_sums.size else 0.0
    return {"rows": int(gpu_sums.shape[0]), "pixels": int(differ.size), "mismatched_pixels": int(differ.sum()),
            "max_abs_diff": float(diff), "exact": bool(not differ.any())}


# --------------------------------------------------------------------------- batched scenes (c3)
def batch_specs(w):
    """Per scene: (kind, triangles, side) drawn from the seeded log-uniform ranges."""
    rng = np.random.default_rng(w["seed"])
    tri = np.exp(rng.uniform(np.log(w["tri_min"]), np.log(w["tri_max"]), w["scenes"])).astype(np.int64)
    side = np.exp(rng.uniform(np.log(w["res_min"]), np.log(w["res_max"]), w["scenes"]))
    side = (np.round(side / 8) * 8).astype(np.int64)
    return [("random" if i % 2 == 0 else "sphere", int(tri[i]), int(side[i])) for i in range(w["scenes"])]


def batch_scene(kind, ntri, seed):
    import cpt

    if kind == "random":
        return cpt.scene_random(max(ntri - 2, 2), seed=seed)
    hair = ntri // 5
    nv = max(4, int(round((max(ntri - hair - 2, 32) / 4) ** 0.5)))
    return cpt.scene_sphere_hairball(2 * nv, nv, hair, seed=seed)


def run_batch(args, w, world, rank, local):
    import torch

    import cpt
    from cpt import autotune
    from cpt.device import BatchRenderer, DeviceLbvh, DeviceScene, make_params, stream_handle, to_device
    from cpt.multi import assign_by_cost, scene_cost

    dev = torch.device("cuda", local if world > 1 else 0)
    t0 = time.perf_counter()
    specs = batch_specs(w)
    # the scenes are independent: each rank renders whole scenes of a cost-balanced share
    shares = assign_by_cost([scene_cost(side * side, ntri, kind != "random") for kind, ntri, side in specs], world)
    mine = shares[rank]
    if not mine:
        raise SystemExit("more ranks than scenes")
    split = w.get("split", 0.0) if args.split is None else args.split
    views, keep, n_tris, pixels, boxes = [], [], 0, 0, []
    for i, (kind, ntri, side) in enumerate(specs):
        if i not in mine:
            continue
        tris, infos = batch_scene(kind, ntri, w["seed"] + i)
        boxes.append(cpt.scene_bounds(tris))
        lb = DeviceLbvh(len(tris), w["bits"], dev)
        d = to_device(tris, dev)
        lb.build(d, check_root=True)
        if kind != "random" and split > 0:  # the hairball scenes traverse a split BVH
            lb.split(split, flags=split_flags(args))
        if args.wide:
            lb.wide(keep_scratch=True, sah=bool(args.wide_sah))
        sc = DeviceScene(infos, None, dev)
        eye, tgt = ((0.5, 0.5, -1.2), (0.5, 0.5, 0.0)) if kind == "random" else ((0.0, 0.35, -3.6), (0.0, 0.0, 0.0))
        cam = cpt.camera_look_at(eye, tgt, fov_deg=45.0, aspect=1.0)
        views.append((lb, sc, cam, side, side))
        keep.append(d)
        n_tris += len(tris)
        pixels += side * side
    gen_s = time.perf_counter() - t0
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()

    def params(wave, sort, stats=False, refill=0, blocks=0, lanes=0):
        return make_params(0, 0, w["spp"], 0, w["bounces"], 3.0, True, w["seed"],
                           cpt.ACCUM_KAHAN, wave_paths=wave, ray_sort=sort, trace_stats=stats, refill_lanes=refill,
                           traverse_blocks_per_sm=blocks, wave_lanes=lanes or args.wave_lanes)

    # --- autotuner (cpt/autotune.py): one warm + one timed frame per candidate, keep the
    # fastest; first the wave size and ray sorting, then the traversal's launch shape
    def time_frame(wave, sort, refill=0, blocks=0, lanes=0):
        br = BatchRenderer(views, params(wave, sort, refill=refill, blocks=blocks, lanes=lanes), dev)
        br.render()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        br.render()
        e1.record(stream)
        torch.cuda.synchronize()
        del br
        torch.cuda.empty_cache()
        return e0.elapsed_time(e1)

    tuned = autotune.tune(time_frame, ((1 << 24, 0), (1 << 25, 0), (1 << 26, 0), (1 << 25, 1)))
    shaped = autotune.tune(time_frame, autotune.launch_candidates(tuned))
    tune = tuned.table + shaped.table
    best = {"wave_paths": shaped.wave_paths, "ray_sort": shaped.ray_sort, "refill_lanes": shaped.refill_lanes,
            "blocks_per_sm": shaped.blocks_per_sm, "wave_lanes": shaped.wave_lanes, "ms": shaped.ms}
    shape = {"refill": best["refill_lanes"], "blocks": best["blocks_per_sm"], "lanes": best["wave_lanes"]}

    # --- instrumented frame: node visits per closest-hit ray
    br = BatchRenderer(views, params(best["wave_paths"], best["ray_sort"], stats=True, **shape), dev)
    br.render()
    torch.cuda.synchronize()
    c = br.counts.cpu().numpy()
    mean_nodes = c[3] / max(c[0] + c[1], 1)
    mean_tris = c[4] / max(c[0] + c[1], 1)
    del br

    # --- one frame captured in a CUDA graph; the device frame counter advances per replay
    counter = torch.zeros(1, dtype=torch.int32, device=dev)
    p = params(best["wave_paths"], best["ray_sort"], **shape)
    p.frame_counter = counter.data_ptr()
    br = BatchRenderer(views, p, dev)
    side_stream = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(side_stream):
        br.render()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        br.render()
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize()
    br.counts.zero_()
    sampler = ClockSampler(local if world > 1 else 0) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    launches0 = cpt.launch_count()
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        graph.replay()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop() if sampler else None
    br.check_status()
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    counts = br.counts.cpu().numpy()
    rays = sum_over_ranks(float(counts[0] + counts[1] + counts[2]), world)
    value = rays / (ms / 1e3) / 1e6
    graph_launches = cpt.launch_count() - launches0  # 0: replays issue no library calls

    # --- profile one graph replay per kernel (events inside the library need direct calls)
    cpt.profile_begin()
    br.render()
    torch.cuda.synchronize()
    prof = cpt.profile_end()
    busy = cpt.profile_busy()
    ext_ms, ext_n = prof.get("k_extend", (0.0, 0))
    ext_ms = busy.get("k_extend", ext_ms)  # two wave lanes overlap their launches: the time any one ran
    closest_frame = float(counts[0] + counts[1]) / args.steps
    node_b = 80.0 if args.wide else 64.0  # a wide node record, or the compact two-child node
    alg = closest_frame * (48 + node_b * mean_nodes + 48.0 * mean_tris)
    peak, peak_kind = measured_peaks()
    ach = alg / (ext_ms / 1e3) / 1e9 if ext_ms else 0.0
    frame_ms = sum(busy.get(k, v[0]) for k, v in prof.items())

    # --- one CUDA graph for a whole frame: every scene's LBVH rebuilt (and the split
    # trees of the hairball scenes), then all scenes rendered; one replay per frame
    hair = [specs[i][0] != "random" and split > 0 for i in mine]
    for (lb, _, _, _, _), h in zip(views, hair):
        if h:
            lb.split(split, keep_scratch=True, flags=split_flags(args))  # scratch stays allocated for the captured rebuilds
        if args.wide:
            lb.wide(keep_scratch=True)
    torch.cuda.synchronize()

    from cpt.device import LbvhBatch, WideBatch

    batch = LbvhBatch([v[0] for v in views], dev)  # every scene's LBVH in one launch sequence
    wbatch = WideBatch([v[0] for v in views], dev) if args.wide else None  # and every wide tree
    batch.build(keep, boxes, check_root=True)

    # the split trees of different scenes are independent: built on a few side streams
    # forked from the frame's stream (and joined before the wide trees), so that the
    # small scenes' kernels run side by side
    split_streams = [torch.cuda.Stream(dev) for _ in range(max(1, args.split_streams))]

    def split_all():
        cur = torch.cuda.current_stream()
        for st in split_streams:
            st.wait_stream(cur)
        j = 0
        for (lb, _, _, _, _), h in zip(views, hair):
            if h:
                lb.split(split, keep_scratch=True, flags=split_flags(args),
                         stream=split_streams[j % len(split_streams)].cuda_stream)
                j += 1
        for st in split_streams:
            cur.wait_stream(st)

    def rebuild_all():
        batch.build(keep, boxes)
        split_all()
        if wbatch is not None:
            wbatch.build()

    counter2 = torch.zeros(1, dtype=torch.int32, device=dev)
    p2 = params(best["wave_paths"], best["ray_sort"], **shape)
    p2.frame_counter = counter2.data_ptr()
    br2 = BatchRenderer(views, p2, dev)
    with torch.cuda.stream(side_stream):
        rebuild_all()
        br2.render()
    torch.cuda.synchronize()
    graph2 = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph2):
        rebuild_all()
        br2.render()
    for _ in range(max(1, args.warmup)):
        graph2.replay()
    torch.cuda.synchronize()
    br2.counts.zero_()
    barrier(world)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        graph2.replay()
    f1.record(stream)
    torch.cuda.synchronize()
    br2.check_status()
    ms2 = max_over_ranks(f0.elapsed_time(f1), world)
    c2n = br2.counts.cpu().numpy()
    rays2 = sum_over_ranks(float(c2n[0] + c2n[1] + c2n[2]), world)
    built_and_rendered = {"mrays_s": round(rays2 / (ms2 / 1e3) / 1e6, 3), "ms_per_step": round(ms2 / args.steps, 3),
                          "note": "one CUDA graph replay per frame: every scene's LBVH (one batched build, "
                                  "cpt_lbvh_build_batch), the split trees of the hairball scenes (on "
                                  f"{len(split_streams)} forked streams), every wide tree "
                                  "(one batched build, cpt_lbvh_wide_batch, largest-child collapse), then the render "
                                  "of all scenes"}
    del graph2, br2

    # --- rebuild of the rank's scenes (device-resident soups): the batched build, and
    # the same scenes built one call each for comparison
    def time_builds(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    build_ms = max_over_ranks(time_builds(lambda: batch.build(keep, boxes)), world)
    per_scene_ms = max_over_ranks(time_builds(lambda: [v[0].build(d) for v, d in zip(views, keep)]), world)
    # the frame's rebuild part by part (outside the graph): the batched LBVH build, the
    # split trees of the hairball scenes, the wide trees
    split_ms = max_over_ranks(time_builds(split_all), world)
    wide_ms = max_over_ranks(time_builds(lambda: wbatch.build()), world) if args.wide else 0.0
    wide_single_ms = max_over_ranks(time_builds(lambda: [v[0].wide(keep_scratch=True) for v in views]), world) \
        if args.wide else 0.0
    for v in views:
        v[0].status()
    n_tris = int(sum_over_ranks(float(n_tris), world))
    pixels = int(sum_over_ranks(float(pixels), world))
    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 3), "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
                "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded host generator)",
                "parallelism": f"scenes partitioned over {world} ranks by estimated cost, no exchange"
                               if world > 1 else "1 GPU",
                "config": {"workload": "c3: " + "64 scenes, log-uniform 10k-2M triangles, 256^2-1024^2, 4 spp, depth 6",
                           "scenes": len(specs), "triangles": int(n_tris), "pixels": int(pixels),
                           "spp_per_step": w["spp"], "depth": w["bounces"] + 1, "morton_bits": w["bits"],
                           "graph": "one CUDA graph replay per frame", "l2": "scene arrays > 126 MB L2"},
                "autotune": {"candidates": tune, "chosen": best},
                "built_and_rendered_per_frame": built_and_rendered,
                "rays_per_step": int(rays / args.steps),
                "roofline": {"bound": "hbm", "kernel": "k_extend", "achieved": round(ach, 1), "peak": peak,
                             "unit": "GB/s", "frac": round(ach / peak, 4), "traffic": None,
                             "bytes_per_ray": f"48 + {node_b:.0f} x {mean_nodes:.2f} nodes + 48 x {mean_tris:.2f} triangles",
                             "busy_ms": round(ext_ms, 3),
                             "kernel_share": {k: round(busy.get(k, v[0]) / frame_ms, 4)
                                              for k, v in sorted(prof.items())}},
                "lbvh": {"mtris_s": round(n_tris / build_ms / 1e3, 2), "ms": round(build_ms, 3),
                         "per_scene_calls_ms": round(per_scene_ms, 3),
                         "frame_rebuild_parts_ms": {"lbvh_batch": round(build_ms, 3), "split_trees": round(split_ms, 3),
                                                    "wide_trees": round(wide_ms, 3),
                                                    "wide_trees_per_scene_calls": round(wide_single_ms, 3)},
                         "per_scene_calls_mtris_s": round(n_tris / per_scene_ms / 1e3, 2),
                         "note": "each rank's scenes in one batched build (cpt_lbvh_build_batch; max over ranks); "
                                 "per_scene_calls = the same scenes built by one cpt_lbvh_build call each"},
                # kernels of one frame (graph nodes) x timed replays; the replays themselves make no
                # library calls (graph_launches counts those: 0)
                "gpu_launches": int(sum(v[1] for v in prof.values()) * args.steps),
                "library_calls_in_timed_region": int(graph_launches),
                "clocks": clocks, "scene_gen_s": round(gen_s, 2), "cpu_baseline": None, "e2e": None}
        print(json.dumps(line), flush=True)
    return 0


def run_reference_arm(args, w, world, rank):
    if rank != 0:
        return 0
    if w["kind"] == "batch":
        print(json.dumps({"impl": "reference", "unavailable": "the reference renders one scene per process; "
                          "the batched workload has no reference counterpart"}), flush=True)
        return 0
    import cpt

    t0 = time.perf_counter()
    tris, infos = make_scene(w)
    gen_s = time.perf_counter() - t0
    cam = make_cameras(w)[0]
    # size one step for ~8 s of CPU work, then warm up and time K steps of that size
    probe = cpu_reference_run(w, tris, infos, cam, w["bits"], target_s=8.0)
    stride = probe["stride"]
    for _ in range(max(0, args.warmup - 1)):
        cpu_reference_run(w, tris, infos, cam, w["bits"], stride=stride)
    rays = 0
    secs = 0.0
    last = probe
    for _ in range(args.steps):
        last = cpu_reference_run(w, tris, infos, cam, w["bits"], stride=stride)
        rays += last["rays"]
        secs += last["render_s"]
    value = rays / secs / 1e6
    line = {"metric": METRIC, "value": round(value, 4), "unit": METRIC, "impl": "reference", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * secs / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded host generator)",
            "config": workload_config(args.workload, w, len(tris), "n/a (CPU)"),
            "cpu_baseline": {"value": round(value, 4), "unit": METRIC, "cores": last["threads"], "kind": last["kind"],
                             "sample": last["sample"]},
            "lbvh": {"mtris_s": round(last["build_mtris_s"], 3), "ms": round(1e3 * last["build_s"], 3)},
            "e2e": {"value": round(value, 4), "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "scene_gen_s": round(gen_s, 2)}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------- our arm
def run_ours(args, w, world, rank, local):
    import torch

    import cpt
    from cpt.device import DeviceLbvh, DeviceRenderer, DeviceScene, make_params, stream_handle, to_device

    dev = torch.device("cuda", local if world > 1 else 0)
    t0 = time.perf_counter()
    tris, infos = make_scene(w)
    gen_s = time.perf_counter() - t0
    n = len(tris)
    W_, H_, spp = w["width"], w["height"], w["spp"]
    cams = make_cameras(w)
    cam = cams[0] if len(cams) == 1 else cams
    deforming = w["kind"] == "deform"
    d_tris = to_device(tris, dev)
    d_rest = to_device(tris, dev) if deforming else None
    scene = DeviceScene(infos, None, dev)
    lb = DeviceLbvh(n, w["bits"], dev)
    lb.build(d_tris, check_root=True)
    split = w.get("split", 0.0) if args.split is None else args.split
    if split > 0:
        lb.split(split, keep_scratch=True, flags=split_flags(args))
    if args.wide:
        lb.wide(keep_scratch=True, sah=bool(args.wide_sah))
    params = make_params(W_, H_, spp, 0, w["bounces"], 3.0, True, w["seed"], cpt.ACCUM_KAHAN,
                         wave_paths=args.wave_paths, ray_sort=bool(args.ray_sort), cameras=len(cams),
                         refill_lanes=args.refill_lanes, traverse_blocks_per_sm=args.blocks_per_sm,
                         wave_lanes=args.wave_lanes)

    def deform_and_rebuild(frame_index):
        # the deforming-mesh step: move the vertices, then a full LBVH rebuild
        cpt.check(cpt.lib.cpt_scene_deform(d_rest.data_ptr(), d_tris.data_ptr(), n, w["amp"], w["omega"],
                                           0.1 * frame_index, stream_handle()), "cpt_scene_deform")
        lb.build(d_tris)
        if split > 0:
            lb.split(split, keep_scratch=True, flags=split_flags(args))
        if args.wide:
            lb.wide(keep_scratch=True)
    rend = DeviceRenderer(params, dev)
    stream = torch.cuda.current_stream()
    # Pipelined rebuild (the deforming workload, LBVH trees): two trees and two triangle
    # buffers; frame f renders tree f % 2 while a side stream deforms and builds frame
    # f + 1's into the other (after the render that last read it). The renderers read
    # the tree through one view struct that takes the current tree's fields at each frame.
    pipelined = deforming and args.c5_pipeline and split <= 0
    view = lb
    if pipelined:
        import ctypes as _ct

        class _ViewTree:  # what the renderers read as "the LBVH": a bvh struct
            def __init__(self):
                self.bvh = cpt.Bvh()

        view = _ViewTree()
        _ct.memmove(_ct.addressof(view.bvh), _ct.addressof(lb.bvh), _ct.sizeof(cpt.Bvh))
        trees = [lb, DeviceLbvh(n, w["bits"], dev)]
        tri_bufs = [d_tris, torch.empty_like(d_tris)]
        bstream = torch.cuda.Stream(dev)
        ev_built = [torch.cuda.Event(), torch.cuda.Event()]
        ev_read = [torch.cuda.Event(), torch.cuda.Event()]
        for e in ev_read:
            e.record(stream)

        def build_tree(frame_index, slot, st):
            cpt.check(cpt.lib.cpt_scene_deform(d_rest.data_ptr(), tri_bufs[slot].data_ptr(), n, w["amp"], w["omega"],
                                               0.1 * frame_index, st.cuda_stream), "cpt_scene_deform")
            trees[slot].build(tri_bufs[slot], stream=st.cuda_stream)
            if args.wide:
                trees[slot].wide(stream=st.cuda_stream, keep_scratch=True)
            ev_built[slot].record(st)

        def use_tree(slot):
            stream.wait_event(ev_built[slot])
            _ct.memmove(_ct.addressof(view.bvh), _ct.addressof(trees[slot].bvh), _ct.sizeof(cpt.Bvh))

    cached = None
    if w.get("cache"):
        # every camera is a view of the same BVH; the cache trains on all of them
        from cpt.device import CachedRenderer, RadianceCache

        rcache = RadianceCache()
        cparams = make_params(W_, H_, spp, 0, w["bounces"], 3.0, True, w["seed"], cpt.ACCUM_KAHAN,
                              wave_paths=args.wave_paths)
        cached = CachedRenderer(rcache, [(view, scene, c_, W_, H_) for c_ in cams], cparams, dev)

    # --- one instrumented frame: node fetches and triangle tests per closest-hit ray
    rend.reset()
    rend.render(lb, scene, cam, frame0=rank * (1 << 24), trace_stats=True)
    torch.cuda.synchronize()
    rend.check_status()
    c = rend.counts.cpu().numpy()
    depth_rays = [int(x) for x in c[8:8 + w["bounces"] + 1]]
    inst_rays_closest = int(c[0] + c[1])
    mean_nodes = c[3] / max(inst_rays_closest, 1)
    mean_tris = c[4] / max(inst_rays_closest, 1)

    # --- warm-up frames (rank r renders its own slice of the sample stream)
    from cpt.multi import rank_frame0, reduce_accumulator

    rend.reset()
    frame = 0

    def frame_step(f0):
        if cached is not None:
            cached.render(frame0=f0)
        else:
            rend.render(view, scene, cam, frame0=f0)

    def pipelined_step(frame_index, f0):
        # render frame_index with its tree; build frame_index + 1's beside it
        cur = frame_index % 2
        use_tree(cur)
        frame_step(f0)
        ev_read[cur].record(stream)
        nxt = 1 - cur
        bstream.wait_event(ev_read[nxt])  # the render of frame_index - 1 read that tree
        build_tree(frame_index + 1, nxt, bstream)

    if pipelined:
        build_tree(0, 0, stream)
    for i in range(args.warmup):
        if pipelined:
            pipelined_step(i, rank_frame0(frame, rank))
        else:
            if deforming:
                deform_and_rebuild(i)
            frame_step(rank_frame0(frame, rank))
        frame += spp
    torch.cuda.synchronize()
    rend.counts.zero_()
    if cached is not None:
        cached.counts.zero_()

    # --- timed frames
    my_accums = cached.accums if cached is not None else [rend.accum]
    display = [torch.empty_like(a) for a in my_accums] if world > 1 else []  # rank 0's reduced images
    sampler = ClockSampler(local if world > 1 else 0) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    launches0 = cpt.launch_count()
    barrier(world)
    torch.cuda.synchronize()
    cpt.profile_begin()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for k in range(args.steps):
        if pipelined:
            pipelined_step(args.warmup + k, rank_frame0(frame, rank))
        else:
            if deforming:
                deform_and_rebuild(args.warmup + k)
            frame_step(rank_frame0(frame, rank))
        frame += spp
        if world > 1:  # the one exchange of the path: framebuffer reduce to rank 0 every frame
            for acc, disp in zip(my_accums, display):
                reduce_accumulator(acc, disp, dst=0, mode=cpt.ACCUM_KAHAN)
    if pipelined:
        stream.wait_stream(bstream)  # the build of the next frame, started in the last step
    ev1.record(stream)
    torch.cuda.synchronize()
    prof = cpt.profile_end()
    busy = cpt.profile_busy()
    barrier(world)
    launches = cpt.launch_count() - launches0
    clocks = sampler.stop() if sampler else None
    rend.check_status()
    if cached is not None:
        cached.check_status()
    ms_total = ev0.elapsed_time(ev1)
    counts = (cached.counts if cached is not None else rend.counts).cpu().numpy()
    rays_local = int(counts[0] + counts[1] + counts[2])
    ms_max = max_over_ranks(ms_total, world)
    rays_all = sum_over_ranks(rays_local, world)
    value = rays_all / (ms_max / 1e3) / 1e6

    # --- roofline of the dominant kernel (closest-hit traversal, k_extend)
    ext_ms, ext_launches = prof.get("k_extend", (0.0, 0))
    # with two wave lanes the launches of the two halves overlap: the kernel's time is the
    # time during which at least one of its launches ran (equal to the sum with one lane)
    ext_busy = busy.get("k_extend", ext_ms)
    rays_closest = int(counts[0] + counts[1])
    node_b = 80.0 if args.wide else 64.0  # a wide node record, or the compact two-child node
    alg_bytes = rays_closest * (32 + 16) + rays_closest * (node_b * mean_nodes + 48.0 * mean_tris)
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (ext_busy / 1e3) / 1e9 if ext_busy > 0 else 0.0
    # DRAM traffic needs ncu, which this run does not use: the per-ray figure of the
    # traversal's capture is in the profile named here, not re-read by the benchmark
    prof_name = ("k_extend_c2_wide.md" if args.wide else "k_extend_c2_split.md" if split > 0 else "k_extend_c2.md")
    roofline = {"bound": "hbm", "kernel": "k_extend", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                if peak_kind == "measured" else "fallback 6650 GB/s",
                "traffic": None, "traffic_note": f"not measured in this run (no ncu); see profiles/{prof_name}",
                "algorithmic_bytes_per_launch": round(alg_bytes / max(ext_launches, 1), 1),
                "avg_launch_ms": round(ext_ms / max(ext_launches, 1), 4), "launches": int(ext_launches),
                "busy_ms": round(ext_busy, 3),
                "achieved_from": "algorithmic bytes of all timed launches / busy_ms (the time at least one "
                                 "k_extend launch ran; the two wave lanes' launches overlap)",
                "bytes_per_ray": f"32 ray + 16 hit + {node_b:.0f} x {mean_nodes:.2f} nodes + 48 x {mean_tris:.2f} triangles",
                "rays_per_depth_first_frame": depth_rays,
                "kernel_share": {k: round(busy.get(k, v[0]) / ms_total, 4) for k, v in sorted(prof.items())}}

    # --- the same frame over the LBVH itself (no split BVH), for comparison
    lbvh_topology = None
    if split > 0 and not deforming and cached is None:
        lb.unsplit()
        rend.render(lb, scene, cam, frame0=rank_frame0(frame, rank))
        torch.cuda.synchronize()
        rend.counts.zero_()
        u0, u1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        u0.record(stream)
        rend.render(lb, scene, cam, frame0=rank_frame0(frame + spp, rank))
        u1.record(stream)
        torch.cuda.synchronize()
        u_ms = max_over_ranks(u0.elapsed_time(u1), world)
        u_rays = sum_over_ranks(int(rend.counts[:3].sum()), world)
        lbvh_topology = {"mrays_s": round(u_rays / (u_ms / 1e3) / 1e6, 3), "ms_per_step": round(u_ms, 3),
                         "note": "one frame traversing the reference-topology LBVH instead of the split BVH"}
        lb.split(split, keep_scratch=True, flags=split_flags(args))
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        lb.split(split, keep_scratch=True, flags=split_flags(args))
        s1.record(stream)
        torch.cuda.synchronize()
        lbvh_topology["split_build_ms"] = round(s0.elapsed_time(s1), 3)
        if args.wide:
            # both collapses timed; the tree left for what follows is the workload's
            for key, sah in (("wide_build_ms", False), ("wide_sah_build_ms", True)):
                lb.wide(keep_scratch=True, sah=sah)
                torch.cuda.synchronize()
                s0.record(stream)
                lb.wide(keep_scratch=True, sah=sah)
                s1.record(stream)
                torch.cuda.synchronize()
                lbvh_topology[key] = round(s0.elapsed_time(s1), 3)
            lb.wide(keep_scratch=True, sah=bool(args.wide_sah))

    # --- LBVH build of the same scene (device-resident triangles); the deforming
    # workload already rebuilt inside every timed step: those builds are reported
    if deforming:
        nb = args.steps
        bprof = {k: v for k, v in prof.items()
                 if k in ("k_bounds", "k_morton", "k_scan_offsets", "k_onesweep", "k_topology", "k_gather_refit")}
        build_ms = max_over_ranks(sum(v[0] for v in bprof.values()) / nb, world)
    else:
        for _ in range(max(3, args.warmup)):
            lb.build(d_tris)
        torch.cuda.synchronize()
        nb = max(5, args.steps)
        cpt.profile_begin()
        b0 = torch.cuda.Event(enable_timing=True)
        b1 = torch.cuda.Event(enable_timing=True)
        b0.record(stream)
        for _ in range(nb):
            lb.build(d_tris)
        b1.record(stream)
        torch.cuda.synchronize()
        bprof = cpt.profile_end()
        build_ms = max_over_ranks(b0.elapsed_time(b1) / nb, world)
    lb.status()
    key_bytes = 4 if w["bits"] == 30 else 8
    passes = 4 if w["bits"] == 30 else 8
    # algorithmic bytes per triangle: Morton 36 in + K+4 out, histogram K, sort 2P(K+4),
    # gather 40+40, topology K + 4 + 8, refit 8 + 36 + 8 + 4 + 24, plus the 64-B node and 48-B record
    bpt = 36 + key_bytes + 4 + key_bytes + 2 * passes * (key_bytes + 4) + 80 + key_bytes + 12 + 80 + 64 + 48
    b_ach = n * bpt / (build_ms / 1e3) / 1e9
    lbvh = {"mtris_s": round(n / build_ms / 1e3, 2), "ms": round(build_ms, 4),
            "roofline": {"bound": "hbm", "achieved": round(b_ach, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(b_ach / peak, 4), "bytes_per_triangle": bpt},
            "kernel_ms_per_build": {k: round(v[0] / nb, 4) for k, v in sorted(bprof.items())}}
    if args.dump_accum and rank == 0:  # the first view's Kahan accumulator after the timed frames (checks)
        torch.cuda.synchronize()
        np.save(args.dump_accum, my_accums[0].cpu().numpy())
    if deforming and pipelined:
        lbvh["note"] = ("every frame's rebuild (deform + cpt_lbvh_build) runs on a side stream beside the previous "
                        "frame's render (two trees): these kernel times include that contention; the uncontended "
                        "build of this mesh is the C2 line's builds_c5_c3.c5_rebuild")

    # --- end to end through the tracer object (host buffers, pinned)
    e2e = None
    if not args.no_e2e and not deforming:
        tr = cpt.Tracer(w["bits"])
        e2e_split = w.get("e2e_split", split) if args.split is None else split
        e2e_treelet = w.get("e2e_treelet", args.treelet) if args.treelet_given is None else args.treelet
        tr.set_split(e2e_split, cpt.SPLIT_TREELET if e2e_treelet and e2e_split > 0 else 0)
        tr.set_wide(bool(args.wide))
        tr.set_settings(bounces=w["bounces"], intensity=3.0, stratified=True, seed=w["seed"] + 7919 * rank)
        # (the tracer object renders frame 0 of its own seed on every rank: e2e ranks are replicas)
        tr.set_camera(cams[0])
        h_tris = torch.empty(tris.nbytes, dtype=torch.uint8, pin_memory=True)
        h_tris.numpy()[:] = tris.view(np.uint8)
        h_infos = torch.empty(infos.nbytes, dtype=torch.uint8, pin_memory=True)
        h_infos.numpy()[:] = infos.view(np.uint8)
        h_img = torch.empty(W_ * H_ * 16, dtype=torch.uint8, pin_memory=True)
        lib = cpt.lib

        def upload():
            cpt.check(lib.cpt_tracer_upload(tr._h, h_tris.data_ptr(), n, h_infos.data_ptr(), n, None, 0, None),
                      "upload")

        def e2e_steps(k):
            """k steps, each: the scene's upload from pinned host memory and its builds, a
            16-spp frame, the image read back to host memory. The tracer keeps two scenes,
            so step i+1's upload and builds are issued before step i's read-back and run
            beside step i's frame."""
            upload()
            tr.raytrace(W_, H_, spp)
            for i in range(k):
                if i + 1 < k:
                    upload()
                cpt.check(lib.cpt_tracer_read_image(tr._h, h_img.data_ptr()), "read_image")
                if i + 1 < k:
                    tr.raytrace(W_, H_, spp)

        e2e_steps(max(1, min(args.warmup, 2)))
        ts = torch.cuda.ExternalStream(tr.stream)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        ne = max(2, min(args.steps, 5))
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        e0.record(ts)
        e0.synchronize()  # (the first upload goes on the tracer's build stream: it starts after e0)
        e2e_steps(ne)
        e1.record(ts)
        e1.synchronize()
        wall = time.perf_counter() - w0
        # upload() restarts the frame counter and the ray counters: every step renders
        # the same first frame, and the counters hold one step's rays
        e_ms = e0.elapsed_time(e1)
        e_rays = float(tr.ray_counts().sum()) * ne
        e_ms_max = max_over_ranks(e_ms, world)
        e_rays_all = sum_over_ranks(e_rays, world)
        e2e = {"value": round(e_rays_all / (e_ms_max / 1e3) / 1e6, 3), "unit": METRIC,
               "h2d_bytes_per_step": int(tris.nbytes + infos.nbytes), "d2h_bytes_per_step": int(W_ * H_ * 16),
               "ms_per_step": round(e_ms_max / ne, 3), "wall_ms_per_step": round(1e3 * wall / ne, 3),
               "steps": ne, "pipelined": "the next step's upload and builds run beside this step's frame "
                                         "(the tracer's two scenes); every step's copies, builds, frame and "
                                         "read-back are inside the timed region",
               "includes": "H2D soup+shading records (pinned), LBVH build"
                                        + (f", split BVH build (extra {e2e_split}"
                                           + (", treelet-restructured" if e2e_treelet else ", Karras topology")
                                           + ")" if e2e_split > 0 else "")
                                        + (", wide tree build" if args.wide else "")
                                        + ", 16-spp frame, D2H image"}
        tr.close()

    # the LBVH timing above rebuilt the tree (dropping the split and wide trees): the
    # measurements below use the benchmark's own traversal tree again
    if not deforming:
        lb.build(d_tris)
        if split > 0:
            lb.split(split, keep_scratch=True, flags=split_flags(args))
        if args.wide:
            lb.wide(keep_scratch=True, sah=bool(args.wide_sah))
        torch.cuda.synchronize()

    # --- radiance cache (the C4 configuration on this scene and tree): time to reach the
    # plain tracer's 64-sample error against an FP64 image, 1-sample cached frames
    cache_c4, r4 = None, None
    if rank == 0 and world == 1 and args.workload == "c2" and not args.no_cache_ratio:
        wc = dict(WORKLOADS["c4"])
        wc.update(width=W_, height=H_)
        if args.rc_warm is not None:
            wc["warm_updates"] = args.rc_warm
        try:
            r4 = cache_experiment(wc, lb, scene, cams[0], dev, True, args.warmup, wc["spp"],
                                  rc_params_for(args, wc["spp"]))
        except Exception as e:  # an extra measurement never takes the main line down
            r4 = None
            cache_c4 = {"error": f"{type(e).__name__}: {e}"[:300]}
    if r4 is not None:
        cache_c4 = {"metric": "time-to-equal-RMSE (cache / plain, vs FP64 image), stratified first bounce",
                    "value": r4["ratio"], "unit": "x", "higher_is_better": False,
                    "value_same_frames": r4["ratio_same_frames"],
                    "note": "value: plain tracer in 16-sample frames (its fastest); value_same_frames: plain "
                            "tracer in frames of the cached tracer's size (1 sample, the C4 configuration)",
                    "plain_same_frames_ms": r4["plain_same_frames_ms"],
                    "plain": r4["plain"], "cache": {k: r4["cache"][k] for k in
                                                    ("spp", "spp_per_frame", "ms", "warm_ms", "reached", "mrays_s",
                                                     "training_samples_last_frame", "training")},
                    "reference": r4["reference"], "curve_tail": r4["cache_curve"][-4:]}

    # --- build measurements at the C5 and C3 scales (default C2 run, rank 0)
    builds = None
    if rank == 0 and world == 1 and args.workload == "c2" and not args.no_extra_builds:
        try:
            builds = extra_builds(dev)
        except Exception as e:  # an extra measurement never takes the main line down
            builds = {"error": f"{type(e).__name__}: {e}"[:300]}
        torch.cuda.empty_cache()

    # --- the other workloads (default C2 run, rank 0): short child runs of C1, C3 and C5
    workloads = None
    if rank == 0 and world == 1 and args.workload == "c2" and not args.no_other_workloads:
        torch.cuda.empty_cache()
        workloads = other_workloads()

    # --- CPU baseline (rank 0, N = 1): the reference's code on every k-th row of frame 0,
    # and the parity of the GPU's frame 0 (FP64 accumulator, same traversal tree as the
    # timed frames) on those rows
    cpu_base, parity, ref_gpu = None, None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_reference_run(w, tris, infos, cams[0], w["bits"], target_s=args.cpu_seconds)
        cpu_base = {"value": round(r["mrays_s"], 4), "unit": METRIC, "cores": r["threads"], "kind": r["kind"],
                    "sample": r["sample"], "build_mtris_s": round(r["build_mtris_s"], 3)}
        if not deforming and cached is None:
            pr = DeviceRenderer(make_params(W_, H_, spp, 0, w["bounces"], 3.0, True, w["seed"], cpt.ACCUM_F64,
                                            wave_paths=args.wave_paths), dev)
            pr.render(lb, scene, cams[0], frame0=0)
            torch.cuda.synchronize()
            pr.check_status()
            acc = pr.accum.view(torch.float64).view(H_, W_, 4)
            gpu_rows = acc[torch.as_tensor(r["rows"].astype(np.int64), device=dev), :, :3].cpu().numpy()
            parity = frame_parity(gpu_rows, r["sums"], spp)
            frame_rays = float(pr.counts[:3].sum())
            parity["against"] = f"{r['kind']} ({'oracle/_ref: the reference compiled from source' if r['kind'] == 'reference' else 'oracle port'}) on the LBVH"
            cpu_base["sample_rays_share"] = round(r["rays"] / max(frame_rays, 1.0), 5)
            cpu_base["sample_rows_share"] = round(len(r["rows"]) / H_, 5)
            del pr
        ref_gpu = reference_gpu(w, tris, infos, cams[0], dev, ms_max / args.steps / spp, rays_all / args.steps / spp)

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 3), "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded host generator)",
                "config": workload_config(args.workload, w, n, "scene arrays (LBVH 1.4 GB, traversal trees more) > "
                                                               "126 MB L2, no flush needed"),
                "rays_per_step": int(rays_all / args.steps), "roofline": roofline, "lbvh": lbvh,
                "traversal_bvh": (("compressed 8-wide tree (cpt_lbvh_wide) over the " if args.wide else "")
                                  + (f"split BVH (cpt_lbvh_split, extra pieces {split} x n"
                                     + (", treelet-restructured" if args.treelet else "") + ")" if split > 0
                                     else "LBVH (reference topology)")), "lbvh_topology": lbvh_topology,
                "cpu_baseline": cpu_base, "parity": parity, "reference_gpu": ref_gpu,
                "radiance_cache_c4": cache_c4, "builds_c5_c3": builds, "workloads": workloads, "e2e": e2e,
                "gpu_launches": int(launches),
                "clocks": clocks,
                "parallelism": f"replicas x{world}: own BVH per GPU, disjoint sample streams, "
                               f"framebuffer reduce to rank 0 per frame" if world > 1 else "1 GPU",
                "scene_gen_s": round(gen_s, 2)}
        print(json.dumps(line), flush=True)
    return 0


def other_workloads(timeout_s=240.0):
    """C1, C3 and C5 as short runs of this script in child processes (the default C2
    line carries their headline figures). Each child is a full run of its workload
    (its own scene, build, warm-up and timed frames, CUDA events, clocks), without the
    CPU baseline and the end-to-end leg; what comes back is the child's JSON line,
    reduced to its measurements."""
    runs = {"c1": ["--steps", "10", "--warmup", "3"], "c3": ["--steps", "3", "--warmup", "3"],
            "c5": ["--steps", "5", "--warmup", "3"]}
    out = {}
    for wl, extra in runs.items():
        cmd = [sys.executable, os.path.abspath(__file__), "--workload", wl, "--no-cpu-baseline", "--no-e2e"] + extra
        t0 = time.perf_counter()
        try:
            p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s, cwd=os.path.dirname(
                os.path.abspath(__file__)))
            lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
            if p.returncode != 0 or not lines:
                out[wl] = {"error": f"exit {p.returncode}: {p.stderr.strip()[-300:]}"}
                continue
            d = json.loads(lines[-1])
        except Exception as e:  # an extra measurement never takes the main line down
            out[wl] = {"error": f"{type(e).__name__}: {e}"[:300]}
            continue
        keep = ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "rays_per_step", "clocks",
                "gpu_launches", "built_and_rendered_per_frame", "lbvh", "parallelism")
        r = {k: d[k] for k in keep if k in d}
        r["workload"] = d.get("config", {}).get("workload")
        if isinstance(d.get("roofline"), dict):
            r["roofline_frac"] = d["roofline"].get("frac")
        r["command"] = "python bench.py " + " ".join(cmd[2:])
        r["child_s"] = round(time.perf_counter() - t0, 1)
        out[wl] = r
    return out


def cache_experiment(w, lb, scene, cam, dev, stratified, warmup, spf, rc_params, nee=False, reach=None):
    """Time-to-equal-RMSE of the radiance cache against the plain tracer on one scene.

    The plain tracer renders plain_spp samples per pixel in frames of 16 samples (time
    T_plain, error RMSE_plain against an FP64-accumulated image of ref_spp samples). The
    cached tracer starts from untrained weights: warm_updates training-only frames
    (cpt_rc_update), then frames of `spf` samples (each trains on the frame's own
    training paths and renders the image) until its error reaches RMSE_plain (time
    T_cache, warm-up included); ratio = T_cache / T_plain. The error is taken on every
    ref_div-th pixel in x and y: the FP64 image is rendered at (W / ref_div) x (H /
    ref_div), whose primary rays are exactly those of that pixel subgrid (the ray through
    pixel x of W is the bilinear blend at x / W). Frames are timed with CUDA events; the
    error checks between them are not. With nee and reach (an RMSE), also measures how
    long the next-event plain tracer takes to reach it, in frames of 1 sample."""
    import torch

    import cpt
    from cpt.device import BatchRenderer, CachedRenderer, RadianceCache, make_params

    W_, H_ = w["width"], w["height"]
    rdiv = w["ref_div"]
    rw, rh = W_ // rdiv, H_ // rdiv
    stream = torch.cuda.current_stream()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    t0 = time.perf_counter()
    refp = make_params(rw, rh, w["ref_spp"], 0, w["bounces"], 3.0, stratified, w["seed"] + 99991, cpt.ACCUM_F64,
                       nee=nee)
    ref = BatchRenderer([(lb, scene, cam, rw, rh)], refp, dev)
    ref.render()
    torch.cuda.synchronize()
    ref.check_status()
    ri = ref.accums[0].view(torch.float64).view(rh, rw, 4)
    ref_img = ri[..., :3] / ri[..., 3:4].clamp(min=1)
    ref_s = time.perf_counter() - t0
    del ref

    def rmse(acc):
        a = acc.view(torch.float32).view(2, H_, W_, 4)[0]
        img = (a[..., :3] / a[..., 3:4].clamp(min=1)).double()[::rdiv, ::rdiv][:rh, :rw]
        return float(torch.sqrt(((img - ref_img) ** 2).mean()))

    pp = make_params(W_, H_, 16, 0, w["bounces"], 3.0, stratified, w["seed"], cpt.ACCUM_KAHAN, nee=nee)
    plain = BatchRenderer([(lb, scene, cam, W_, H_)], pp, dev)
    for i in range(max(1, warmup)):
        plain.render(frame0=100000 + 16 * i)
    torch.cuda.synchronize()

    def plain_run(frame_spp):
        """The plain tracer's first plain_spp samples in frames of frame_spp samples: time,
        and the accumulator (the same samples in the same order whatever the frame size)."""
        plain.accums[0].zero_()
        plain.counts.zero_()
        t = 0.0
        for f in range(w["plain_spp"] // frame_spp):
            t += timed(lambda: plain.render(frame0=frame_spp * f, spp=frame_spp))
        return t

    t_plain_same = plain_run(spf) if spf != 16 else None  # frames of the cached tracer's size
    t_plain = plain_run(16)
    plain.check_status()
    rmse_plain = rmse(plain.accums[0])
    plain_rays = int(plain.counts[:3].sum())
    reach_out = None
    if reach is not None:
        plain.accums[0].zero_()
        t_r, k, got = 0.0, 0, None
        while k < w["plain_spp"]:
            t_r += timed(lambda: plain.render(frame0=k, spp=1))
            k += 1
            e = rmse(plain.accums[0])
            if e <= reach:
                got = e
                break
        reach_out = {"target_rmse": round(reach, 6), "spp": k, "ms": round(t_r, 2),
                     "rmse": None if got is None else round(got, 6)}
    del plain

    rc = RadianceCache(rc_params)
    cp = make_params(W_, H_, spf, 0, w["bounces"], 3.0, stratified, w["seed"], cpt.ACCUM_KAHAN, nee=nee)
    cr = CachedRenderer(rc, [(lb, scene, cam, W_, H_)], cp, dev)
    cr.render(frame0=200000)  # warm the kernels on a throwaway network
    torch.cuda.synchronize()
    rc.reset(1337)
    cr.accums[0].zero_()
    cr.counts.zero_()
    cpt.profile_begin()
    launches0 = cpt.launch_count()
    t_cache = 0.0
    for u in range(w["warm_updates"]):
        t_cache += timed(lambda: cr.update(frame0=300000 + u))
    t_warm = t_cache
    spp, curve, reached = 0, [], False
    while spp < w["max_spp"]:
        t_cache += timed(lambda: cr.render(frame0=spp))
        spp += spf
        e = rmse(cr.accums[0])
        curve.append((spp, round(t_cache, 1), round(e, 6)))
        if e <= rmse_plain:
            reached = True
            break
    prof = cpt.profile_end()
    launches = cpt.launch_count() - launches0
    cr.check_status()
    cache_rays = int(cr.counts[:3].sum())
    samples_last = rc.sample_count()
    rc.close()
    # the curve at the plain tracer's sample count, for the record
    return {"stratified": stratified, "nee": nee, "ratio": round(t_cache / t_plain, 4) if reached else None,
            "ratio_same_frames": (round(t_cache / t_plain_same, 4) if reached and t_plain_same else None),
            "plain_same_frames_ms": None if t_plain_same is None else round(t_plain_same, 2),
            "t_cache_ms": round(t_cache, 2), "cache_curve": curve if len(curve) <= 80 else curve[::4] + curve[-1:],
            "plain_to_reference_rmse": reach_out,
            "plain": {"spp": w["plain_spp"], "frames_spp": 16, "ms": round(t_plain, 2), "rmse": round(rmse_plain, 6),
                      "mrays_s": round(plain_rays / t_plain / 1e3, 3)},
            "cache": {"spp": spp, "spp_per_frame": spf, "warm_updates": w["warm_updates"],
                      "warm_ms": round(t_warm, 2), "ms": round(t_cache, 2), "reached": reached,
                      "mrays_s": round(cache_rays / t_cache / 1e3, 3), "training_samples_last_frame": samples_last,
                      "training": f"about {rc_params.train_samples} of a frame's own paths traced to full depth, "
                                  f"every {max(1, rc_params.train_interval)} frame(s)",
                      "kernel_ms": {k: round(v[0], 3) for k, v in sorted(prof.items())}},
            "reference": {"resolution": f"{rw}x{rh} (every {rdiv}th pixel of {W_}x{H_})",
                          "spp": w["ref_spp"], "accum": "f64", "s": round(ref_s, 2)},
            "launches": int(launches)}


def rc_params_for(args, spf):
    """2^16 training paths and 4 optimiser steps per training frame (one render call of
    `spf` samples; every --rc-interval-th frame trains), or — with --rc-per-sample — per
    image sample."""
    from cpt.device import rc_default_params

    p = rc_default_params(train_interval=args.rc_interval)
    if args.rc_train_paths:
        p.train_samples = args.rc_train_paths
    if args.rc_per_sample:
        p.train_samples *= spf
        p.train_steps *= spf
    return p


def run_cache(args, w, world, rank, local):
    """The radiance-cache workload (cache_experiment) on the C2 scene, stratified and
    independent first bounces, and with next-event estimation in both tracers."""
    import torch

    import cpt
    from cpt.device import DeviceLbvh, DeviceScene, to_device

    dev = torch.device("cuda", local if world > 1 else 0)
    tris, infos = make_scene(w)
    n = len(tris)
    cam = make_cameras(w)[0]
    lb = DeviceLbvh(n, w["bits"], dev)
    lb.build(to_device(tris, dev), check_root=True)
    split = w.get("split", 0.0) if args.split is None else args.split
    if split > 0:
        lb.split(split, flags=split_flags(args))
    if args.wide:
        lb.wide(sah=bool(args.wide_sah))
    scene = DeviceScene(infos, None, dev)
    scene.build_emitters(lb)
    spf = w["spp"]
    rcp = rc_params_for(args, spf)

    def experiment(stratified, nee=False, reach=None):
        return cache_experiment(w, lb, scene, cam, dev, stratified, args.warmup, spf, rcp, nee=nee, reach=reach)

    main_run = experiment(True)
    alt = experiment(False)
    nee_runs = ([experiment(True, True, main_run["plain"]["rmse"]), experiment(False, True, alt["plain"]["rmse"])]
                if args.nee else [])

    def nee_summary(ref_run, nee_run):
        """Next-event estimation against the reference estimator's plain 64-sample
        RMSE: the plain tracer with it, and the cached tracer with it."""
        target, t_ref = ref_run["plain"]["rmse"], ref_run["plain"]["ms"]
        r = nee_run["plain_to_reference_rmse"]
        first = next((c for c in nee_run["cache_curve"] if c[2] <= target), None)
        return {"target_rmse": target, "reference_plain_ms": t_ref,
                "plain_nee_ratio": round(r["ms"] / t_ref, 4) if r and r["rmse"] is not None else None,
                "plain_nee": r,
                "cache_nee_ratio": round(first[1] / t_ref, 4) if first else None,
                "cache_nee": {"spp": first[0], "ms": first[1], "rmse": first[2]} if first else None,
                "cache_vs_plain_both_nee": nee_run["ratio"]}
    if rank == 0:
        line = {"metric": "time-to-equal-RMSE (cache / plain, vs FP64 image)", "value": main_run["ratio"],
                "value_same_frames": main_run["ratio_same_frames"],
                "note": "value: plain tracer in 16-sample frames (its fastest); value_same_frames: plain tracer in "
                        "frames of the cached tracer's size",
                "unit": "x", "n_gpus": world, "steps": main_run["cache"]["spp"] // spf, "warmup": args.warmup,
                "ms_per_step": round(main_run["cache"]["ms"] / max(1, main_run["cache"]["spp"] // spf), 3),
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 tracing, bf16 MLP (f32 accumulate)", "data": "synthetic (seeded host generator)",
                "config": workload_config("c4", w, n, "scene arrays (LBVH 1.4 GB, traversal trees more) > 126 MB L2, "
                                                "no flush needed"),
                "stratified": main_run, "unstratified": alt,
                "next_event": ({"stratified": nee_summary(main_run, nee_runs[0]),
                                "unstratified": nee_summary(alt, nee_runs[1]),
                                "runs": {"stratified": nee_runs[0], "unstratified": nee_runs[1]}}
                               if nee_runs else None),
                "rc_params": {"train_samples": rcp.train_samples, "train_steps": rcp.train_steps,
                              "learning_rate": rcp.learning_rate, "beta2": rcp.beta2},
                "gpu_launches": main_run["launches"]}
        print(json.dumps(line), flush=True)
    return 0


def split_flags(args) -> int:
    """cpt_lbvh_split flags of the run: treelet restructuring on request."""
    import cpt

    return cpt.SPLIT_TREELET if args.treelet else 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c2")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extra-builds", action="store_true",
                    help="c2: skip the C5-scale rebuild and the C3 batched build measurements")
    ap.add_argument("--no-other-workloads", action="store_true",
                    help="c2: skip the C1, C3 and C5 runs (short child runs reported under 'workloads')")
    ap.add_argument("--no-cache-ratio", action="store_true",
                    help="c2: skip the radiance cache's time-to-equal-RMSE measurement (the C4 configuration)")
    ap.add_argument("--res", default=None, help="override resolution WxH (profiling runs)")
    ap.add_argument("--spp", type=int, default=None, help="override samples per frame (profiling runs)")
    ap.add_argument("--sphere", default=None, help="override the sphere's grid NUxNV (profiling runs)")
    ap.add_argument("--hair", type=int, default=None, help="override the hairball's triangle count (profiling runs)")
    ap.add_argument("--scenes", type=int, default=None, help="c3: override the scene count (profiling runs)")
    ap.add_argument("--wave-paths", type=int, default=0, help="paths per wave (0: library default)")
    ap.add_argument("--ray-sort", type=int, default=0, help="1: coherence-sort bounce queues")
    ap.add_argument("--refill-lanes", type=int, default=0,
                    help="traversal warps take new rays below this many busy lanes (0: library default)")
    ap.add_argument("--blocks-per-sm", type=int, default=0,
                    help="resident traversal blocks per SM (0: occupancy)")
    ap.add_argument("--wave-lanes", type=int, default=0,
                    help="1: one launch sequence per wave, 2: two half-waves on two streams (0: library default)")
    ap.add_argument("--wide", type=int, default=None,
                    help="1: traverse the compressed 8-wide tree built from the (split) binary tree, 0: the binary "
                         "tree (default per workload)")
    ap.add_argument("--wide-sah", type=int, default=None,
                    help="1: the surface-area collapse (CPT_WIDE_SAH) for trees built once before the timed frames; "
                         "trees rebuilt inside a timed step always use the faster largest-child collapse "
                         "(default per workload)")
    ap.add_argument("--dump-accum", default=None, help="save the first view's accumulator after the timed frames "
                                                        "(a .npy path; for checks)")
    ap.add_argument("--c5-pipeline", type=int, default=1,
                    help="c5: build frame f+1's tree on a side stream while frame f renders (two trees); 0: rebuild "
                         "then render, one after the other")
    ap.add_argument("--split-streams", type=int, default=8,
                    help="c3: side streams for the split trees of the frame's rebuild (1: one after another)")
    ap.add_argument("--rc-per-sample", action="store_true",
                    help="c4: 2^16 training suffixes per image sample instead of per render call (frame)")
    ap.add_argument("--rc-interval", type=int, default=16,
                    help="radiance cache: train on every n-th frame's own paths (the others only read the cache)")
    ap.add_argument("--rc-warm", type=int, default=None,
                    help="radiance cache: training-only updates before the first cached frame (default per workload)")
    ap.add_argument("--rc-train-paths", type=int, default=0,
                    help="radiance cache: training paths per training frame (0: the library default, 2^16)")
    ap.add_argument("--nee", type=int, default=1,
                    help="c4: also compare with next-event estimation in both tracers (1) or not (0)")
    ap.add_argument("--split", type=float, default=None,
                    help="split traversal BVH extra-piece ratio (0: traverse the LBVH; default per workload)")
    ap.add_argument("--treelet", type=int, default=None,
                    help="1: treelet restructuring of the split BVH's topology (CPT_SPLIT_TREELET), 0: the Karras "
                         "topology (default per workload)")
    args = ap.parse_args()
    w = dict(WORKLOADS[args.workload])
    if args.wide is None:
        args.wide = int(w.get("wide", 0))
    if args.wide_sah is None:
        args.wide_sah = int(w.get("wide_sah", 0))
    args.treelet_given = args.treelet
    if args.treelet is None:
        args.treelet = int(w.get("treelet", 0))
    if args.res:
        w["width"], w["height"] = (int(x) for x in args.res.lower().split("x"))
    if args.spp:
        w["spp"] = args.spp
    if args.rc_warm is not None and "warm_updates" in w:
        w["warm_updates"] = args.rc_warm
    if args.sphere:
        w["nu"], w["nv"] = (int(x) for x in args.sphere.lower().split("x"))
    if args.hair is not None:
        w["n_hair"] = args.hair
    if args.scenes is not None:
        w["scenes"] = args.scenes
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        return run_reference_arm(args, w, world, rank)
    world, rank, local = dist_setup(args.gpus)
    try:
        if w["kind"] == "batch":
            return run_batch(args, w, world, rank, local)
        if args.workload == "c4":
            return run_cache(args, w, world, rank, local)
        return run_ours(args, w, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
