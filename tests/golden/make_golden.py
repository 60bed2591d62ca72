"""Regenerates the golden LBVH / traversal fixtures from the reference itself.

Runs the reference's own CUDA::BVHBuilder::build and CUDA::trace
(source/application/cuda/BVHBuilder.cu:207-269, trace.h:73-169), compiled on the
host by `make -C oracle ref` (oracle/_ref/libref.so for the shipped 30-bit key
configuration, libref64.so for the 63-bit one), on small seeded inputs, and
stores inputs and outputs as .npz files here. The tests compare the oracle and
the GPU path against these files, so they need neither the reference tree nor
its compiled form at run time.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "cuda-path-tracer_b200"))

import cpt  # noqa: E402  (host-only scene generator, no GPU needed)
from oracle import cpu  # noqa: E402


def quantized(tris: np.ndarray, step: float) -> np.ndarray:
    """Snap vertices to a coarse grid: many equal centroids -> many equal keys."""
    t = tris.copy()
    for f in ("v0", "v1", "v2"):
        t[f] = (np.round(t[f] / step) * step).astype(np.float32)
    return t


def rays_for(tris: np.ndarray, n: int, seed: int) -> np.ndarray:
    """Half the rays aim at random triangle centroids (hits), half are random
    (mostly misses); an eighth have an exactly zero x direction component."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(-0.3, 1.3, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    pick = rng.integers(0, len(tris), n // 2)
    cen = (tris["v0"][pick] + tris["v1"][pick] + tris["v2"][pick]) / 3.0
    d[: n // 2] = (cen - o[: n // 2]).astype(np.float32)
    d[n // 2: n // 2 + n // 8, 0] = 0.0  # axis-parallel: 1/d = inf in the slab test
    return np.concatenate([o, d], 1).astype(np.float32)


CASES = {
    # name: (generator, bits)
    "random2k_30": (lambda: cpt.scene_random(2000, seed=7)[0], 30),
    "random2k_63": (lambda: cpt.scene_random(2000, seed=7)[0], 63),
    "ties1k_30": (lambda: quantized(cpt.scene_random(1000, seed=3)[0], 0.125), 30),
    "sphere_63": (lambda: cpt.scene_sphere_hairball(24, 12, 300, seed=5)[0], 63),
    "tiny2_30": (lambda: cpt.scene_random(0, seed=1)[0], 30),  # the 2-triangle emitter quad alone
}


def main() -> None:
    for name, (gen, bits) in CASES.items():
        tris = np.ascontiguousarray(gen())
        box = cpu.enclosing_box(tris)
        r = cpu.build(tris, bits, box=box, use_ref=True)
        rays = rays_for(tris, 512, seed=len(tris))
        ref = cpu.ref_lib(bits)
        ref.ref_set_geometry(r.tris.ctypes.data, r.children.ctypes.data, r.node_boxes.ctypes.data, len(r.tris))
        t = np.zeros(len(rays), np.float32)
        idx = np.zeros(len(rays), np.uint32)
        uv = np.zeros((len(rays), 2), np.float32)
        ref.ref_trace(rays.ctypes.data, len(rays), t.ctypes.data, idx.ctypes.data, uv.ctypes.data, 1)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), bits=np.int32(bits), tris_in=tris, box=box,
                            tris=r.tris, keys=r.keys, children=r.children, parents_leaf=r.parents_leaf,
                            parents_internal=r.parents_internal, node_boxes=r.node_boxes, rays=rays, t=t, idx=idx,
                            uv=uv)
        print(name, len(tris), "hits", int((idx != cpu.INVALID).sum()))


if __name__ == "__main__":
    main()
