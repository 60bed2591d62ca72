"""Runs the reference's own GPU code (oracle/_ref/librefgpu.so) in a process of its own.

TEST AND BASELINE INFRASTRUCTURE ONLY. The tests and the benchmark's baseline leg
call `run(...)`, which starts this file as a child process: the reference's thrust
and CUDA runtime then live in a process that has loaded nothing else, and whatever
happens there ends that process, not the caller. Inputs and outputs travel as one
.npz file each.

    python -m oracle.refgpu_child <in.npz> <out.npz>

in.npz: tris (40-B records as uint8), infos (192-B records as uint8, optional), box
(6 float32), op ("build" | "render"), and for render: width, height, cam15, bounces,
intensity, stratified, warmup, frames, seed; for build: reps, outputs.
out.npz: the timings as float arrays, and the build's arrays or the render's image.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def run(op: str, tris: np.ndarray, box, infos=None, timeout: float = 600.0, **kw) -> dict:
    """Runs `op` in a child process and returns its results (numpy arrays and floats);
    raises RuntimeError with the child's exit status and the end of its stderr."""
    with tempfile.TemporaryDirectory() as d:
        src, dst = os.path.join(d, "in.npz"), os.path.join(d, "out.npz")
        arrays = {"tris": np.ascontiguousarray(tris).view(np.uint8), "box": np.asarray(box, np.float32),
                  "op": np.array(op)}
        if infos is not None:
            arrays["infos"] = np.ascontiguousarray(infos).view(np.uint8)
        for k, v in kw.items():
            arrays[k] = np.asarray(v)
        np.savez(src, **arrays)
        p = subprocess.run([sys.executable, "-m", "oracle.refgpu_child", src, dst], cwd=os.path.dirname(HERE),
                           capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0 or not os.path.exists(dst):
            raise RuntimeError(f"reference GPU child exited {p.returncode}: {p.stderr[-800:].strip()}")
        with np.load(dst) as z:
            return {k: z[k] for k in z.files}


def _trace(what: str) -> None:
    if os.environ.get("CPT_REFGPU_TRACE"):
        print(f"refgpu_child: {what}", file=sys.stderr, flush=True)


def _main(src: str, dst: str) -> int:
    sys.path.insert(0, os.path.dirname(HERE))
    _trace("start")
    from oracle import cpu

    _trace("oracle imported")
    cpu.refgpu_lib()
    _trace("library loaded")

    z = np.load(src)
    op = str(z["op"])
    tris = z["tris"].view(cpu.TRIANGLE_DTYPE)
    box = z["box"]
    out = {}
    if op == "build":
        stats, r = cpu.refgpu_build(tris, box=box, reps=int(z["reps"]), outputs=bool(z["outputs"]))
        out.update({k: np.float64(v) for k, v in stats.items()})
        if r is not None:
            out.update(tris_out=r.tris.view(np.uint8), children=r.children, parents_leaf=r.parents_leaf,
                       parents_internal=r.parents_internal, node_boxes=r.node_boxes.view(np.float32))
    elif op == "render":
        infos = z["infos"]
        stats, img = cpu.refgpu_render(tris, infos, int(z["width"]), int(z["height"]), z["cam15"], int(z["bounces"]),
                                       float(z["intensity"]), bool(z["stratified"]), int(z["warmup"]),
                                       int(z["frames"]), int(z["seed"]), box=box, image=True)
        out.update({k: np.float64(v) for k, v in stats.items()})
        out["image"] = img
    else:
        print(json.dumps({"error": f"unknown op {op}"}), file=sys.stderr)
        return 2
    _trace(f"{op} returned")
    np.savez(dst, **out)
    _trace("results written")
    return 0


if __name__ == "__main__":
    sys.exit(_main(sys.argv[1], sys.argv[2]))
