"""ctypes access to the CPU oracle (liboracle.so) and, when it was compiled, to the
reference's own builder / traversal (oracle/_ref/libref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the
checker and by bench.py's CPU-baseline leg. Nothing in the product imports it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref.so")      # reference, 30-bit keys (as shipped)
REF64_LIB = os.path.join(HERE, "_ref", "libref64.so")  # reference, 63-bit key configuration
REFGPU_LIB = os.path.join(HERE, "_ref", "librefgpu.so")  # reference's GPU LBVH build (sm_100a), 30-bit as shipped

TRIANGLE_DTYPE = np.dtype([("v0", "<f4", 3), ("v1", "<f4", 3), ("v2", "<f4", 3), ("info_idx", "<u4")])
BBOX_DTYPE = np.dtype([("min", "<f4", 3), ("max", "<f4", 3)])
INVALID = 0xFFFFFFFF
FLT_MAX = np.float32(3.4028234663852886e38)


class OCam(ctypes.Structure):
    _fields_ = [("eye", ctypes.c_float * 3), ("dirs", (ctypes.c_float * 3) * 4), ("inv_view_proj", ctypes.c_float * 16),
                ("jitter_x", ctypes.c_float), ("jitter_y", ctypes.c_float), ("jitter", ctypes.c_uint32)]


def _p(a):
    return None if a is None else a.ctypes.data


_oracle = None
_ref = {}


def oracle_lib() -> ctypes.CDLL:
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_LIB):
            raise ImportError(f"{ORACLE_LIB} missing: run `make -C oracle`")
        L = ctypes.CDLL(ORACLE_LIB)
        P, U, I, F = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_float
        L.orc_morton.argtypes = [P, U, P, I, P]
        L.orc_enclosing_box.argtypes = [P, U, P]
        L.orc_build.argtypes = [P, U, P, I, P, P, P, P, P, P]
        L.orc_build.restype = I
        L.orc_trace.argtypes = [P, P, P, U, P, U, I, P, P, P, P]
        L.orc_render.argtypes = [P, P, P, U, P, P, U, U, U, U, U, U, U, U, F, I, U, U, ctypes.POINTER(OCam), U, P, P]
        L.orc_render_f64.argtypes = [P, P, P, U, P, P, U, U, U, U, U, U, F, I, U, U, ctypes.POINTER(OCam), P]
        L.orc_philox.argtypes = [P, U, U, P]
        L.orc_sincos_turns.argtypes = [P, U, P, P]
        L.orc_corner_dirs.argtypes = [ctypes.POINTER(OCam), U, U, U, P]
        L.orc_heatmap.argtypes = [P, P, ctypes.POINTER(OCam), U, U, P, P, P]
        L.orc_set_textures.argtypes = [P, U]
        L.orc_tex_sample.argtypes = [P, P, U, P]
        L.orc_emitters.argtypes = [P, U, P, U, U, P]
        L.orc_emitters.restype = U
        L.orc_set_nee.argtypes = [P]
        L.orc_treelet.argtypes = [P, U, P, U]
        L.orc_treelet.restype = I
        _oracle = L
    return _oracle


def ref_available(bits: int = 30) -> bool:
    return os.path.exists(REF_LIB if bits == 30 else REF64_LIB)


def ref_lib(bits: int = 30) -> ctypes.CDLL:
    if bits not in _ref:
        path = REF_LIB if bits == 30 else REF64_LIB
        if not os.path.exists(path):
            raise ImportError(f"{path} missing: run `make -C oracle ref` where the reference tree exists")
        L = ctypes.CDLL(path)
        P, U, I, F = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_float
        L.ref_build.argtypes = [P, U, P, I, P, P, P, P, P, P]
        L.ref_build.restype = I
        L.ref_set_geometry.argtypes = [P, P, P, U]
        L.ref_trace.argtypes = [P, U, P, P, P, I]
        L.ref_render.argtypes = [P, P, U, U, U, U, U, U, U, U, F, I, U, U, P, P, P, I]
        L.ref_render.restype = I
        L.ref_render_rows.argtypes = [P, P, U, U, U, P, U, U, U, U, F, I, U, U, P, P, P, I]
        L.ref_render_rows.restype = I
        _ref[bits] = L
    return _ref[bits]


_refgpu = None


def refgpu_available() -> bool:
    return os.path.exists(REFGPU_LIB)


def refgpu_lib() -> ctypes.CDLL:
    global _refgpu
    if _refgpu is None:
        if not os.path.exists(REFGPU_LIB):
            raise ImportError(f"{REFGPU_LIB} missing: run `make -C oracle ref` where the reference tree exists")
        L = ctypes.CDLL(REFGPU_LIB)
        P, U, I = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int
        L.refgpu_build.argtypes = [P, U, P, I, P, P, P, P, P, P, P, P]
        L.refgpu_build.restype = I
        L.refgpu_key_bits.restype = I
        F = ctypes.c_float
        L.refgpu_render.argtypes = [P, U, P, P, U, U, U, P, U, F, I, U, U, U, P, P, P]
        L.refgpu_render.restype = I
        _refgpu = L
    return _refgpu


def refgpu_build(tris: np.ndarray, box=None, reps: int = 5, outputs: bool = False):
    """The reference's own GPU build (CUDA::BVHBuilder::build compiled for sm_100a) on
    the current device: ({"ms_mean", "ms_min", "wall_ms_mean"}, BuildResult or None).
    The BuildResult holds the last build's reference-format arrays (keys left zero)."""
    tris = np.ascontiguousarray(tris)
    n = len(tris)
    box = enclosing_box(tris) if box is None else np.ascontiguousarray(box, np.float32)
    L = refgpu_lib()
    ms, lo, wall = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    r = BuildResult(n, int(L.refgpu_key_bits())) if outputs else None
    arrs = [r.tris, r.children, r.parents_leaf, r.parents_internal, r.node_boxes] if outputs else [None] * 5
    rc = L.refgpu_build(_p(tris), n, _p(box), int(reps), ctypes.byref(ms), ctypes.byref(lo), ctypes.byref(wall),
                        *[_p(a) for a in arrs])
    if rc != 0:
        raise RuntimeError(f"refgpu_build failed (rc {rc})")
    return {"ms_mean": ms.value, "ms_min": lo.value, "wall_ms_mean": wall.value}, r


def refgpu_render(tris: np.ndarray, infos: np.ndarray, width: int, height: int, cam15, bounces: int,
                  intensity: float = 3.0, stratified: bool = True, warmup: int = 2, frames: int = 8, seed: int = 1,
                  box=None, image: bool = False):
    """The reference's own renderer on the current GPU (Scene::upload's LBVH build, then
    raytrace_kernel launches of one sample per pixel): ({"ms_per_frame", "build_ms"},
    running-mean image (height, width, 4) or None)."""
    tris = np.ascontiguousarray(tris)
    infos = np.ascontiguousarray(infos)
    box = enclosing_box(tris) if box is None else np.ascontiguousarray(box, np.float32)
    cam15 = np.ascontiguousarray(cam15, np.float32)
    L = refgpu_lib()
    ms, bms = ctypes.c_float(), ctypes.c_float()
    img = np.zeros((height, width, 4), np.float32) if image else None
    info_count = infos.nbytes // 192  # CUDA::TriangleInfo records (TriangleInfo.h:31-75), 192 B each
    rc = L.refgpu_render(_p(tris), len(tris), _p(box), _p(infos), info_count, width, height, _p(cam15), bounces,
                         intensity, int(stratified), warmup, frames, seed, ctypes.byref(ms), ctypes.byref(bms),
                         _p(img))
    if rc != 0:
        raise RuntimeError(f"refgpu_render failed (rc {rc})")
    return {"ms_per_frame": ms.value, "build_ms": bms.value}, img


class BuildResult:
    def __init__(self, n: int, bits: int):
        self.tris = np.zeros(n, TRIANGLE_DTYPE)
        self.keys = np.zeros(n, np.uint32 if bits == 30 else np.uint64)
        self.children = np.zeros(n - 1, np.uint32)
        self.parents_leaf = np.zeros(n, np.uint32)
        self.parents_internal = np.zeros(n - 1, np.uint32)
        self.node_boxes = np.zeros(n - 1, BBOX_DTYPE)

    def arrays(self):
        return (self.tris, self.keys, self.children, self.parents_leaf, self.parents_internal, self.node_boxes)


def enclosing_box(tris: np.ndarray) -> np.ndarray:
    out = np.zeros(6, np.float32)
    oracle_lib().orc_enclosing_box(_p(tris), len(tris), _p(out))
    return out


def morton(tris: np.ndarray, box: np.ndarray, bits: int) -> np.ndarray:
    keys = np.zeros(len(tris), np.uint32 if bits == 30 else np.uint64)
    oracle_lib().orc_morton(_p(tris), len(tris), _p(np.ascontiguousarray(box, np.float32)), bits, _p(keys))
    return keys


def build(tris: np.ndarray, bits: int, box=None, use_ref: bool = False) -> BuildResult:
    tris = np.ascontiguousarray(tris)
    n = len(tris)
    box = enclosing_box(tris) if box is None else np.ascontiguousarray(box, np.float32)
    r = BuildResult(n, bits)
    fn = ref_lib(bits).ref_build if use_ref else oracle_lib().orc_build
    rc = fn(_p(tris), n, _p(box), bits, *[_p(a) for a in r.arrays()])
    if rc != 0:
        raise ValueError(f"build rejected its input (rc {rc})")
    return r


def treelet(records: np.ndarray, n: int, leaf_boxes: np.ndarray, gamma: int = 4) -> np.ndarray:
    """One round of the split tree's treelet restructuring (cpt_treelet.c) over a copy
    of the 96-B records ((n - 1) x 24 float32); leaf_boxes: (n, 6) lo xyz, hi xyz."""
    out = np.ascontiguousarray(records, np.float32).reshape(-1, 24)[: n - 1].copy()
    lb = np.ascontiguousarray(leaf_boxes, np.float32).reshape(n, 6)
    if oracle_lib().orc_treelet(_p(out), n, _p(lb), gamma) != 0:
        raise ValueError("treelet restructuring met a malformed tree")
    return out


def records_of(b: BuildResult) -> tuple[np.ndarray, np.ndarray]:
    """The LBVH as 96-B traversal records (internal child slot: its box; leaf child slot:
    v0, the leaf index, v1 - v0, v2 - v0; the Node word; right = left + 1) and the
    leaves' triangle boxes."""
    n = b.tris.size
    v0, v1, v2 = (b.tris[k].astype(np.float32) for k in ("v0", "v1", "v2"))
    leaf_boxes = np.concatenate([np.minimum(np.minimum(v0, v1), v2), np.maximum(np.maximum(v0, v1), v2)], 1)
    boxes = np.concatenate([b.node_boxes["min"], b.node_boxes["max"]], 1).astype(np.float32)
    rec = np.zeros((n - 1, 24), np.float32)
    words = b.children
    for side in (0, 1):
        idx = (words >> 2) + side
        internal = ((words >> side) & 1).astype(bool)
        slot = np.zeros((n - 1, 10), np.float32)
        slot[internal, :6] = boxes[idx[internal]]
        li = idx[~internal]
        slot[~internal, 0:3] = v0[li]
        slot[~internal, 3] = li.astype(np.uint32).view(np.float32)
        slot[~internal, 4:7] = v1[li] - v0[li]
        slot[~internal, 7:10] = v2[li] - v0[li]
        rec[:, 10 * side:10 * side + 10] = slot
    rec[:, 20] = words.view(np.float32)
    rec[:, 21] = ((words >> 2) + 1).astype(np.uint32).view(np.float32)
    return rec, leaf_boxes


def trace(b: BuildResult, rays: np.ndarray, any_hit: bool = False, use_ref: bool = False, stats: bool = False,
          threads: int = 0):
    """rays: (m, 6) float32 origin+direction. Returns (t, idx, uv[, stats(m,5)])."""
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
    m = len(rays)
    t = np.zeros(m, np.float32)
    idx = np.zeros(m, np.uint32)
    uv = np.zeros((m, 2), np.float32)
    st = np.zeros((m, 5), np.uint64) if stats else None
    if use_ref:
        if any_hit:
            raise ValueError("the reference has closest-hit traversal only")
        L = ref_lib()
        L.ref_set_geometry(_p(b.tris), _p(b.children), _p(b.node_boxes), len(b.tris))
        L.ref_trace(_p(rays), m, _p(t), _p(idx), _p(uv), threads)
    else:
        oracle_lib().orc_trace(_p(b.tris), _p(b.children), _p(b.node_boxes), len(b.tris), _p(rays), m, int(any_hit),
                               _p(t), _p(idx), _p(uv), _p(st))
    return (t, idx, uv, st) if stats else (t, idx, uv)


def ocam_from(eye, dirs, inv_view_proj=None, jitter=0, jitter_x=0.0, jitter_y=0.0) -> OCam:
    c = OCam()
    for a in range(3):
        c.eye[a] = float(eye[a])
    d = np.asarray(dirs, np.float32).reshape(4, 3)
    for i in range(4):
        for a in range(3):
            c.dirs[i][a] = float(d[i, a])
    if inv_view_proj is not None:
        m = np.asarray(inv_view_proj, np.float32).reshape(16)
        for k in range(16):
            c.inv_view_proj[k] = float(m[k])
    c.jitter = int(jitter)
    c.jitter_x = float(jitter_x)
    c.jitter_y = float(jitter_y)
    return c


class OTex(ctypes.Structure):
    _fields_ = [("rgba", ctypes.c_void_p), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32)]


class _Textures:
    """Installs a texture table (list of (H, W, 4) uint8 arrays) for one oracle call."""

    def __init__(self, images):
        self.images = [np.ascontiguousarray(im, np.uint8) for im in (images or [])]
        self.table = (OTex * max(1, len(self.images)))()
        for k, im in enumerate(self.images):
            self.table[k] = OTex(im.ctypes.data, im.shape[1], im.shape[0])

    def __enter__(self):
        oracle_lib().orc_set_textures(ctypes.addressof(self.table) if self.images else None, len(self.images))
        return self

    def __exit__(self, *exc):
        oracle_lib().orc_set_textures(None, 0)


def tex_sample(image: np.ndarray, uv: np.ndarray) -> np.ndarray:
    """tex2D<float4> of an (H, W, 4) uint8 image at (n, 2) float32 coordinates -> (n, 4)."""
    image = np.ascontiguousarray(image, np.uint8)
    uv = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
    out = np.zeros((len(uv), 4), np.float32)
    t = OTex(image.ctypes.data, image.shape[1], image.shape[0])
    oracle_lib().orc_tex_sample(ctypes.addressof(t), _p(uv), len(uv), _p(out))
    return out


def emitters(b: BuildResult, infos: np.ndarray, cap: int) -> tuple[np.ndarray, int]:
    """Emitter table (next-event estimation) of a build: (float32 array of
    4 + 12 * cap words, emitters found)."""
    table = np.zeros(4 + 12 * cap, np.float32)
    infos = np.ascontiguousarray(infos)
    found = oracle_lib().orc_emitters(_p(b.tris), len(b.tris), _p(infos), len(infos), cap, _p(table))
    return table, int(found)


def render(b: BuildResult, infos: np.ndarray, lights, width: int, height: int, spp: int, frame0: int, bounces: int,
           intensity: float, stratified: bool, seed: int, cam: OCam, rows=None, camera_index: int = 0,
           textures=None, nee_table: np.ndarray | None = None):
    """Per-sample radiance (spp, rows, width, 3) float32 and ray counts (3,).

    textures: list of (H, W, 4) uint8 images indexed by albedo_idx / normal_map_idx.
    nee_table: an emitter table (emitters()) to render with next-event estimation."""
    r0, r1 = (0, height) if rows is None else rows
    rad = np.zeros((spp, r1 - r0, width, 3), np.float32)
    counts = np.zeros(3, np.uint64)
    nl = 0 if lights is None else len(lights)
    table = None if nee_table is None else np.ascontiguousarray(nee_table, np.float32)
    with _Textures(textures):
        oracle_lib().orc_set_nee(_p(table))
        try:
            _render_call(b, infos, lights, nl, width, height, r0, r1, spp, frame0, bounces, intensity, stratified,
                         seed, cam, camera_index, rad, counts)
        finally:
            oracle_lib().orc_set_nee(None)
    return rad, counts


def _render_call(b, infos, lights, nl, width, height, r0, r1, spp, frame0, bounces, intensity, stratified, seed, cam,
                 camera_index, rad, counts):
    oracle_lib().orc_render(_p(b.tris), _p(b.children), _p(b.node_boxes), len(b.tris), _p(infos),
                            _p(lights) if nl else None, nl, width, height, r0, r1, spp, frame0, bounces, intensity,
                            int(stratified), seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF, ctypes.byref(cam),
                            camera_index, _p(rad), _p(counts))


def render_f64(b: BuildResult, infos: np.ndarray, lights, width: int, height: int, spp: int, frame0: int, bounces: int,
               intensity: float, stratified: bool, seed: int, cam: OCam, textures=None) -> np.ndarray:
    out = np.zeros((height, width, 3), np.float64)
    nl = 0 if lights is None else len(lights)
    with _Textures(textures):
        oracle_lib().orc_render_f64(_p(b.tris), _p(b.children), _p(b.node_boxes), len(b.tris), _p(infos),
                                    _p(lights) if nl else None, nl, width, height, spp, frame0, bounces, intensity,
                                    int(stratified), seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF, ctypes.byref(cam),
                                    _p(out))
    return out


def ref_render(b: BuildResult, infos: np.ndarray, lights, width: int, height: int, rows, spp: int, frame0: int,
               bounces: int, intensity: float, stratified: bool, seed: int, cam15: np.ndarray, threads: int = 0):
    """Reference-function integrator: per-pixel f32 sum over spp for rows [r0, r1); ray counts."""
    L = ref_lib()
    L.ref_set_geometry(_p(b.tris), _p(b.children), _p(b.node_boxes), len(b.tris))
    r0, r1 = rows
    out = np.zeros((r1 - r0, width, 3), np.float32)
    counts = np.zeros(3, np.uint64)
    nl = 0 if lights is None else len(lights)
    cam15 = np.ascontiguousarray(cam15, np.float32)
    L.ref_render(_p(infos), _p(lights) if nl else None, nl, width, height, r0, r1, spp, frame0, bounces, intensity,
                 int(stratified), seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF, _p(cam15), _p(out), _p(counts),
                 threads)
    return out, counts


def ref_render_rows(b: BuildResult, infos: np.ndarray, lights, width: int, height: int, rows, spp: int, frame0: int,
                    bounces: int, intensity: float, stratified: bool, seed: int, cam15: np.ndarray, threads: int = 0,
                    bits: int = 30):
    """Reference-function integrator over a list of rows: per-pixel float64 sums of
    the spp samples (sample order), shape (len(rows), width, 3); ray counts."""
    L = ref_lib(bits)
    L.ref_set_geometry(_p(b.tris), _p(b.children), _p(b.node_boxes), len(b.tris))
    rows = np.ascontiguousarray(rows, np.uint32)
    out = np.zeros((len(rows), width, 3), np.float64)
    counts = np.zeros(3, np.uint64)
    nl = 0 if lights is None else len(lights)
    cam15 = np.ascontiguousarray(cam15, np.float32)
    rc = L.ref_render_rows(_p(infos), _p(lights) if nl else None, nl, width, height, _p(rows), len(rows), spp, frame0,
                           bounces, intensity, int(stratified), seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF, _p(cam15),
                           _p(out), _p(counts), threads)
    if rc != 0:
        raise ValueError("ref_render_rows: a row index is outside the image")
    return out, counts


def render_rows(b: BuildResult, infos: np.ndarray, width: int, height: int, rows, spp: int, frame0: int, bounces: int,
                intensity: float, stratified: bool, seed: int, cam: OCam):
    """The oracle's integrator over a list of rows, float64 per-pixel sums (as
    ref_render_rows); ray counts."""
    out = np.zeros((len(rows), width, 3), np.float64)
    counts = np.zeros(3, np.uint64)
    for k, y in enumerate(rows):
        rad, cnt = render(b, infos, None, width, height, spp, frame0, bounces, intensity, stratified, seed, cam,
                          rows=(int(y), int(y) + 1))
        for x in rad:  # sample order
            out[k] += x[0].astype(np.float64)
        counts += cnt
    return out, counts


def heatmap(b: BuildResult, cam: OCam, width: int, height: int, base):
    rgba = np.zeros((height, width, 4), np.float32)
    counts = np.zeros((height, width), np.uint32)
    bc = np.asarray(base, np.float32)
    oracle_lib().orc_heatmap(_p(b.children), _p(b.node_boxes), ctypes.byref(cam), width, height, _p(bc), _p(rgba),
                             _p(counts))
    return rgba, counts


def philox(ctr, k0: int, k1: int) -> np.ndarray:
    c = np.asarray(ctr, np.uint32)
    out = np.zeros(4, np.uint32)
    oracle_lib().orc_philox(_p(c), k0, k1, _p(out))
    return out


def sincos_turns(u: np.ndarray):
    u = np.ascontiguousarray(u, np.float32)
    s = np.zeros_like(u)
    c = np.zeros_like(u)
    oracle_lib().orc_sincos_turns(_p(u), len(u), _p(s), _p(c))
    return s, c


# ---------------------------------------------------------------- accumulators (numpy float32 = IEEE per op)
def accumulate_kahan(samples: np.ndarray, init=None):
    """samples (spp, ..., 3) in sample order -> (sum, comp, count) as the device's Kahan accumulator;
    init: a (sum, comp, count) to continue from."""
    if init is None:
        init = (np.zeros(samples.shape[1:], np.float32), np.zeros(samples.shape[1:], np.float32), 0)
    s, c = np.array(init[0], np.float32), np.array(init[1], np.float32)
    for x in samples:
        y = (x - c).astype(np.float32)
        t = (s + y).astype(np.float32)
        c = ((t - s).astype(np.float32) - y).astype(np.float32)
        s = t
    return s, c, np.float32(init[2] + len(samples))


def accumulate_lerp(samples: np.ndarray, frame0: int, prev=None):
    """Reference running mean (cuda_path_tracer.cu:416-417): img = hit + t * (prev - hit), t = f / (f + 1)."""
    img = np.zeros(samples.shape[1:], np.float32) if prev is None else prev.astype(np.float32)
    for s, x in enumerate(samples):
        f = np.float32(frame0 + s)
        t = np.float32(f / np.float32(f + np.float32(1.0)))
        img = (x + (t * (img - x).astype(np.float32)).astype(np.float32)).astype(np.float32)
    return img
