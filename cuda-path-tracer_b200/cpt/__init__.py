"""Python bindings for the B200 LBVH builder and path tracer (libcpt.so).

Thin ctypes layer over the C ABI declared in include/cpt.h. Device buffers are
passed as integer addresses (e.g. ``torch.Tensor.data_ptr()``), streams as
``cudaStream_t`` integers (``torch.cuda.current_stream().cuda_stream``). The
library is the compute path; there is no fallback: importing this module
raises if ``libcpt.so`` is missing, and every call that fails raises
:class:`CptError` with the library's status code.

The numpy record types below match the reference's layouts byte for byte
(``CUDA::Triangle`` 40 B, ``BBox`` 24 B, ``CUDA::TriangleInfo`` 192 B,
``CUDA::DirectionalLight`` 28 B).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcpt.so")

OK = 0
ERRORS = {
    1: "invalid argument",
    2: "CUDA runtime error",
    3: "scratch buffer too small",
    4: "non-finite vertex coordinate",
    5: "device-side wait timed out",
    6: "traversal stack overflow",
    7: "root box volume differs from the enclosing box",
    8: "no CUDA device",
    9: "device-side index out of range (corrupt input)",
    10: "tree taller than the traversal stack (split BVH not built)",
}
ERR_INVALID_ARGUMENT, ERR_CUDA, ERR_SCRATCH_TOO_SMALL, ERR_NONFINITE_INPUT = 1, 2, 3, 4
ERR_DEVICE_TIMEOUT, ERR_STACK_OVERFLOW, ERR_CHECK_FAILED, ERR_NO_DEVICE, ERR_BAD_INDEX = 5, 6, 7, 8, 9
BUILD_CHECK = 1
MAX_BATCH_SCENES = 64
BUILD_TEST_WITHHOLD = 2  # test of the bounded sort wait: tile 0 of the first pass never publishes


def build_lookback_limit(log2_polls: int) -> int:
    """cpt_lbvh_build flag bits: a look-back poll limit of 2^log2_polls per tile."""
    return (int(log2_polls) & 31) << 8


ACCUM_KAHAN, ACCUM_LERP, ACCUM_F64 = 0, 1, 2
INVALID_INDEX = 0xFFFFFFFF
SPLIT_TREELET = 2
WIDE_SAH = 1  # cpt_lbvh_wide flag: surface-area collapse
TRAVERSAL_STACK = 64

TRIANGLE_DTYPE = np.dtype([("v0", "<f4", 3), ("v1", "<f4", 3), ("v2", "<f4", 3), ("info_idx", "<u4")])
BBOX_DTYPE = np.dtype([("min", "<f4", 3), ("max", "<f4", 3)])
VERTEX_DTYPE = np.dtype([("color", "<f4", 3), ("uv", "<f4", 2), ("normal", "<f4", 3), ("tangent", "<f4", 3),
                         ("bitangent", "<f4", 3)])
MATERIAL_DTYPE = np.dtype([("emission", "<f4", 3), ("specularity", "<f4"), ("albedo_idx", "<u4"),
                           ("normal_map_idx", "<u4")])
TRIANGLE_INFO_DTYPE = np.dtype([("vertices", VERTEX_DTYPE, 3), ("material", MATERIAL_DTYPE)])
DIR_LIGHT_DTYPE = np.dtype([("color", "<f4", 3), ("direction", "<f4", 3), ("intensity", "<f4")])
assert TRIANGLE_DTYPE.itemsize == 40 and BBOX_DTYPE.itemsize == 24
assert TRIANGLE_INFO_DTYPE.itemsize == 192 and DIR_LIGHT_DTYPE.itemsize == 28


class CptError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: {ERRORS.get(code, 'unknown error')} (status {code})")
        self.code = code


class Bvh(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("morton_bits", ctypes.c_int32), ("tris", ctypes.c_void_p),
                ("keys", ctypes.c_void_p), ("children", ctypes.c_void_p), ("parents_leaf", ctypes.c_void_p),
                ("parents_internal", ctypes.c_void_p), ("node_boxes", ctypes.c_void_p), ("nodes", ctypes.c_void_p),
                ("status", ctypes.c_void_p), ("split_nodes", ctypes.c_void_p), ("split_capacity", ctypes.c_uint32),
                ("wide_nodes", ctypes.c_void_p), ("wide_tris", ctypes.c_void_p), ("wide_capacity", ctypes.c_uint32)]


class Scene(ctypes.Structure):
    _fields_ = [("infos", ctypes.c_void_p), ("info_count", ctypes.c_uint32), ("lights", ctypes.c_void_p),
                ("light_count", ctypes.c_uint32), ("textures", ctypes.c_void_p), ("texture_count", ctypes.c_uint32),
                ("emitters", ctypes.c_void_p)]


class Camera(ctypes.Structure):
    _fields_ = [("eye", ctypes.c_float * 3), ("dirs", (ctypes.c_float * 3) * 4), ("inv_view_proj", ctypes.c_float * 16),
                ("jitter_x", ctypes.c_float), ("jitter_y", ctypes.c_float), ("jitter", ctypes.c_uint32)]

    def as_array(self) -> np.ndarray:
        """15 floats: eye, then corner directions 00, 10, 11, 01."""
        return np.array(list(self.eye) + [self.dirs[c][a] for c in range(4) for a in range(3)], np.float32)


class View(ctypes.Structure):
    _fields_ = [("bvh", ctypes.POINTER(Bvh)), ("scene", ctypes.POINTER(Scene)), ("camera", Camera),
                ("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("accum", ctypes.c_void_p)]


MAX_VIEWS = 64


class RenderParams(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("spp", ctypes.c_uint32),
                ("frame0", ctypes.c_uint32), ("bounces", ctypes.c_uint32), ("indirect_intensity", ctypes.c_float),
                ("stratified", ctypes.c_uint32), ("seed_lo", ctypes.c_uint32), ("seed_hi", ctypes.c_uint32),
                ("accum_mode", ctypes.c_uint32), ("ref_grid", ctypes.c_uint32), ("wave_paths", ctypes.c_uint32),
                ("trace_stats", ctypes.c_uint32), ("ray_sort", ctypes.c_uint32), ("cameras", ctypes.c_uint32),
                ("frame_counter", ctypes.c_void_p), ("nee", ctypes.c_uint32), ("refill_lanes", ctypes.c_uint32),
                ("traverse_blocks_per_sm", ctypes.c_uint32), ("wave_lanes", ctypes.c_uint32)]


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libcpt.so not built ({LIB_PATH}); run `make -C cuda-path-tracer_b200` "
                          "or __graft_entry__.build()")
    return ctypes.CDLL(LIB_PATH)


lib = _load()

_P, _U32, _I32, _SZ, _F = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_size_t, ctypes.c_float


class RcParams(ctypes.Structure):
    _fields_ = [("learning_rate", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float),
                ("epsilon", ctypes.c_float), ("ema_decay", ctypes.c_float), ("train_samples", ctypes.c_uint32),
                ("train_steps", ctypes.c_uint32), ("seed", ctypes.c_uint32), ("train_interval", ctypes.c_uint32)]
_PROTOS = {
    "cpt_bvh_bytes": (_SZ, [_U32, _I32]),
    "cpt_bvh_bind": (_I32, [_P, _SZ, _U32, _I32, ctypes.POINTER(Bvh)]),
    "cpt_lbvh_scratch_bytes": (_SZ, [_U32, _I32]),
    "cpt_lbvh_build": (_I32, [_P, _U32, _P, _I32, ctypes.POINTER(Bvh), _P, _SZ, _U32, _P]),
    "cpt_lbvh_build_static": (_I32, [_P, _U32, _P, _I32, ctypes.POINTER(Bvh), _U32, _P]),
    "cpt_lbvh_batch_scratch_bytes": (_SZ, [_P, _U32, _I32]),
    "cpt_lbvh_build_batch": (_I32, [_P, _P, _U32, _P, _I32, _P, _P, _SZ, _U32, _P]),
    "cpt_status_check": (_I32, [_P, _P]),
    "cpt_trace": (_I32, [ctypes.POINTER(Bvh), _P, _U32, _I32, _P, _P, _P]),
    "cpt_accum_bytes": (_SZ, [_U32, _U32, _U32]),
    "cpt_render_scratch_bytes": (_SZ, [ctypes.POINTER(RenderParams)]),
    "cpt_render": (_I32, [ctypes.POINTER(Bvh), ctypes.POINTER(Scene), ctypes.c_void_p,
                          ctypes.POINTER(RenderParams), _P, _P, _SZ, _P, _P, _P]),
    "cpt_resolve": (_I32, [_P, _U32, _U32, _U32, _P, _P]),
    "cpt_lbvh_wide_bytes": (_SZ, [_U32, _U32, ctypes.POINTER(_SZ), ctypes.POINTER(_SZ)]),
    "cpt_lbvh_wide": (_I32, [ctypes.POINTER(Bvh), _U32, _P, _SZ, _P, _SZ, _P, _SZ, _P]),
    "cpt_lbvh_wide_batch_scratch_bytes": (_SZ, [_P, _U32]),
    "cpt_lbvh_wide_batch": (_I32, [_P, _U32, _P, _P, _P, _P, _P, _SZ, _P]),
    "cpt_emitters_bytes": (_SZ, [_U32, _U32]),
    "cpt_emitters_build": (_I32, [ctypes.POINTER(Bvh), ctypes.POINTER(Scene), _U32, _P, _SZ,
                                  ctypes.POINTER(_U32), _P]),
    "cpt_render_views_scratch_bytes": (_SZ, [_P, _U32, ctypes.POINTER(RenderParams)]),
    "cpt_render_views": (_I32, [_P, _U32, ctypes.POINTER(RenderParams), _P, _SZ, _P, _P, _P]),
    "cpt_rc_default_params": (None, [ctypes.POINTER(RcParams)]),
    "cpt_rc_param_count": (_SZ, []),
    "cpt_rc_create": (_I32, [ctypes.POINTER(_P), ctypes.POINTER(RcParams), _P]),
    "cpt_rc_destroy": (None, [_P]),
    "cpt_rc_reset": (_I32, [_P, _U32, _P]),
    "cpt_rc_get_weights": (_I32, [_P, _P, _P]),
    "cpt_rc_set_weights": (_I32, [_P, _P, _P]),
    "cpt_rc_infer": (_I32, [_P, _P, _U32, _P, _P, _P]),
    "cpt_rc_train": (_I32, [_P, _P, _U32, _P, _U32, ctypes.POINTER(_F), _P]),
    "cpt_rc_render_scratch_bytes": (_SZ, [_P, _P, _U32, ctypes.POINTER(RenderParams)]),
    "cpt_rc_render": (_I32, [_P, _P, _U32, ctypes.POINTER(RenderParams), _P, _SZ, _P, _P, _P]),
    "cpt_rc_update": (_I32, [_P, _P, _U32, ctypes.POINTER(RenderParams), _P, _SZ, _P, _P, _P]),
    "cpt_rc_sample_count": (_I32, [_P, ctypes.POINTER(_U32), _P]),
    "cpt_rc_samples": (_I32, [_P, ctypes.POINTER(_P)]),
    "cpt_tracer_create": (_I32, [ctypes.POINTER(_P), _I32]),
    "cpt_tracer_destroy": (None, [_P]),
    "cpt_tracer_upload": (_I32, [_P, _P, _U32, _P, _U32, _P, _U32, _P]),
    "cpt_tracer_upload_textures": (_I32, [_P, _P, _U32]),
    "cpt_tracer_set_split": (_I32, [_P, _F, _U32]),
    "cpt_tracer_set_nee": (_I32, [_P, _U32]),
    "cpt_tracer_set_wide": (_I32, [_P, _U32]),
    "cpt_tracer_set_primary_rays": (_I32, [_P, _P]),
    "cpt_tracer_set_eye": (_I32, [_P, _P]),
    "cpt_tracer_set_camera": (_I32, [_P, ctypes.POINTER(Camera)]),
    "cpt_tracer_set_settings": (_I32, [_P, _U32, _F, _U32, _U32, _U32, _U32]),
    "cpt_tracer_raytrace": (_I32, [_P, _U32, _U32, _U32]),
    "cpt_tracer_reset_frames": (None, [_P]),
    "cpt_tracer_frame": (_U32, [_P]),
    "cpt_tracer_read_image": (_I32, [_P, _P]),
    "cpt_tracer_resolve": (_I32, [_P, _P]),
    "cpt_tracer_get_progress": (_I32, [_P, _P, _SZ, ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    "cpt_tracer_set_progress": (_I32, [_P, _P, _SZ, _U32, _U32, _U32, _U32]),
    "cpt_tracer_ray_counts": (_I32, [_P, _P]),
    "cpt_tracer_stream": (_P, [_P]),
    "cpt_tracer_bvh": (ctypes.POINTER(Bvh), [_P]),
    "cpt_scene_random": (_U32, [_U32, _U32, _F, _F, _F, _F, _F, _F, _P, _P]),
    "cpt_scene_sphere_hairball": (_U32, [_U32, _U32, _F, _U32, _F, _U32, _F, _F, _F, _F, _P, _P]),
    "cpt_scene_bounds": (None, [_P, _U32, _P]),
    "cpt_scene_deform": (_I32, [_P, _P, _U32, _F, _F, _F, _P]),
    "cpt_texture_create": (_I32, [_P, _U32, _U32, ctypes.POINTER(ctypes.c_uint64)]),
    "cpt_texture_destroy": (None, [ctypes.c_uint64]),
    "cpt_texture_sample": (_I32, [ctypes.c_uint64, _P, _U32, _P, _P]),
    "cpt_lbvh_split_bytes": (_SZ, [_U32, _I32, _F, _U32, ctypes.POINTER(_SZ)]),
    "cpt_lbvh_split": (_I32, [ctypes.POINTER(Bvh), _F, _U32, _P, _SZ, _P, _SZ, _P]),
    "cpt_obj_load": (_I32, [ctypes.c_char_p, _F, _P, _F, _P, _P, _U32, ctypes.POINTER(_U32)]),
    "cpt_bvh_heatmap": (_I32, [ctypes.POINTER(Bvh), ctypes.POINTER(Camera), _U32, _U32, _P, _P, _P, _P]),
    "cpt_camera_look_at": (None, [_P, _P, _P, _F, _F, _F, _F, ctypes.POINTER(Camera)]),
    "cpt_profile_begin": (_I32, []),
    "cpt_profile_end": (_I32, []),
    "cpt_profile_get": (_I32, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_ulonglong)]),
    "cpt_profile_get_busy": (_I32, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]),
    "cpt_version": (ctypes.c_char_p, []),
    "cpt_launch_count": (ctypes.c_ulonglong, []),
}
for _name, (_res, _args) in _PROTOS.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args

# Every symbol the header declares (tests check the export list against include/cpt.h).
EXPORTED = tuple(_PROTOS)


def check(code: int, what: str) -> None:
    if code != OK:
        raise CptError(code, what)


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


# ---------------------------------------------------------------- host helpers
def scene_random(n_random: int, seed: int = 0, edge_min: float = 0.005, edge_max: float = 0.02, albedo: float = 0.7,
                 light_y: float = 1.25, light_size: float = 0.5, light_emission: float = 10.0):
    """Random-triangle scene (centroids in the unit cube) plus a quad emitter.
    Returns (triangles, infos) as numpy record arrays."""
    cap = n_random + 2
    tris = np.zeros(cap, TRIANGLE_DTYPE)
    infos = np.zeros(cap, TRIANGLE_INFO_DTYPE)
    n = lib.cpt_scene_random(n_random, seed, edge_min, edge_max, albedo, light_y, light_size, light_emission,
                             _ptr(tris), _ptr(infos))
    return tris[:n], infos[:n]


def scene_sphere_hairball(nu: int, nv: int, n_hair: int, seed: int = 0, amp: float = 0.1, hair_radius: float = 1.3,
                          albedo: float = 0.7, light_y: float = 2.0, light_size: float = 1.0,
                          light_emission: float = 10.0):
    """fBm-displaced lat-long sphere (2*nu*nv triangles) + n_hair thin triangles + a quad emitter."""
    cap = 2 * nu * nv + n_hair + 2
    tris = np.zeros(cap, TRIANGLE_DTYPE)
    infos = np.zeros(cap, TRIANGLE_INFO_DTYPE)
    n = lib.cpt_scene_sphere_hairball(nu, nv, amp, n_hair, hair_radius, seed, albedo, light_y, light_size,
                                      light_emission, _ptr(tris), _ptr(infos))
    return tris[:n], infos[:n]


def load_obj(path: str, scale: float = 1.0, translate=(0.0, 0.0, 0.0), default_grey: float = 0.7):
    """OBJ/MTL file -> (triangles, infos) numpy records (extractScene semantics)."""
    n = ctypes.c_uint32()
    tr = np.asarray(translate, np.float32)
    check(lib.cpt_obj_load(path.encode(), scale, _ptr(tr), default_grey, None, None, 0, ctypes.byref(n)),
          "cpt_obj_load")
    tris = np.zeros(n.value, TRIANGLE_DTYPE)
    infos = np.zeros(n.value, TRIANGLE_INFO_DTYPE)
    check(lib.cpt_obj_load(path.encode(), scale, _ptr(tr), default_grey, _ptr(tris), _ptr(infos), n.value,
                           ctypes.byref(n)), "cpt_obj_load")
    return tris, infos


def bvh_heatmap(bvh: "Bvh", cam: "Camera", width: int, height: int, base_color, rgba_dev: int, counts_dev: int = 0,
                stream: int = 0) -> None:
    bc = np.asarray(base_color, np.float32)
    check(lib.cpt_bvh_heatmap(ctypes.byref(bvh), ctypes.byref(cam), width, height, _ptr(bc), rgba_dev,
                              counts_dev or None, stream), "cpt_bvh_heatmap")


def scene_bounds(tris: np.ndarray) -> np.ndarray:
    out = np.zeros(6, np.float32)
    lib.cpt_scene_bounds(_ptr(tris), len(tris), _ptr(out))
    return out


def camera_look_at(eye, target, up=(0.0, 1.0, 0.0), fov_deg: float = 45.0, aspect: float = 1.0,
                   znear: float = 0.3, zfar: float = 30.0) -> Camera:
    cam = Camera()
    e = np.asarray(eye, np.float32)
    t = np.asarray(target, np.float32)
    u = np.asarray(up, np.float32)
    lib.cpt_camera_look_at(_ptr(e), _ptr(t), _ptr(u), fov_deg, aspect, znear, zfar, ctypes.byref(cam))
    return cam


# ---------------------------------------------------------------- device calls
def bvh_bytes(n: int, bits: int) -> int:
    return int(lib.cpt_bvh_bytes(n, bits))


def lbvh_scratch_bytes(n: int, bits: int) -> int:
    return int(lib.cpt_lbvh_scratch_bytes(n, bits))


def bvh_bind(mem: int, nbytes: int, n: int, bits: int) -> Bvh:
    b = Bvh()
    check(lib.cpt_bvh_bind(mem, nbytes, n, bits, ctypes.byref(b)), "cpt_bvh_bind")
    return b


def lbvh_build(tris_dev: int, n: int, bits: int, bvh: Bvh, scratch: int, scratch_bytes: int, box=None,
               flags: int = 0, stream: int = 0) -> None:
    box_arr = None if box is None else np.ascontiguousarray(box, np.float32)
    rc = lib.cpt_lbvh_build(tris_dev, n, None if box_arr is None else _ptr(box_arr), bits, ctypes.byref(bvh), scratch,
                            scratch_bytes, flags, stream)
    check(rc, "cpt_lbvh_build")


def status_check(status_dev: int, stream: int = 0) -> None:
    check(lib.cpt_status_check(status_dev, stream), "device status")


def trace(bvh: Bvh, rays_dev: int, n: int, any_hit: bool, hits_dev: int, stats_dev: int = 0, stream: int = 0) -> None:
    check(lib.cpt_trace(ctypes.byref(bvh), rays_dev, n, int(any_hit), hits_dev, stats_dev or None, stream),
          "cpt_trace")


def accum_bytes(width: int, height: int, mode: int) -> int:
    return int(lib.cpt_accum_bytes(width, height, mode))


def render_scratch_bytes(params: RenderParams) -> int:
    return int(lib.cpt_render_scratch_bytes(ctypes.byref(params)))


def render(bvh: Bvh, scene: Scene, cam, params: RenderParams, accum: int, scratch: int, scratch_bytes: int,
           ray_counts: int = 0, status: int = 0, stream: int = 0) -> None:
    """cam: a Camera or a ctypes array of params.cameras Cameras."""
    check(lib.cpt_render(ctypes.byref(bvh), ctypes.byref(scene), ctypes.addressof(cam), ctypes.byref(params), accum,
                         scratch, scratch_bytes, ray_counts or None, status or None, stream), "cpt_render")


def emitters_bytes(n: int, max_emitters: int) -> int:
    return int(lib.cpt_emitters_bytes(n, max_emitters))


def emitters_build(bvh: Bvh, scene: Scene, max_emitters: int, table: int, table_bytes: int, stream: int = 0,
                   sync: bool = True) -> int | None:
    """Emitter table of bvh's emissive triangles (next-event estimation). With sync,
    returns the number of emitters (raises if more than max_emitters)."""
    count = _U32(0)
    check(lib.cpt_emitters_build(ctypes.byref(bvh), ctypes.byref(scene), max_emitters, table, table_bytes,
                                 ctypes.byref(count) if sync else None, stream), "cpt_emitters_build")
    return int(count.value) if sync else None


def resolve(accum: int, width: int, height: int, mode: int, rgba: int, stream: int = 0) -> None:
    check(lib.cpt_resolve(accum, width, height, mode, rgba, stream), "cpt_resolve")


def launch_count() -> int:
    return int(lib.cpt_launch_count())


RAY_COUNTS = 72
KERNELS = ("k_bounds", "k_morton", "k_scan_offsets", "k_onesweep", "k_topology", "k_gather_refit", "k_trace",
           "k_generate", "k_extend", "k_shade", "k_wave_counts", "k_accumulate", "k_resolve", "k_ray_sort",
           "k_rc_infer", "k_rc_train", "k_rc_adam", "k_rc_collect", "k_occlude")


def profile_begin() -> None:
    check(lib.cpt_profile_begin(), "cpt_profile_begin")


def profile_end() -> dict:
    """Synchronizes the recorded events; returns {kernel: (total_ms, launches)}."""
    check(lib.cpt_profile_end(), "cpt_profile_end")
    out = {}
    for k in KERNELS:
        ms, n = ctypes.c_double(), ctypes.c_ulonglong()
        check(lib.cpt_profile_get(k.encode(), ctypes.byref(ms), ctypes.byref(n)), "cpt_profile_get")
        if n.value:
            out[k] = (ms.value, int(n.value))
    return out


def profile_busy() -> dict:
    """After profile_end: {kernel: milliseconds during which at least one of its launches ran}."""
    out = {}
    for k in KERNELS:
        ms = ctypes.c_double()
        check(lib.cpt_profile_get_busy(k.encode(), ctypes.byref(ms)), "cpt_profile_get_busy")
        if ms.value:
            out[k] = ms.value
    return out


class Texture:
    """One RGBA8 image as a texture object with the reference's sampler state
    (Scene.cu:57-81): normalized coordinates, bilinear, wrap, read as [0, 1] floats."""

    def __init__(self, rgba8: np.ndarray):
        img = np.ascontiguousarray(rgba8, np.uint8)
        if img.ndim != 3 or img.shape[2] != 4:
            raise ValueError("texture must be (height, width, 4) uint8")
        self.height, self.width = int(img.shape[0]), int(img.shape[1])
        self.texels = img
        h = ctypes.c_uint64()
        check(lib.cpt_texture_create(_ptr(img), self.width, self.height, ctypes.byref(h)), "cpt_texture_create")
        self.handle = int(h.value)

    def close(self) -> None:
        if self.handle:
            lib.cpt_texture_destroy(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def texture_handles(textures) -> np.ndarray:
    """cudaTextureObject_t table (uint64) for a list of Texture."""
    return np.array([t.handle for t in textures], np.uint64)


class Tracer:
    """Reference-facing tracer (CUDAPathTracer): host buffers in, image out."""

    def __init__(self, morton_bits: int = 63):
        h = ctypes.c_void_p()
        check(lib.cpt_tracer_create(ctypes.byref(h), morton_bits), "cpt_tracer_create")
        self._h = h

    def close(self) -> None:
        if self._h:
            lib.cpt_tracer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, tris: np.ndarray, infos: np.ndarray, lights: np.ndarray | None = None, box=None) -> None:
        tris = np.ascontiguousarray(tris)
        infos = np.ascontiguousarray(infos)
        nl = 0 if lights is None else len(lights)
        lp = None if nl == 0 else _ptr(np.ascontiguousarray(lights))
        box_arr = None if box is None else np.ascontiguousarray(box, np.float32)
        check(lib.cpt_tracer_upload(self._h, _ptr(tris), len(tris), _ptr(infos), len(infos), lp, nl,
                                    None if box_arr is None else _ptr(box_arr)), "cpt_tracer_upload")

    def set_split(self, extra_ratio: float, flags: int = 0) -> None:
        check(lib.cpt_tracer_set_split(self._h, float(extra_ratio), int(flags)), "cpt_tracer_set_split")

    def set_wide(self, on) -> None:
        """Every later upload also builds the compressed wide tree and renders through it
        (True / 1; 2: with the surface-area collapse, for a scene uploaded once)."""
        check(lib.cpt_tracer_set_wide(self._h, int(on)), "cpt_tracer_set_wide")

    def set_nee(self, on: bool) -> None:
        """Next-event estimation on / off (restarts the accumulation when it changes)."""
        check(lib.cpt_tracer_set_nee(self._h, int(bool(on))), "cpt_tracer_set_nee")

    def upload_textures(self, textures) -> None:
        table = texture_handles(textures)
        check(lib.cpt_tracer_upload_textures(self._h, _ptr(table) if len(table) else None, len(table)),
              "cpt_tracer_upload_textures")

    def set_camera(self, cam: Camera) -> None:
        check(lib.cpt_tracer_set_camera(self._h, ctypes.byref(cam)), "cpt_tracer_set_camera")

    def set_primary_rays(self, dirs) -> None:
        d = np.ascontiguousarray(dirs, np.float32).reshape(12)
        check(lib.cpt_tracer_set_primary_rays(self._h, _ptr(d)), "cpt_tracer_set_primary_rays")

    def set_eye(self, eye) -> None:
        e = np.ascontiguousarray(eye, np.float32).reshape(3)
        check(lib.cpt_tracer_set_eye(self._h, _ptr(e)), "cpt_tracer_set_eye")

    def set_settings(self, bounces: int = 1, intensity: float = 3.0, stratified: bool = True, seed: int = 0,
                     accum_mode: int = ACCUM_KAHAN) -> None:
        check(lib.cpt_tracer_set_settings(self._h, bounces, intensity, int(stratified), seed & 0xFFFFFFFF,
                                          (seed >> 32) & 0xFFFFFFFF, accum_mode), "cpt_tracer_set_settings")

    def raytrace(self, width: int, height: int, spp: int = 1) -> None:
        check(lib.cpt_tracer_raytrace(self._h, width, height, spp), "cpt_tracer_raytrace")

    def reset_frames(self) -> None:
        lib.cpt_tracer_reset_frames(self._h)

    @property
    def frame(self) -> int:
        return int(lib.cpt_tracer_frame(self._h))

    def read_image(self, width: int, height: int, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((height, width, 4), np.float32)
        check(lib.cpt_tracer_read_image(self._h, _ptr(out)), "cpt_tracer_read_image")
        return out

    def get_progress(self, width: int, height: int, accum_mode: int) -> tuple[np.ndarray, int]:
        """(accumulator bytes, next frame) of the last raytrace at width x height, whose
        accumulator mode must be accum_mode (the tracer reports its own; a mismatch raises)."""
        out = np.empty(accum_bytes(width, height, accum_mode), np.uint8)
        frame, mode = ctypes.c_uint32(), ctypes.c_uint32()
        check(lib.cpt_tracer_get_progress(self._h, _ptr(out), out.nbytes, ctypes.byref(frame), ctypes.byref(mode)),
              "cpt_tracer_get_progress")
        if mode.value != accum_mode:
            raise CptError(ERR_INVALID_ARGUMENT, f"cpt_tracer_get_progress: tracer accumulates in mode {mode.value}")
        return out, frame.value

    def set_progress(self, accum: np.ndarray, width: int, height: int, frame: int, accum_mode: int) -> None:
        a = np.ascontiguousarray(accum).reshape(-1).view(np.uint8)
        check(lib.cpt_tracer_set_progress(self._h, _ptr(a), a.nbytes, width, height, frame, accum_mode),
              "cpt_tracer_set_progress")

    def resolve(self, rgba_dev: int) -> None:
        """Writes the image into device memory (float4 per pixel) on the tracer's stream."""
        check(lib.cpt_tracer_resolve(self._h, rgba_dev), "cpt_tracer_resolve")

    def ray_counts(self) -> np.ndarray:
        out = np.zeros(3, np.uint64)
        check(lib.cpt_tracer_ray_counts(self._h, _ptr(out)), "cpt_tracer_ray_counts")
        return out

    @property
    def stream(self) -> int:
        return int(lib.cpt_tracer_stream(self._h) or 0)

    def bvh(self) -> Bvh:
        return lib.cpt_tracer_bvh(self._h).contents
