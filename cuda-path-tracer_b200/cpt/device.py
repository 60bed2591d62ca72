"""Device-memory plumbing for the C ABI using torch tensors as allocations.

torch provides the allocator, the stream and (for several GPUs) torch.distributed;
all compute is in libcpt.so. Buffers are uint8 tensors on the current CUDA device;
their addresses go to the library.
"""
from __future__ import annotations

import numpy as np
import torch

import ctypes

from . import (ACCUM_KAHAN, BBOX_DTYPE, RcParams, BUILD_CHECK, TRIANGLE_DTYPE, Bvh, Camera, RenderParams, Scene, View, accum_bytes,
               bvh_bind, bvh_bytes, check, emitters_build, emitters_bytes, lbvh_build, lbvh_scratch_bytes, lib, render, render_scratch_bytes, resolve,
               status_check, texture_handles, trace, WIDE_SAH)


def stream_handle(stream: torch.cuda.Stream | None = None) -> int:
    s = stream or torch.cuda.current_stream()
    return int(s.cuda_stream)


def dev_bytes(nbytes: int, device=None) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device or "cuda")


def to_device(a: np.ndarray, device=None) -> torch.Tensor:
    """Copy a numpy array (any dtype) into a fresh uint8 device tensor."""
    flat = np.ascontiguousarray(a).view(np.uint8).reshape(-1)
    return torch.from_numpy(flat.copy()).to(device or "cuda")


def to_host(t: torch.Tensor, dtype, count: int | None = None, offset_bytes: int = 0) -> np.ndarray:
    raw = t.detach().cpu().numpy().view(np.uint8)
    dt = np.dtype(dtype)
    n = (raw.size - offset_bytes) // dt.itemsize if count is None else count
    return raw[offset_bytes:offset_bytes + n * dt.itemsize].view(dt).copy()


class DeviceLbvh:
    """A built LBVH in device memory: one allocation for the outputs, one for scratch."""

    def __init__(self, n: int, bits: int, device=None):
        self.n, self.bits = int(n), int(bits)
        self.mem = dev_bytes(bvh_bytes(self.n, self.bits), device)
        self.scratch_bytes = lbvh_scratch_bytes(self.n, self.bits)
        self.scratch = dev_bytes(self.scratch_bytes, device)
        self.bvh: Bvh = bvh_bind(self.mem.data_ptr(), self.mem.numel(), self.n, self.bits)

    def build(self, tris: torch.Tensor | int, box=None, check_root: bool = False, stream: int | None = None,
              flags: int = 0) -> None:
        """cpt_lbvh_build into this object's arrays; `flags` adds cpt_lbvh_build flag
        bits (the look-back limit and its test hook) to the check flag."""
        ptr = tris if isinstance(tris, int) else tris.data_ptr()
        lbvh_build(ptr, self.n, self.bits, self.bvh, self.scratch.data_ptr(), self.scratch_bytes, box=box,
                   flags=(BUILD_CHECK if check_root else 0) | int(flags),
                   stream=stream_handle() if stream is None else stream)

    def status(self, stream: int | None = None) -> None:
        status_check(self.bvh.status, stream_handle() if stream is None else stream)

    def status_words(self) -> np.ndarray:
        """The four device status words (synchronizes): status bits, trace pool,
        wide node count, wide triangle record count."""
        torch.cuda.synchronize(self.mem.device)
        off = self.bvh.status - self.mem.data_ptr()
        return self.mem[off:off + 16].cpu().numpy().view(np.uint32).copy()

    def wide(self, stream: int | None = None, keep_scratch: bool = False, sah: bool = False) -> None:
        """Builds the compressed 8-wide traversal tree (cpt_lbvh_wide) from the binary
        tree in use (the split tree when one was built); tracing and rendering then
        traverse it. Call again after every build or split. sah: the surface-area
        collapse (CPT_WIDE_SAH; a slower build, a faster traversal)."""
        leaves = self.bvh.split_capacity if self.bvh.split_nodes else self.n
        flags = WIDE_SAH if sah else 0
        nb, tb = ctypes.c_size_t(), ctypes.c_size_t()
        sb = int(lib.cpt_lbvh_wide_bytes(leaves, flags, ctypes.byref(nb), ctypes.byref(tb)))
        if not sb:
            raise ValueError("wide BVH parameters rejected")
        dev = self.mem.device
        if getattr(self, "wide_nodes", None) is None or self.wide_nodes.numel() < nb.value:
            self.wide_nodes = dev_bytes(nb.value, dev)
        if getattr(self, "wide_tris", None) is None or self.wide_tris.numel() < tb.value:
            self.wide_tris = dev_bytes(tb.value, dev)
        if getattr(self, "wide_scratch", None) is None or self.wide_scratch.numel() < sb:
            self.wide_scratch = dev_bytes(sb, dev)
        check(lib.cpt_lbvh_wide(ctypes.byref(self.bvh), flags, self.wide_nodes.data_ptr(), self.wide_nodes.numel(),
                                self.wide_tris.data_ptr(), self.wide_tris.numel(), self.wide_scratch.data_ptr(),
                                self.wide_scratch.numel(), stream_handle() if stream is None else stream),
              "cpt_lbvh_wide")
        if not keep_scratch:
            self.wide_scratch = None

    def unwide(self) -> None:
        """Back to the binary tree for tracing and rendering."""
        self.bvh.wide_nodes = None
        self.bvh.wide_tris = None
        self.bvh.wide_capacity = 0

    def split(self, extra_ratio: float = 1.0, stream: int | None = None, keep_scratch: bool = False,
              flags: int = 0) -> None:
        """Builds the split traversal BVH (cpt_lbvh_split) over the built tree; tracing
        and rendering then traverse it. Call again after every build."""
        nb = ctypes.c_size_t()
        sb = int(lib.cpt_lbvh_split_bytes(self.n, self.bits, float(extra_ratio), int(flags), ctypes.byref(nb)))
        if not sb:
            raise ValueError("split BVH parameters rejected")
        dev = self.mem.device
        if getattr(self, "split_nodes", None) is None or self.split_nodes.numel() < nb.value:
            self.split_nodes = dev_bytes(nb.value, dev)
        if getattr(self, "split_scratch", None) is None or self.split_scratch.numel() < sb:
            self.split_scratch = dev_bytes(sb, dev)
        check(lib.cpt_lbvh_split(ctypes.byref(self.bvh), float(extra_ratio), int(flags), self.split_nodes.data_ptr(),
                                 self.split_nodes.numel(), self.split_scratch.data_ptr(), self.split_scratch.numel(),
                                 stream_handle() if stream is None else stream), "cpt_lbvh_split")
        if not keep_scratch:
            torch.cuda.current_stream().synchronize()
            self.split_scratch = None

    def unsplit(self) -> None:
        """Back to traversing the LBVH itself (a wide tree built from the split tree goes too)."""
        self.bvh.split_nodes = None
        self.bvh.split_capacity = 0
        self.unwide()

    def download(self) -> dict:
        """Reference-format arrays plus the compact records, as numpy."""
        n, b = self.n, self.bvh
        base = self.mem.data_ptr()

        def get(ptr, dtype, count):
            off = ptr - base
            nbytes = np.dtype(dtype).itemsize * count
            return self.mem[off:off + nbytes].cpu().numpy().view(dtype).copy()

        return {
            "tris": get(b.tris, TRIANGLE_DTYPE, n),
            "keys": get(b.keys, np.uint32 if self.bits == 30 else np.uint64, n),
            "children": get(b.children, np.uint32, n - 1),
            "parents_leaf": get(b.parents_leaf, np.uint32, n),
            "parents_internal": get(b.parents_internal, np.uint32, n - 1),
            "node_boxes": get(b.node_boxes, BBOX_DTYPE, n - 1),
            "nodes": get(b.nodes, np.float32, 24 * (n - 1)).reshape(n - 1, 24),
        }

    def trace(self, rays: torch.Tensor, any_hit: bool = False, stats: bool = False):
        """rays: float32 device tensor (m, 8). Returns (hits (m,4) float32 tensor, stats (m,2) int32 or None)."""
        m = rays.shape[0]
        hits = torch.empty((m, 4), dtype=torch.float32, device=rays.device)
        st = torch.zeros((m, 2), dtype=torch.int32, device=rays.device) if stats else None
        trace(self.bvh, rays.data_ptr(), m, any_hit, hits.data_ptr(), st.data_ptr() if stats else 0, stream_handle())
        return hits, st


class DeviceScene:
    """Shading inputs (TriangleInfo records, directional lights, texture table) in device memory.

    textures: list of cpt.Texture indexed by the records' albedo_idx / normal_map_idx
    (the caller keeps them alive while this scene renders)."""

    def __init__(self, infos: np.ndarray, lights: np.ndarray | None = None, device=None, textures=None):
        self.infos = to_device(infos, device)
        self.n_infos = len(infos)
        self.n_lights = 0 if lights is None else len(lights)
        self.lights = to_device(lights, device) if self.n_lights else None
        self.textures = list(textures or [])
        table = texture_handles(self.textures)
        self.texture_table = to_device(table.view(np.uint8), device) if len(table) else None
        self.scene = Scene(self.infos.data_ptr(), self.n_infos, self.lights.data_ptr() if self.n_lights else None,
                           self.n_lights, self.texture_table.data_ptr() if len(table) else None, len(table))
        self.emitters = None
        self.emitter_count = None

    def build_emitters(self, lbvh: "DeviceLbvh", max_emitters: int = 1 << 16, stream: int | None = None,
                       sync: bool = True) -> int | None:
        """(Re)builds the emitter table of lbvh's triangles for next-event estimation
        and attaches it to this scene. Call again after every rebuild of lbvh."""
        nbytes = emitters_bytes(lbvh.n, max_emitters)
        if self.emitters is None or self.emitters.numel() < nbytes:
            self.emitters = dev_bytes(nbytes, self.infos.device)
        self.scene.emitters = self.emitters.data_ptr()
        self.emitter_count = emitters_build(lbvh.bvh, self.scene, max_emitters, self.emitters.data_ptr(), nbytes,
                                            stream_handle() if stream is None else stream, sync)
        return self.emitter_count


class WideBatch:
    """cpt_lbvh_wide_batch over a list of DeviceLbvh whose binary trees (LBVH or split
    tree) are built: their wide trees (largest-child collapse) in one launch sequence.
    Sized for the trees in use when created; build() again after every rebuild."""

    def __init__(self, lbvhs, device=None):
        if not lbvhs:
            raise ValueError("empty batch")
        self.lbvhs = list(lbvhs)
        k = len(self.lbvhs)
        leaves = [lb.bvh.split_capacity if lb.bvh.split_nodes else lb.n for lb in self.lbvhs]
        self.leaves = (ctypes.c_uint32 * k)(*leaves)
        for lb, nl in zip(self.lbvhs, leaves):
            nb, tb = ctypes.c_size_t(), ctypes.c_size_t()
            if not lib.cpt_lbvh_wide_bytes(nl, 0, ctypes.byref(nb), ctypes.byref(tb)):
                raise ValueError("wide BVH parameters rejected")
            dev = lb.mem.device
            if getattr(lb, "wide_nodes", None) is None or lb.wide_nodes.numel() < nb.value:
                lb.wide_nodes = dev_bytes(nb.value, dev)
            if getattr(lb, "wide_tris", None) is None or lb.wide_tris.numel() < tb.value:
                lb.wide_tris = dev_bytes(tb.value, dev)
        self.bvh_ptrs = (ctypes.c_void_p * k)(*[ctypes.addressof(lb.bvh) for lb in self.lbvhs])
        self.nodes = (ctypes.c_void_p * k)(*[lb.wide_nodes.data_ptr() for lb in self.lbvhs])
        self.node_bytes = (ctypes.c_size_t * k)(*[lb.wide_nodes.numel() for lb in self.lbvhs])
        self.tris = (ctypes.c_void_p * k)(*[lb.wide_tris.data_ptr() for lb in self.lbvhs])
        self.tri_bytes = (ctypes.c_size_t * k)(*[lb.wide_tris.numel() for lb in self.lbvhs])
        self.scratch_bytes = int(lib.cpt_lbvh_wide_batch_scratch_bytes(self.leaves, k))
        if not self.scratch_bytes:
            raise ValueError("wide batch rejected (tree count or sizes)")
        self.scratch = dev_bytes(self.scratch_bytes, device)

    def build(self, stream: int | None = None) -> None:
        rc = lib.cpt_lbvh_wide_batch(self.bvh_ptrs, len(self.lbvhs), self.nodes, self.node_bytes, self.tris,
                                     self.tri_bytes, self.scratch.data_ptr(), self.scratch_bytes,
                                     stream_handle() if stream is None else stream)
        check(rc, "cpt_lbvh_wide_batch")


class LbvhBatch:
    """cpt_lbvh_build_batch over a list of DeviceLbvh (one key width): their LBVHs
    built by one launch sequence; each output is the single build's."""

    def __init__(self, lbvhs, device=None):
        if not lbvhs:
            raise ValueError("empty batch")
        bits = {lb.bits for lb in lbvhs}
        if len(bits) != 1:
            raise ValueError("one key width per batch")
        self.lbvhs = list(lbvhs)
        self.bits = bits.pop()
        k = len(self.lbvhs)
        self.n = (ctypes.c_uint32 * k)(*[lb.n for lb in self.lbvhs])
        self.bvh_ptrs = (ctypes.c_void_p * k)(*[ctypes.addressof(lb.bvh) for lb in self.lbvhs])
        self.scratch_bytes = int(lib.cpt_lbvh_batch_scratch_bytes(self.n, k, self.bits))
        if not self.scratch_bytes:
            raise ValueError("batch rejected (scene count, sizes or key width)")
        self.scratch = dev_bytes(self.scratch_bytes, device)

    def build(self, tris, boxes, check_root: bool = False, stream: int | None = None) -> None:
        """tris: one device tensor (or pointer) per scene; boxes: (scenes, 6) host boxes."""
        k = len(self.lbvhs)
        ptrs = (ctypes.c_void_p * k)(*[t if isinstance(t, int) else t.data_ptr() for t in tris])
        bx = np.ascontiguousarray(boxes, np.float32).reshape(k, 6)
        rc = lib.cpt_lbvh_build_batch(ptrs, self.n, k, bx.ctypes.data, self.bits, self.bvh_ptrs,
                                      self.scratch.data_ptr(), self.scratch_bytes, BUILD_CHECK if check_root else 0,
                                      stream_handle() if stream is None else stream)
        check(rc, "cpt_lbvh_build_batch")


def make_params(width, height, spp, frame0=0, bounces=3, intensity=3.0, stratified=True, seed=0,
                accum_mode=ACCUM_KAHAN, ref_grid=False, wave_paths=0, trace_stats=False,
                ray_sort=False, cameras=1, nee=False, refill_lanes=0, traverse_blocks_per_sm=0,
                wave_lanes=0) -> RenderParams:
    return RenderParams(width, height, spp, frame0, bounces, intensity, int(stratified), seed & 0xFFFFFFFF,
                        (seed >> 32) & 0xFFFFFFFF, accum_mode, int(ref_grid), wave_paths, int(trace_stats),
                        int(ray_sort), cameras, None, int(nee), int(refill_lanes), int(traverse_blocks_per_sm),
                        int(wave_lanes))


class DeviceRenderer:
    """Accumulator + wave scratch for one image size / mode."""

    def __init__(self, params: RenderParams, device=None):
        self.params = params
        self.ncam = max(1, params.cameras)
        self.accum_stride = accum_bytes(params.width, params.height, params.accum_mode)
        self.accum = dev_bytes(self.accum_stride * self.ncam, device)
        self.accum.zero_()
        self.scratch_bytes = render_scratch_bytes(params)
        if not self.scratch_bytes:
            raise ValueError("render parameters rejected")
        self.scratch = dev_bytes(self.scratch_bytes, device)
        self.counts = torch.zeros(72, dtype=torch.int64, device=device or "cuda")
        self.status = torch.zeros(4, dtype=torch.int32, device=device or "cuda")
        self.image = torch.empty((params.height, params.width, 4), dtype=torch.float32, device=device or "cuda")

    def reset(self) -> None:
        self.accum.zero_()
        self.counts.zero_()
        self.status.zero_()

    def render(self, lbvh: DeviceLbvh, scene: DeviceScene, cam, spp: int | None = None,
               frame0: int | None = None, trace_stats: bool | None = None) -> None:
        """cam: one Camera, or a sequence of params.cameras Cameras."""
        p = RenderParams.from_buffer_copy(self.params)
        if spp is not None:
            p.spp = spp
        if frame0 is not None:
            p.frame0 = frame0
        if trace_stats is not None:
            p.trace_stats = int(trace_stats)
        if isinstance(cam, Camera):
            cams = (Camera * 1)(cam)
        else:
            cams = (Camera * len(cam))(*cam)
        if len(cams) != self.ncam:
            raise ValueError(f"{len(cams)} cameras given, params.cameras = {self.ncam}")
        render(lbvh.bvh, scene.scene, cams, p, self.accum.data_ptr(), self.scratch.data_ptr(), self.scratch_bytes,
               self.counts.data_ptr(), self.status.data_ptr(), stream_handle())

    def resolve(self, camera: int = 0) -> torch.Tensor:
        p = self.params
        resolve(self.accum.data_ptr() + camera * self.accum_stride, p.width, p.height, p.accum_mode,
                self.image.data_ptr(), stream_handle())
        return self.image

    def check_status(self) -> None:
        status_check(self.status.data_ptr(), stream_handle())


class BatchRenderer:
    """Several views — (BVH, shading scene, camera, resolution) — rendered in the
    same wavefront launches; one accumulator per view."""

    def __init__(self, views, params: RenderParams, device=None):
        """views: list of (DeviceLbvh, DeviceScene, Camera, width, height)."""
        self.params = params
        self._keep = views
        n = len(views)
        self.views = (View * n)()
        self.accums = []
        for i, (lb, sc, cam, w, h) in enumerate(views):
            acc = dev_bytes(accum_bytes(w, h, params.accum_mode), device)
            acc.zero_()
            self.accums.append(acc)
            self.views[i] = View(ctypes.pointer(lb.bvh), ctypes.pointer(sc.scene), cam, w, h, acc.data_ptr())
        self.scratch_bytes = int(lib.cpt_render_views_scratch_bytes(self.views, n, ctypes.byref(params)))
        if not self.scratch_bytes:
            raise ValueError("render parameters rejected")
        self.scratch = dev_bytes(self.scratch_bytes, device)
        self.counts = torch.zeros(72, dtype=torch.int64, device=device or "cuda")
        self.status = torch.zeros(4, dtype=torch.int32, device=device or "cuda")

    def render(self, frame0: int | None = None, stream: int | None = None, spp: int | None = None) -> None:
        p = RenderParams.from_buffer_copy(self.params)
        if frame0 is not None:
            p.frame0 = frame0
        if spp is not None:
            if spp > self.params.spp:
                raise ValueError("spp above the scratch's sizing")
            p.spp = spp
        check(lib.cpt_render_views(self.views, len(self.accums), ctypes.byref(p), self.scratch.data_ptr(),
                                   self.scratch_bytes, self.counts.data_ptr(), self.status.data_ptr(),
                                   stream_handle() if stream is None else stream), "cpt_render_views")

    def check_status(self) -> None:
        status_check(self.status.data_ptr(), stream_handle())


RC_LAYERS = ((96, 64), (64, 64), (64, 64), (64, 64), (64, 16))


def rc_default_params(**kw) -> RcParams:
    p = RcParams()
    lib.cpt_rc_default_params(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class RadianceCache:
    """The MLP radiance cache (cpt_rc_*): weights, Adam state and training buffers
    on the device; cached rendering of views (list of (DeviceLbvh, DeviceScene,
    Camera, width, height)) into per-view accumulators."""

    def __init__(self, params: RcParams | None = None):
        self.params = params or rc_default_params()
        h = ctypes.c_void_p()
        check(lib.cpt_rc_create(ctypes.byref(h), ctypes.byref(self.params), stream_handle()), "cpt_rc_create")
        self._h = h
        self.n_params = int(lib.cpt_rc_param_count())

    def close(self) -> None:
        if self._h:
            lib.cpt_rc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self, seed: int) -> None:
        check(lib.cpt_rc_reset(self._h, seed, stream_handle()), "cpt_rc_reset")

    def get_weights(self) -> list[np.ndarray]:
        flat = np.empty(self.n_params, np.float32)
        check(lib.cpt_rc_get_weights(self._h, flat.ctypes.data, stream_handle()), "cpt_rc_get_weights")
        out, o = [], 0
        for fi, fo in RC_LAYERS:
            out.append(flat[o:o + fi * fo].reshape(fi, fo).copy())
            o += fi * fo
        return out

    def set_weights(self, layers) -> None:
        flat = np.ascontiguousarray(np.concatenate([np.asarray(w, np.float32).reshape(-1) for w in layers]))
        assert flat.size == self.n_params
        check(lib.cpt_rc_set_weights(self._h, flat.ctypes.data, stream_handle()), "cpt_rc_set_weights")

    def infer(self, samples: torch.Tensor, box) -> torch.Tensor:
        """samples: (n, 16) float32 device tensor -> (n, 3) predictions."""
        samples = samples.contiguous()
        n = samples.shape[0]
        out = torch.empty((n, 4), dtype=torch.float32, device=samples.device)
        b = np.ascontiguousarray(box, np.float32)
        check(lib.cpt_rc_infer(self._h, samples.data_ptr(), n, b.ctypes.data, out.data_ptr(), stream_handle()),
              "cpt_rc_infer")
        return out[:, :3]

    def train(self, samples: torch.Tensor, box, steps: int = 1) -> float:
        samples = samples.contiguous()
        b = np.ascontiguousarray(box, np.float32)
        loss = ctypes.c_float()
        check(lib.cpt_rc_train(self._h, samples.data_ptr(), samples.shape[0], b.ctypes.data, steps,
                               ctypes.byref(loss), stream_handle()), "cpt_rc_train")
        return float(loss.value)

    def sample_count(self) -> int:
        n = ctypes.c_uint32()
        check(lib.cpt_rc_sample_count(self._h, ctypes.byref(n), stream_handle()), "cpt_rc_sample_count")
        return int(n.value)

    def samples(self) -> np.ndarray:
        """This frame's training samples (n, 16) as a host array."""
        n = self.sample_count()
        p = ctypes.c_void_p()
        check(lib.cpt_rc_samples(self._h, ctypes.byref(p)), "cpt_rc_samples")
        if n == 0:
            return np.empty((0, 16), np.float32)
        torch.cuda.synchronize()
        return torch.as_tensor(_DeviceArray(p.value, (n, 16), "<f4"), device="cuda").cpu().numpy()


class _DeviceArray:
    """A library-owned device buffer seen through __cuda_array_interface__."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"data": (int(ptr), False), "shape": tuple(shape), "typestr": typestr,
                                         "version": 3}


class CachedRenderer(BatchRenderer):
    """BatchRenderer whose frames go through the radiance cache (cpt_rc_render)."""

    def __init__(self, cache: RadianceCache, views, params: RenderParams, device=None):
        super().__init__(views, params, device)
        self.cache = cache
        self.rc_scratch_bytes = int(lib.cpt_rc_render_scratch_bytes(cache._h, self.views, len(self.accums),
                                                                    ctypes.byref(params)))
        if not self.rc_scratch_bytes:
            raise ValueError("render parameters rejected")
        self.rc_scratch = dev_bytes(self.rc_scratch_bytes, device)

    def render(self, frame0: int | None = None, stream: int | None = None) -> None:
        p = RenderParams.from_buffer_copy(self.params)
        if frame0 is not None:
            p.frame0 = frame0
        check(lib.cpt_rc_render(self.cache._h, self.views, len(self.accums), ctypes.byref(p),
                                self.rc_scratch.data_ptr(), self.rc_scratch_bytes, self.counts.data_ptr(),
                                self.status.data_ptr(), stream_handle() if stream is None else stream),
              "cpt_rc_render")

    def update(self, frame0: int | None = None, stream: int | None = None) -> None:
        """Training paths and optimizer steps only (no image)."""
        p = RenderParams.from_buffer_copy(self.params)
        if frame0 is not None:
            p.frame0 = frame0
        check(lib.cpt_rc_update(self.cache._h, self.views, len(self.accums), ctypes.byref(p),
                                self.rc_scratch.data_ptr(), self.rc_scratch_bytes, self.counts.data_ptr(),
                                self.status.data_ptr(), stream_handle() if stream is None else stream),
              "cpt_rc_update")
