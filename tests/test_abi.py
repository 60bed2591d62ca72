"""The C-ABI library on the CPU: it loads, exports exactly what include/cpt.h
declares, sizes its buffers sensibly, rejects bad arguments before touching the
device, and its host-side scene / camera helpers behave."""
import ctypes
import os
import re

import numpy as np
import pytest

import cpt
from conftest import ROOT
from oracle import cpu


def declared_functions():
    src = open(os.path.join(ROOT, "include", "cpt.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(cpt_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_function():
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(cpt.lib, n), n
    assert set(names) == set(cpt.EXPORTED)


def test_version_and_launch_counter():
    assert b"sm_100a" in cpt.lib.cpt_version()
    assert cpt.launch_count() >= 0


def test_layouts_match_reference():
    assert cpt.TRIANGLE_DTYPE.itemsize == cpu.oracle_lib().orc_sizeof_triangle() == 40
    assert cpt.BBOX_DTYPE.itemsize == cpu.oracle_lib().orc_sizeof_bbox() == 24
    assert cpt.TRIANGLE_INFO_DTYPE.itemsize == cpu.oracle_lib().orc_sizeof_triangle_info() == 192
    if cpu.ref_available(30):
        r = cpu.ref_lib(30)
        assert r.ref_sizeof_triangle() == 40 and r.ref_sizeof_bbox() == 24
        assert r.ref_sizeof_node() == 4 and r.ref_sizeof_triangle_info() == 192


@pytest.mark.parametrize("bits", [30, 63])
def test_buffer_sizes(bits):
    k = 4 if bits == 30 else 8
    for n in (2, 3, 1000, 1 << 20):
        outputs = n * 40 + n * k + (n - 1) * 4 + n * 4 + (n - 1) * 4 + (n - 1) * 24 + (n - 1) * 96
        assert outputs <= cpt.bvh_bytes(n, bits) <= outputs + 9 * 256
        s = cpt.lbvh_scratch_bytes(n, bits)
        assert s >= n * (k + 8)
    assert cpt.bvh_bytes(1, bits) == 0 and cpt.lbvh_scratch_bytes(1, bits) == 0
    assert cpt.bvh_bytes(100, 31) == 0


def test_bind_lays_out_disjoint_aligned_arrays():
    n = 1000
    size = cpt.bvh_bytes(n, 63)
    b = cpt.bvh_bind(1 << 20, size, n, 63)
    ptrs = [b.tris, b.keys, b.children, b.parents_leaf, b.parents_internal, b.node_boxes, b.nodes, b.status]
    assert all(p % 256 == 0 for p in ptrs)
    assert ptrs == sorted(ptrs) and ptrs[-1] < (1 << 20) + size
    with pytest.raises(cpt.CptError) as e:
        cpt.bvh_bind(1 << 20, size - 1, n, 63)
    assert e.value.code == cpt.ERR_SCRATCH_TOO_SMALL


def test_build_rejects_bad_arguments_without_device_work():
    b = cpt.bvh_bind(1 << 20, cpt.bvh_bytes(100, 30), 100, 30)
    for args in [(0, 100, 30), (256, 1, 30), (256, 100, 31)]:
        with pytest.raises(cpt.CptError) as e:
            cpt.lbvh_build(args[0], args[1], args[2], b, 1 << 30, 1 << 30)
        assert e.value.code == cpt.ERR_INVALID_ARGUMENT
    with pytest.raises(cpt.CptError) as e:  # scratch smaller than required
        cpt.lbvh_build(256, 100, 30, b, 1 << 30, 16)
    assert e.value.code == cpt.ERR_SCRATCH_TOO_SMALL
    with pytest.raises(cpt.CptError) as e:  # misaligned triangle pointer
        cpt.lbvh_build(260, 100, 30, b, 1 << 30, 1 << 30)
    assert e.value.code == cpt.ERR_INVALID_ARGUMENT
    # flag bits: unknown ones, and the look-back test hook without a short explicit
    # poll limit (none, or above 2^16 polls), are refused before any device work
    for flags in (4, 1 << 16, cpt.BUILD_TEST_WITHHOLD, cpt.BUILD_TEST_WITHHOLD | cpt.build_lookback_limit(17)):
        with pytest.raises(cpt.CptError) as e:
            cpt.lbvh_build(256, 100, 30, b, 1 << 30, 1 << 30, flags=flags)
        assert e.value.code == cpt.ERR_INVALID_ARGUMENT, flags


def test_static_build_limits_without_device_work():
    # the no-allocation build: its fixed scratch covers every accepted size for both key
    # widths; sizes above the limit, n < 2 and bad key widths are refused on the host
    # before the library looks for a device
    max_n, scratch = 131072, 8 << 20
    for bits in (30, 63):
        assert cpt.lbvh_scratch_bytes(max_n, bits) <= scratch
        assert cpt.lbvh_scratch_bytes(2, bits) <= scratch
    b = cpt.bvh_bind(1 << 20, cpt.bvh_bytes(100, 30), 100, 30)
    call = cpt.lib.cpt_lbvh_build_static
    for n in (max_n + 1, 1 << 24, 0xFFFFFFFF):
        assert call(256, n, None, 30, ctypes.byref(b), 0, None) == cpt.ERR_SCRATCH_TOO_SMALL
    for n, bits in ((0, 30), (1, 63), (100, 31), (100, 64)):
        assert call(256, n, None, bits, ctypes.byref(b), 0, None) == cpt.ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("bits", [30, 63])
def test_split_sizes_and_flags(bits):
    # split tree sizing (host-only): records for the pieces, scratch per piece, 8 B more
    # per piece with treelet restructuring; unknown flags (bit 0 once chose a clustered
    # topology, since removed) refused
    def sizes(n, ratio, flags):
        nb = ctypes.c_size_t()
        sb = cpt.lib.cpt_lbvh_split_bytes(n, bits, ctypes.c_float(ratio), flags, ctypes.byref(nb))
        return int(sb), nb.value

    n = 100_000
    for ratio in (0.0, 1.0, 8.0):
        cap = n + int(np.floor(ratio * n))
        s0, nb0 = sizes(n, ratio, 0)
        s1, nb1 = sizes(n, ratio, cpt.SPLIT_TREELET)
        assert nb0 == nb1 >= (cap - 1) * 96
        assert s0 > 0 and s1 - s0 >= 8 * cap
    assert sizes(n, 1.0, 1)[0] == 0
    assert sizes(n, 1.0, cpt.SPLIT_TREELET | 1)[0] == 0
    assert sizes(n, 1.0, 4)[0] == 0
    assert sizes(1, 1.0, 0)[0] == 0
    # ratios cpt_lbvh_split refuses get no size either (0..64, not NaN or infinite)
    assert sizes(n, 64.0, 0)[0] > 0
    for ratio in (64.5, -0.5, float("nan"), float("inf")):
        assert sizes(n, ratio, 0)[0] == 0, ratio


def test_wide_sizes_and_flags():
    # wide tree sizing (host-only): nodes for the binary tree's internal nodes, two record
    # positions per leaf, more scratch with the surface-area collapse's cost tables,
    # unknown flags refused; the batched build's scratch is the trees' own plus bounds
    def sizes(leaves, flags):
        nb, tb = ctypes.c_size_t(), ctypes.c_size_t()
        sb = cpt.lib.cpt_lbvh_wide_bytes(leaves, flags, ctypes.byref(nb), ctypes.byref(tb))
        return int(sb), nb.value, tb.value

    leaves = 100_000
    s0, nb, tb = sizes(leaves, 0)
    s1, nb1, tb1 = sizes(leaves, cpt.WIDE_SAH)
    assert s0 > 0 and nb == nb1 >= (leaves - 1) * 80 and tb == tb1 >= 2 * leaves * 48
    assert s1 - s0 >= 44 * (leaves - 1)  # parent, arrivals, choice word and 8 costs per node
    assert sizes(leaves, 2)[0] == 0 and sizes(1, 0)[0] == 0
    arr = (ctypes.c_uint32 * 3)(1000, leaves, 5)
    b3 = int(cpt.lib.cpt_lbvh_wide_batch_scratch_bytes(arr, 3))
    assert b3 >= sum(sizes(x, 0)[0] for x in (1000, leaves, 5))
    assert cpt.lib.cpt_lbvh_wide_batch_scratch_bytes(arr, 0) == 0
    assert cpt.lib.cpt_lbvh_wide_batch_scratch_bytes(None, 3) == 0
    assert cpt.lib.cpt_lbvh_wide_batch_scratch_bytes((ctypes.c_uint32 * 65)(*([100] * 65)), 65) == 0
    assert cpt.lib.cpt_lbvh_wide_batch_scratch_bytes((ctypes.c_uint32 * 2)(100, 1), 2) == 0


def test_render_sizes_and_rejections():
    from cpt import RenderParams
    p = RenderParams(64, 48, 4, 0, 3, 3.0, 1, 0, 0, cpt.ACCUM_KAHAN, 0, 0)
    s = cpt.render_scratch_bytes(p)
    assert s >= 64 * 48 * 4 * (32 * 2 + 16 + 32)
    assert cpt.accum_bytes(64, 48, cpt.ACCUM_KAHAN) == 64 * 48 * 32
    assert cpt.accum_bytes(64, 48, cpt.ACCUM_LERP) == 64 * 48 * 16
    assert cpt.accum_bytes(64, 48, cpt.ACCUM_F64) == 64 * 48 * 32
    bad = RenderParams(0, 48, 4, 0, 3, 3.0, 1, 0, 0, 0, 0, 0)
    assert cpt.render_scratch_bytes(bad) == 0
    deep = RenderParams(8, 8, 1, 0, 100, 3.0, 1, 0, 0, 0, 0, 0)
    assert cpt.render_scratch_bytes(deep) == 0


def test_every_entry_point_refuses_null_arguments():
    # null handles and buffers are refused on the host with CPT_ERR_INVALID_ARGUMENT,
    # before any device call, and never dereferenced
    L = cpt.lib
    calls = {
        "cpt_lbvh_build_static": lambda: L.cpt_lbvh_build_static(None, 10, None, 30, None, 0, None),
        "cpt_bvh_bind": lambda: L.cpt_bvh_bind(None, 0, 10, 30, None),
        "cpt_status_check": lambda: L.cpt_status_check(None, None),
        "cpt_lbvh_wide": lambda: L.cpt_lbvh_wide(None, 0, None, 0, None, 0, None, 0, None),
        "cpt_lbvh_wide_batch": lambda: L.cpt_lbvh_wide_batch(None, 1, None, None, None, None, None, 0, None),
        "cpt_emitters_build": lambda: L.cpt_emitters_build(None, None, 4, None, 0, None, None),
        "cpt_render": lambda: L.cpt_render(None, None, None, None, None, None, 0, None, None, None),
        "cpt_render_views": lambda: L.cpt_render_views(None, 0, None, None, 0, None, None, None),
        "cpt_resolve": lambda: L.cpt_resolve(None, 8, 8, 0, None, None),
        "cpt_bvh_heatmap": lambda: L.cpt_bvh_heatmap(None, None, 8, 8, None, None, None, None),
        "cpt_scene_deform": lambda: L.cpt_scene_deform(None, None, 10, 1.0, 1.0, 0.0, None),
        "cpt_texture_create": lambda: L.cpt_texture_create(None, 4, 4, None),
        "cpt_texture_sample": lambda: L.cpt_texture_sample(0, None, 4, None, None),
        "cpt_rc_create": lambda: L.cpt_rc_create(None, None, None),
        "cpt_rc_reset": lambda: L.cpt_rc_reset(None, 1, None),
        "cpt_rc_get_weights": lambda: L.cpt_rc_get_weights(None, None, None),
        "cpt_rc_set_weights": lambda: L.cpt_rc_set_weights(None, None, None),
        "cpt_rc_infer": lambda: L.cpt_rc_infer(None, None, 4, None, None, None),
        "cpt_rc_train": lambda: L.cpt_rc_train(None, None, 4, None, 1, None, None),
        "cpt_rc_render": lambda: L.cpt_rc_render(None, None, 0, None, None, 0, None, None, None),
        "cpt_rc_update": lambda: L.cpt_rc_update(None, None, 0, None, None, 0, None, None, None),
        "cpt_rc_sample_count": lambda: L.cpt_rc_sample_count(None, None, None),
        "cpt_rc_samples": lambda: L.cpt_rc_samples(None, None),
        "cpt_tracer_create": lambda: L.cpt_tracer_create(None, 30),
        "cpt_tracer_upload": lambda: L.cpt_tracer_upload(None, None, 10, None, 1, None, 0, None),
        "cpt_tracer_upload_textures": lambda: L.cpt_tracer_upload_textures(None, None, 0),
        "cpt_tracer_set_split": lambda: L.cpt_tracer_set_split(None, 1.0, 0),
        "cpt_tracer_set_wide": lambda: L.cpt_tracer_set_wide(None, 1),
        "cpt_tracer_set_nee": lambda: L.cpt_tracer_set_nee(None, 1),
        "cpt_tracer_set_primary_rays": lambda: L.cpt_tracer_set_primary_rays(None, None),
        "cpt_tracer_set_eye": lambda: L.cpt_tracer_set_eye(None, None),
        "cpt_tracer_set_camera": lambda: L.cpt_tracer_set_camera(None, None),
        "cpt_tracer_set_settings": lambda: L.cpt_tracer_set_settings(None, 1, 3.0, 1, 0, 0, 0),
        "cpt_tracer_ray_counts": lambda: L.cpt_tracer_ray_counts(None, None),
        "cpt_tracer_get_progress": lambda: L.cpt_tracer_get_progress(None, None, 0, None, None),
        "cpt_tracer_set_progress": lambda: L.cpt_tracer_set_progress(None, None, 0, 8, 8, 1, 0),
        "cpt_tracer_resolve": lambda: L.cpt_tracer_resolve(None, None),
    }
    for name, call in calls.items():
        assert call() == cpt.ERR_INVALID_ARGUMENT, name
    # calls without a status accept a null handle
    L.cpt_tracer_destroy(None)
    L.cpt_rc_destroy(None)
    L.cpt_tracer_reset_frames(None)
    assert L.cpt_tracer_frame(None) == 0 and not L.cpt_tracer_stream(None) and not L.cpt_tracer_bvh(None)


def test_tracer_calls_refuse_a_null_tracer():
    # no tracer exists without a device; the calls still refuse a null handle on the host
    assert cpt.lib.cpt_tracer_resolve(None, 256) == cpt.ERR_INVALID_ARGUMENT
    assert cpt.lib.cpt_tracer_read_image(None, 256) == cpt.ERR_INVALID_ARGUMENT
    assert cpt.lib.cpt_tracer_raytrace(None, 8, 8, 1) == cpt.ERR_INVALID_ARGUMENT


def test_scene_random_geometry():
    tris, infos = cpt.scene_random(5000, seed=1, edge_min=0.005, edge_max=0.02, light_y=1.25, light_size=0.5)
    assert len(tris) == 5002
    v = np.stack([tris["v0"], tris["v1"], tris["v2"]], 1)[:5000]
    cen = v.mean(1)
    assert cen.min() > -0.03 and cen.max() < 1.03
    # vertices are centre + e_k * u_k with e_k < 0.02: pairwise distances below 0.04
    for a, b in ((0, 1), (1, 2), (0, 2)):
        assert np.linalg.norm(v[:, a] - v[:, b], axis=1).max() < 0.0401
    assert np.all(tris["info_idx"] == np.arange(5002))
    e = infos["material"]["emission"]
    assert np.all(e[:5000] == 0) and np.all(e[5000:] == 10)
    assert np.allclose(tris[5000:]["v0"][:, 1], 1.25)
    again = cpt.scene_random(5000, seed=1)[0]
    assert again.tobytes() == tris.tobytes()
    assert cpt.scene_random(5000, seed=2)[0].tobytes() != tris.tobytes()


def test_scene_sphere_hairball_geometry():
    tris, infos = cpt.scene_sphere_hairball(64, 32, 2000, seed=3)
    assert len(tris) == 2 * 64 * 32 + 2000 + 2
    sph = np.stack([tris["v0"], tris["v1"], tris["v2"]], 1)[: 2 * 64 * 32]
    r = np.linalg.norm(sph, axis=2)
    assert r.min() > 0.85 and r.max() < 1.15
    hair = np.stack([tris["v0"], tris["v1"], tris["v2"]], 1)[2 * 64 * 32: -2]
    length = np.linalg.norm(hair[:, 1] - hair[:, 0], axis=1)
    assert length.min() >= 0.0499 and length.max() <= 0.2001
    assert np.linalg.norm(hair.mean(1), axis=1).max() < 1.3 + 0.11


def test_scene_bounds_equals_oracle():
    tris, _ = cpt.scene_random(3000, seed=9)
    assert np.array_equal(cpt.scene_bounds(tris), cpu.enclosing_box(tris))


def test_camera_corners_match_oracle_unjittered():
    cam = cpt.camera_look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.0), fov_deg=45.0, aspect=1.0)
    d = cam.as_array()[3:].reshape(4, 3)
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-6)
    # right-handed look-at along +z: screen right is world -x; 00 is bottom-left, 11 top-right
    assert d[0][1] < 0 and d[1][1] < 0 and d[2][1] > 0 and d[3][1] > 0
    assert d[0][0] > 0 and d[1][0] < 0 and np.isclose(d[0][0], -d[1][0], atol=1e-6)
    t = np.tan(np.radians(22.5))
    assert np.allclose(d[:, 2], 1.0 / np.sqrt(1.0 + 2.0 * t * t), atol=1e-6)
    # the unjittered per-sample derivation from inv_view_proj reproduces the corners
    o = cpu.ocam_from(cam.eye, d, np.ctypeslib.as_array(cam.inv_view_proj), jitter=1, jitter_x=0.0, jitter_y=0.0)
    out = np.zeros((4, 3), np.float32)
    cpu.oracle_lib().orc_corner_dirs(ctypes.byref(o), 0, 0, 0, out.ctypes.data)
    assert np.allclose(out, d, atol=2e-6)


def test_cpp_header_compiles():
    """include/cpt.hpp (the C++ mirror classes) compiles as C++17 against cpt.h."""
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(root, "include"),
                        "-I", "/usr/local/cuda/include", os.path.join(root, "tests", "cpp", "cpp_api_test.cpp")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
