"""The oracle (oracle/cpt_oracle.c) against the reference itself.

Two anchors: the golden fixtures in tests/golden/ (produced by the reference's
own builder and traversal, see tests/golden/make_golden.py), and — where the
reference was compiled in this checkout (oracle/_ref/) — a live comparison on
larger inputs. Bit-exact throughout: Morton keys, sorted order, topology and
boxes are integer/selection work; hit distances follow the reference's
operation order without contraction.
"""
import numpy as np
import pytest

import cpt
from conftest import GOLDEN_CASES, load_golden, quantized, rays_at
from oracle import cpu


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_build_matches_golden(name):
    g = load_golden(name)
    r = cpu.build(g["tris_in"], int(g["bits"]), box=g["box"])
    assert same_bits(r.keys, g["keys"])
    assert same_bits(r.tris, g["tris"])
    assert same_bits(r.children, g["children"])
    assert same_bits(r.parents_leaf, g["parents_leaf"])
    assert same_bits(r.parents_internal, g["parents_internal"])
    assert same_bits(r.node_boxes, g["node_boxes"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_trace_matches_golden(name):
    g = load_golden(name)
    r = cpu.build(g["tris_in"], int(g["bits"]), box=g["box"])
    t, idx, uv = cpu.trace(r, g["rays"])
    assert same_bits(t, g["t"])
    assert same_bits(idx, g["idx"])
    hit = g["idx"] != cpu.INVALID
    assert same_bits(uv[hit], g["uv"][hit])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_any_hit_equals_closest_hit_occlusion(name):
    g = load_golden(name)
    r = cpu.build(g["tris_in"], int(g["bits"]), box=g["box"])
    t, _, _ = cpu.trace(r, g["rays"], any_hit=True)
    assert np.array_equal(t < cpu.FLT_MAX, g["t"] < cpu.FLT_MAX)


def test_golden_root_box_is_enclosing_box():
    # BVHBuilder.cu:258-265: the root box equals the caller's enclosing box.
    for name in GOLDEN_CASES:
        g = load_golden(name)
        root = g["node_boxes"][0]
        assert np.array_equal(np.concatenate([root["min"], root["max"]]), g["box"])


LIVE = [(30, "random"), (63, "random"), (30, "ties"), (63, "sphere")]


@pytest.mark.parametrize("bits,kind", LIVE)
def test_oracle_build_matches_reference_live(bits, kind):
    if not cpu.ref_available(bits):
        pytest.skip("reference not compiled in this checkout (make -C oracle ref)")
    if kind == "random":
        tris = cpt.scene_random(65536, seed=11)[0]
    elif kind == "ties":
        tris = quantized(cpt.scene_random(30000, seed=12)[0], 1.0 / 64)
    else:
        tris = cpt.scene_sphere_hairball(128, 64, 4000, seed=13)[0]
    o = cpu.build(tris, bits)
    r = cpu.build(tris, bits, use_ref=True)
    for a, b in zip(o.arrays(), r.arrays()):
        assert same_bits(a, b)


@pytest.mark.parametrize("bits", [30, 63])
def test_oracle_trace_matches_reference_live(bits):
    if not cpu.ref_available(bits):
        pytest.skip("reference not compiled in this checkout (make -C oracle ref)")
    tris = cpt.scene_sphere_hairball(96, 48, 3000, seed=21)[0]
    b = cpu.build(tris, bits)
    rays = rays_at(tris, 20000, seed=3, spread=(-2.0, 2.0))
    t, idx, uv = cpu.trace(b, rays)
    tr, ir, uvr = cpu.trace(b, rays, use_ref=True)
    assert same_bits(t, tr) and same_bits(idx, ir)
    hit = ir != cpu.INVALID
    assert hit.sum() > 1000
    assert same_bits(uv[hit], uvr[hit])


def test_oracle_render_matches_reference_functions():
    """The oracle integrator against the same loop written over the reference's
    own CUDA::trace / computeL / toHemisphere / TriangleInfo code (ref_render)."""
    if not cpu.ref_available(30):
        pytest.skip("reference not compiled in this checkout (make -C oracle ref)")
    tris, infos = cpt.scene_random(4000, seed=5)
    lights = np.zeros(2, cpt.DIR_LIGHT_DTYPE)
    lights[0] = ((1.0, 0.9, 0.8), (0.3, -1.0, 0.2), 1.5)
    lights[1] = ((0.2, 0.3, 1.0), (-0.5, -0.7, 0.4), 0.7)
    lights["direction"] /= np.linalg.norm(lights["direction"], axis=1, keepdims=True)
    b = cpu.build(tris, 30)
    cam = cpt.camera_look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.0))
    w = h = 24
    for lt in (None, lights):
        rad, cnt = cpu.render(b, infos, lt, w, h, 3, 5, 3, 3.0, True, 99, cpu.ocam_from(cam.eye, cam.as_array()[3:]))
        s, rc = cpu.ref_render(b, infos, lt, w, h, (0, h), 3, 5, 3, 3.0, True, 99, cam.as_array())
        acc = rad[0].copy()
        for k in range(1, 3):
            acc = (acc + rad[k]).astype(np.float32)
        if lt is None:
            assert same_bits(acc, s)
        else:  # pow() in the specular term: libm on both sides, same inputs -> same bits here
            np.testing.assert_allclose(acc, s, rtol=1e-6, atol=1e-7)
        assert np.array_equal(cnt, rc)


def test_philox_known_answers():
    # Random123 known-answer vectors for Philox4x32-10.
    assert list(cpu.philox([0, 0, 0, 0], 0, 0)) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(cpu.philox([0xFFFFFFFF] * 4, 0xFFFFFFFF, 0xFFFFFFFF)) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6,
                                                                           0x6D5451FD]
    assert list(cpu.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], 0xA4093822, 0x299F31D0)) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_sincos_turns_accuracy():
    u = (np.arange(1 << 16, dtype=np.float64) / (1 << 16)).astype(np.float32)
    s, c = cpu.sincos_turns(u)
    ang = 2.0 * np.pi * u.astype(np.float64)
    assert np.max(np.abs(s - np.sin(ang))) < 3e-7
    assert np.max(np.abs(c - np.cos(ang))) < 3e-7


def test_morton_known_answers():
    # morton.h:84-102 / 63-67: all-ones corners of the quantization grid.
    t = np.zeros(2, cpu.TRIANGLE_DTYPE)
    t[1]["v0"] = t[1]["v1"] = t[1]["v2"] = (1.0, 1.0, 1.0)
    box = np.array([0, 0, 0, 1, 1, 1], np.float32)
    assert list(cpu.morton(t, box, 30)) == [0, 0x3FFFFFFF]
    assert list(cpu.morton(t, box, 63)) == [0, 0x7FFFFFFFFFFFFFFF]
    t[1]["v0"] = t[1]["v1"] = t[1]["v2"] = (1.0, 0.0, 0.0)
    assert cpu.morton(t, box, 63)[1] == 0x1249249249249249


def test_build_rejects_fewer_than_two():
    with pytest.raises(ValueError):
        cpu.build(np.zeros(1, cpu.TRIANGLE_DTYPE), 30, box=np.array([0, 0, 0, 1, 1, 1], np.float32))


def test_row_sample_renders_match_reference_functions():
    """The benchmark's CPU leg renders a stride of rows with float64 per-pixel sums:
    the reference-function loop (ref_render_rows) and the oracle's integrator give
    the same bits and ray counts on the same rows; rows outside the image are refused."""
    if not cpu.ref_available(30):
        pytest.skip("reference not compiled in this checkout (make -C oracle ref)")
    tris, infos = cpt.scene_random(4000, seed=6)
    b = cpu.build(tris, 30)
    w, h = 32, 24
    cam = cpt.camera_look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.0), aspect=w / h)
    rows = np.array([1, 6, 11, 16, 21], np.uint32)
    ref, rc = cpu.ref_render_rows(b, infos, None, w, h, rows, 3, 2, 3, 3.0, True, 8, cam.as_array())
    orc, oc = cpu.render_rows(b, infos, w, h, rows, 3, 2, 3, 3.0, True, 8, cpu.ocam_from(cam.eye, cam.as_array()[3:]))
    assert ref.tobytes() == orc.tobytes()
    assert np.array_equal(rc, oc) and rc[0] == len(rows) * w * 3
    assert (ref > 0).any()
    with pytest.raises(ValueError):
        cpu.ref_render_rows(b, infos, None, w, h, np.array([h], np.uint32), 1, 0, 3, 3.0, True, 8, cam.as_array())
