"""OBJ/MTL ingest (cpt_obj_load) with extractScene semantics, on files the test
writes; the reference's own fixture meshes are read only where its tree exists."""
import os

import numpy as np
import pytest

import cpt
from scene_files import write_box

REF_MESHES = "/root/reference/assets/meshes"


def test_box_counts_materials_and_emitter(tmp_path):
    tris, infos = cpt.load_obj(write_box(str(tmp_path)))
    walls = 5 * 6 * 6 * 2
    assert len(tris) == walls + 2 + 5 * 2
    assert np.all(tris["info_idx"] == np.arange(len(tris)))
    e = infos["material"]["emission"]
    lamp = np.nonzero(e.sum(1) > 0)[0]
    assert list(lamp) == [walls, walls + 1]
    assert np.allclose(e[lamp], (17, 12, 4))
    col = infos["vertices"]["color"]
    assert np.allclose(col[0], 0.73) and np.allclose(col[3 * 72], (0.63, 0.06, 0.05))
    assert np.all(infos["material"]["albedo_idx"] == cpt.INVALID_INDEX)
    assert np.allclose(infos["material"]["specularity"][0], 10.0)


def test_fan_triangulation_and_negative_indices(tmp_path):
    tris, _ = cpt.load_obj(write_box(str(tmp_path)))
    # first floor quad: corners (-1,-1,-1), (-2/3,-1,-1), (-2/3,-1,-2/3), (-1,-1,-2/3)
    q0, q1 = tris[0], tris[1]
    assert np.allclose(q0["v0"], (-1, -1, -1)) and np.allclose(q0["v1"], (-1 + 2 / 6, -1, -1))
    assert np.allclose(q1["v0"], q0["v0"]) and np.allclose(q1["v1"], q0["v2"])


def test_normals_given_or_geometric(tmp_path):
    tris, infos = cpt.load_obj(write_box(str(tmp_path)))
    n = infos["vertices"]["normal"]
    # walls have no vn: the geometric normal of the world-space triangle, unit length
    e1 = tris["v1"] - tris["v0"]
    e2 = tris["v2"] - tris["v0"]
    g = np.cross(e1, e2)
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    assert np.allclose(n[:72, 0], g[:72], atol=1e-6)
    # block faces carry their file normals and uvs
    assert np.allclose(n[-10:-2, 0], [(0, 0, -1)] * 2 + [(1, 0, 0)] * 2 + [(0, 0, 1)] * 2 + [(-1, 0, 0)] * 2)
    assert np.allclose(n[-2:, :], (0, 1, 0))
    uv = infos["vertices"]["uv"][-10]
    assert np.allclose(uv, [(0, 0), (1, 0), (1, 1)])


def test_scale_and_translate(tmp_path):
    p = write_box(str(tmp_path))
    a, _ = cpt.load_obj(p)
    b, _ = cpt.load_obj(p, scale=5.0, translate=(1.0, 2.0, 3.0))
    assert np.allclose(b["v0"], a["v0"] * 5.0 + (1.0, 2.0, 3.0))


def test_missing_file_and_small_capacity(tmp_path):
    import ctypes

    n = ctypes.c_uint32()
    assert cpt.lib.cpt_obj_load(b"/nonexistent.obj", 1.0, None, 0.7, None, None, 0, ctypes.byref(n)) == 1
    p = write_box(str(tmp_path)).encode()
    t = np.zeros(3, cpt.TRIANGLE_DTYPE)
    assert cpt.lib.cpt_obj_load(p, 1.0, None, 0.7, t.ctypes.data, None, 3, ctypes.byref(n)) == cpt.ERR_SCRATCH_TOO_SMALL


@pytest.mark.skipif(not os.path.isdir(REF_MESHES), reason="reference assets not present")
def test_reference_fixture_meshes():
    tris, infos = cpt.load_obj(os.path.join(REF_MESHES, "bunny.obj"))
    assert len(tris) == 4968
    tris, infos = cpt.load_obj(os.path.join(REF_MESHES, "cornell-box", "CornellBox-Original.obj"), scale=5.0)
    assert len(tris) == 36
    assert (infos["material"]["emission"].sum(1) > 0).sum() == 2
