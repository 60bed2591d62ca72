"""OBJ/MTL ingest (cpt_obj_load) with extractScene semantics, on files the test
writes; the reference's own fixture meshes are read only where its tree exists."""
import os

import numpy as np
import pytest

import cpt
from scene_files import write_box

# the reference checkout's fixture meshes, when a checkout is present (CPT_REFERENCE_ROOT)
REF_MESHES = os.path.join(os.environ.get("CPT_REFERENCE_ROOT", "/root/reference"), "assets", "meshes")


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


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def _count(path):
    import ctypes

    n = ctypes.c_uint32()
    rc = cpt.lib.cpt_obj_load(path.encode(), 1.0, None, 0.7, None, None, 0, ctypes.byref(n))
    return rc, n.value


def test_invalid_uv_and_normal_indices_are_errors(tmp_path):
    head = "v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nvn 0 0 1\n"
    assert _count(_write(tmp_path, "ok.obj", head + "f 1/1/1 2/1/1 3/-1/-1\n")) == (cpt.OK, 1)
    for face in ("f 1/0/1 2/1/1 3/1/1",      # uv index 0
                 "f 1/2/1 2/1/1 3/1/1",      # uv index past the uvs read
                 "f 1/1/-2 2/1/1 3/1/1",     # negative normal index before the first normal
                 "f 1//5 2//1 3//1",         # normal index past the normals read
                 "f 1/-2147483648/1 2/1/1 3/1/1",
                 "f 0 2 3", "f 1 2 4", "f -4 2 3"):
        assert _count(_write(tmp_path, "bad.obj", head + face + "\n"))[0] == cpt.ERR_INVALID_ARGUMENT, face


def test_long_lines_keep_every_vertex(tmp_path):
    # a 3000-gon on one line (about 14 KB): fanned into 2998 triangles, none dropped
    k = 3000
    ang = np.arange(k) * (2 * np.pi / k)
    verts = "".join(f"v {np.cos(a):.6f} {np.sin(a):.6f} 0\n" for a in ang)
    face = "f " + " ".join(str(i + 1) for i in range(k)) + "\n"
    assert len(face) > 8192
    tris, _ = cpt.load_obj(_write(tmp_path, "ngon.obj", verts + face + "v 0 0 1\nf 1 2 3001\n"))
    assert len(tris) == k - 2 + 1
    assert np.allclose(tris[-2]["v2"], (np.cos(ang[-1]), np.sin(ang[-1]), 0), atol=1e-6)
    assert np.allclose(tris[-1]["v2"], (0, 0, 1))


def test_several_material_libraries_on_one_line(tmp_path):
    _write(tmp_path, "a.mtl", "newmtl red\nKd 1 0 0\n")
    _write(tmp_path, "b.mtl", "newmtl lamp\nKd 1 1 1\nKe 5 5 5\n")
    obj = _write(tmp_path, "two.obj", "mtllib a.mtl b.mtl\nv 0 0 0\nv 1 0 0\nv 0 1 0\n"
                                      "usemtl red\nf 1 2 3\nusemtl lamp\nf 1 3 2\n")
    tris, infos = cpt.load_obj(obj)
    assert np.allclose(infos["vertices"]["color"][0], (1, 0, 0))
    assert np.allclose(infos["material"]["emission"][1], (5, 5, 5))
