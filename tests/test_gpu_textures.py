"""Albedo and normal-map textures on the GPU against the oracle's restatement of
the reference's sampler (Scene.cu:57-81) and of extractInfo / unpackNormal
(cuda_path_tracer.cu:85-138).

Hardware bilinear filtering holds its weights in fixed point (8 fraction bits);
how it rounds them is not documented, so the oracle rounds to nearest and the
tolerances below allow one step of the weight grid per axis: a sampled value
differs by at most 2/256 from the oracle's. Everything that does not depend on a
sampled value (rays, hits, counts) stays bit-exact."""
import numpy as np
import pytest
import torch

import cpt
from cpt.device import DeviceLbvh, DeviceRenderer, DeviceScene, make_params, to_device
from oracle import cpu

pytestmark = pytest.mark.gpu

W, H = 64, 48
SAMPLE_TOL = 2.0 / 256 + 1e-5   # one weight step per axis


def rgba_noise(h, w, seed):
    return np.random.default_rng(seed).integers(0, 256, (h, w, 4), dtype=np.uint8)


def normal_map(h, w, seed, tilt=0.6):
    # tangent-space normals around +z, encoded as (n + 1) / 2 in bytes
    rng = np.random.default_rng(seed)
    n = np.concatenate([rng.uniform(-tilt, tilt, (h, w, 2)), np.ones((h, w, 1))], 2)
    n /= np.linalg.norm(n, axis=2, keepdims=True)
    out = np.full((h, w, 4), 255, np.uint8)
    out[..., :3] = np.rint((n + 1.0) * 0.5 * 255.0).astype(np.uint8)
    return out


def dir_lights():
    l = np.zeros(2, cpt.DIR_LIGHT_DTYPE)
    l[0] = ((1.0, 0.9, 0.8), (0.3, -1.0, 0.2), 1.5)
    l[1] = ((0.2, 0.3, 1.0), (-0.5, -0.7, 0.4), 0.7)
    l["direction"] /= np.linalg.norm(l["direction"], axis=1, keepdims=True)
    return l.astype(cpt.DIR_LIGHT_DTYPE)


def textured_scene(albedo_tex=True, normal_tex=False, n_random=3000, seed=11):
    """Random triangles (albedo texture on every other one) in front of a wall at
    z = 1 carrying the albedo texture and, optionally, the normal map."""
    tris_r, infos_r = cpt.scene_random(n_random, seed=seed)
    rng = np.random.default_rng(seed)
    n0 = len(tris_r)
    infos_r["vertices"]["uv"] = rng.uniform(-1.5, 2.5, (n0, 3, 2)).astype(np.float32)
    if albedo_tex:
        infos_r["material"]["albedo_idx"][: n0 - 2: 2] = 0
    wall = np.zeros(2, cpt.TRIANGLE_DTYPE)
    corners = np.array([[-1.0, -0.6, 1.0], [2.0, -0.6, 1.0], [2.0, 1.6, 1.0], [-1.0, 1.6, 1.0]], np.float32)
    uvs = np.array([[0.0, 0.0], [3.0, 0.0], [3.0, 2.0], [0.0, 2.0]], np.float32)
    wi = np.zeros(2, cpt.TRIANGLE_INFO_DTYPE)
    for k, (a, b, c) in enumerate(((0, 1, 2), (0, 2, 3))):
        wall[k]["v0"], wall[k]["v1"], wall[k]["v2"] = corners[a], corners[b], corners[c]
        wall[k]["info_idx"] = n0 + k
        for j, v in enumerate((a, b, c)):
            vx = wi[k]["vertices"][j]
            vx["color"] = (0.6, 0.6, 0.6)
            vx["uv"] = uvs[v]
            vx["normal"] = (0.0, 0.0, -1.0)
            vx["tangent"] = (1.0, 0.0, 0.0)
            vx["bitangent"] = (0.0, 1.0, 0.0)
        wi[k]["material"]["albedo_idx"] = 0 if albedo_tex else cpt.INVALID_INDEX
        wi[k]["material"]["normal_map_idx"] = 1 if normal_tex else cpt.INVALID_INDEX
    infos_r["material"]["normal_map_idx"] = cpt.INVALID_INDEX
    infos_r["material"]["albedo_idx"][infos_r["material"]["albedo_idx"] != 0] = cpt.INVALID_INDEX
    tris = np.concatenate([tris_r, wall]).astype(cpt.TRIANGLE_DTYPE)
    infos = np.concatenate([infos_r, wi]).astype(cpt.TRIANGLE_INFO_DTYPE)
    cam = cpt.camera_look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.0), aspect=W / H)
    images = [rgba_noise(37, 53, seed + 1), normal_map(29, 41, seed + 2)]
    return tris, infos, cam, images


def ocam(cam):
    return cpu.ocam_from(cam.eye, cam.as_array()[3:], np.ctypeslib.as_array(cam.inv_view_proj))


def render_pair(tris, infos, cam, images, spp=4, frame0=3, bounces=0, seed=21, lights=None, table=None):
    """(gpu Kahan sum, oracle Kahan sum, gpu counts, oracle counts)."""
    lights = dir_lights() if lights is None else lights
    textures = [cpt.Texture(im) for im in images]
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris), check_root=True)
    sc = DeviceScene(infos, lights, textures=textures if table is None else table(textures))
    r = DeviceRenderer(make_params(W, H, spp, frame0, bounces, 3.0, True, seed, cpt.ACCUM_KAHAN))
    r.render(lb, sc, cam)
    torch.cuda.synchronize()
    r.check_status()
    g = r.accum.cpu().numpy().view(np.float32).reshape(2, H, W, 4)[0][..., :3]
    b = cpu.build(tris, 30)
    rad, counts = cpu.render(b, infos, lights, W, H, spp, frame0, bounces, 3.0, True, seed, ocam(cam),
                             textures=images)
    s, _, _ = cpu.accumulate_kahan(rad)
    return g, s, r.counts.cpu().numpy()[:3].astype(np.uint64), counts


def test_sampler_matches_oracle(cuda):
    im = rgba_noise(37, 53, 4)
    tex = cpt.Texture(im)
    rng = np.random.default_rng(5)
    centres = np.array([[(i + 0.5) / 53, (j + 0.5) / 37] for j in range(37) for i in range(53)], np.float32)
    uv = np.concatenate([centres, rng.uniform(-2.0, 3.0, (50_000, 2)).astype(np.float32)])
    d_uv = torch.from_numpy(uv).cuda()
    out = torch.empty((len(uv), 4), dtype=torch.float32, device="cuda")
    cpt.check(cpt.lib.cpt_texture_sample(tex.handle, d_uv.data_ptr(), len(uv), out.data_ptr(), None),
              "cpt_texture_sample")
    torch.cuda.synchronize()
    g = out.cpu().numpy()
    o = cpu.tex_sample(im, uv)
    nc = len(centres)
    np.testing.assert_allclose(g[:nc], im.reshape(-1, 4) / 255.0, atol=1e-6)
    assert np.abs(g - o).max() <= SAMPLE_TOL
    assert np.abs(g - o).mean() < 1.0 / 256


def test_albedo_texture_direct_light(cuda):
    tris, infos, cam, images = textured_scene()
    spp = 4
    g, s, gc, oc = render_pair(tris, infos, cam, images, spp=spp)
    assert np.array_equal(gc, oc)
    # per sample: (sum over lights of the running light sum, at most 3.7) x albedo error
    err = np.abs(g - s)
    assert err.max() <= spp * 3.7 * SAMPLE_TOL
    assert err.mean() <= spp * 0.01
    assert g.std() > 0.05 * spp


def test_albedo_texture_paths_keep_the_rays(cuda):
    # albedo steers no ray: every ray and count equal, radiance within the
    # product of per-bounce albedo tolerances
    tris, infos, cam, images = textured_scene()
    spp, bounces = 4, 3
    g, s, gc, oc = render_pair(tris, infos, cam, images, spp=spp, bounces=bounces)
    assert np.array_equal(gc, oc) and gc[1] > 0
    err = np.abs(g - s)
    assert err.max() <= spp * (3.7 + 3.0 * 2.2 * 6) * SAMPLE_TOL
    assert err.mean() <= spp * 0.01


def test_normal_map_direct_light(cuda):
    tris, infos, cam, images = textured_scene(normal_tex=True)
    spp = 4
    g, s, gc, oc = render_pair(tris, infos, cam, images, spp=spp)
    assert np.array_equal(gc, oc)
    err = np.abs(g - s)
    # a normal component differs by at most 2 x SAMPLE_TOL: a few degrees at most
    assert err.max() <= spp * 3.7 * 0.03
    assert err.mean() <= spp * 0.01
    # the map is in effect: without it the wall shades differently
    flat = infos.copy()
    flat["material"]["normal_map_idx"] = cpt.INVALID_INDEX
    g0, _, _, _ = render_pair(tris, flat, cam, images, spp=spp)
    assert np.abs(g - g0).mean() > 10 * err.mean()


def test_normal_map_paths_close_in_the_mean(cuda):
    # the normal steers the bounce, so paths may part; compare image means
    tris, infos, cam, images = textured_scene(normal_tex=True)
    g, s, _, _ = render_pair(tris, infos, cam, images, spp=8, bounces=2)
    assert abs(g.mean() - s.mean()) <= 0.02 * s.mean()


def test_index_past_the_table_is_absent(cuda):
    tris, infos, cam, images = textured_scene()
    plain = infos.copy()
    plain["material"]["albedo_idx"] = cpt.INVALID_INDEX
    g_plain, s_plain, _, _ = render_pair(tris, plain, cam, [])
    g_none, _, _, _ = render_pair(tris, infos, cam, [])       # indices 0 with an empty table
    assert g_plain.tobytes() == g_none.tobytes() == s_plain.tobytes()


def test_tracer_object_textures(cuda):
    tris, infos, cam, images = textured_scene(normal_tex=True)
    textures = [cpt.Texture(im) for im in images]
    t = cpt.Tracer(30)
    t.upload(tris, infos, dir_lights())
    t.upload_textures(textures)
    t.set_camera(cam)
    t.set_settings(bounces=2, intensity=3.0, stratified=True, seed=21)
    t.raytrace(W, H, 4)
    img = t.read_image(W, H)
    lb = DeviceLbvh(len(tris), 30)
    lb.build(to_device(tris), check_root=True)
    r = DeviceRenderer(make_params(W, H, 4, 0, 2, 3.0, True, 21, cpt.ACCUM_KAHAN))
    r.render(lb, DeviceScene(infos, dir_lights(), textures=textures), cam)
    ref = r.resolve().cpu().numpy()
    assert img.tobytes() == ref.tobytes()
    t.close()
