"""Next-event estimation in the oracle (CPU): the emitter table against a numpy
restatement, and the estimator's mean against the reference estimator's."""
import numpy as np

import cpt
from oracle import cpu


def _scene(n=3000, seed=3, emissive_frac=0.0):
    tris, infos = cpt.scene_random(n, seed=seed)
    if emissive_frac:
        rng = np.random.default_rng(seed)
        pick = rng.random(len(infos) - 2) < emissive_frac
        infos["material"]["emission"][: len(infos) - 2][pick] = rng.uniform(0.05, 0.5, (pick.sum(), 3))
    return tris, infos


def test_emitter_table_matches_numpy():
    tris, infos = _scene(emissive_frac=0.2)
    b = cpu.build(tris, 30)
    cap = 4096
    table, found = cpu.emitters(b, infos, cap)
    st = b.tris
    e = infos["material"]["emission"][st["info_idx"]]
    emissive = ((e[:, 0] + e[:, 1]) + e[:, 2]) > np.float32(1e-7)
    idx = np.nonzero(emissive)[0]
    assert found == len(idx) > 256
    hdr = table[:4].view(np.uint32)
    assert hdr[0] == found and hdr[2] == found and hdr[3] == 0
    rec = table[4:].reshape(-1, 12)[:found]
    assert np.array_equal(rec[:, 11].view(np.uint32), idx.astype(np.uint32))
    v0, v1, v2 = st["v0"][idx], st["v1"][idx], st["v2"][idx]
    e1, e2 = v1 - v0, v2 - v0
    assert rec[:, 4:7].tobytes() == e1.tobytes() and rec[:, 8:11].tobytes() == e2.tobytes()
    c = np.stack([e1[:, 1] * e2[:, 2] - e2[:, 1] * e1[:, 2], e1[:, 2] * e2[:, 0] - e2[:, 2] * e1[:, 0],
                  e1[:, 0] * e2[:, 1] - e2[:, 0] * e1[:, 1]], 1)
    area = np.float32(0.5) * np.sqrt((c[:, 0] * c[:, 0] + c[:, 1] * c[:, 1]) + c[:, 2] * c[:, 2])
    assert rec[:, 7].tobytes() == area.astype(np.float32).tobytes()
    # segment-wise sums, as the table defines them
    seg = 256
    totals = [np.float32(0)] * ((found + seg - 1) // seg)
    for s in range(len(totals)):
        acc = np.float32(0)
        for a in area[s * seg:(s + 1) * seg]:
            acc = np.float32(acc + a)
        totals[s] = acc
    total = np.float32(0)
    for t in totals:
        total = np.float32(total + t)
    assert table[1] == total
    cdf = rec[:, 3]
    assert np.all(np.diff(cdf) >= 0) and cdf[-1] == np.float32(1.0)


def test_emitter_table_overflow_and_empty():
    tris, infos = _scene(emissive_frac=0.2)
    b = cpu.build(tris, 30)
    table, found = cpu.emitters(b, infos, 16)
    hdr = table[:4].view(np.uint32)
    assert found > 16 and hdr[0] == 0 and hdr[2] == found and hdr[3] == 1
    infos2 = infos.copy()
    infos2["material"]["emission"] = 0
    table, found = cpu.emitters(b, infos2, 16)
    assert found == 0 and table[:4].view(np.uint32)[0] == 0


def test_nee_mean_matches_reference_estimator():
    """The same expectation: image means of the two estimators agree within the
    standard error of their difference (independent samples, 24 x 16 pixels)."""
    tris, infos = _scene(n=2000, seed=4)
    b = cpu.build(tris, 30)
    w, h = 24, 16
    cam = cpt.camera_look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.0), aspect=w / h)
    oc = cpu.ocam_from(cam.eye, cam.as_array()[3:])
    table, found = cpu.emitters(b, infos, 64)
    assert found == 2
    spp = 96
    plain, cp = cpu.render(b, infos, None, w, h, spp, 0, 3, 3.0, False, 11, oc)
    nee, cn = cpu.render(b, infos, None, w, h, spp, 0, 3, 3.0, False, 11, oc, nee_table=table)
    assert cp[2] == 0 and cn[2] > 0  # shadow rays only with next-event estimation
    mp, mn = plain.astype(np.float64).mean(0), nee.astype(np.float64).mean(0)
    vp, vn = plain.astype(np.float64).var(0) / spp, nee.astype(np.float64).var(0) / spp
    d = mn - mp
    se = np.sqrt((vp + vn).mean() / d.size)
    assert mp.mean() > 0.01
    assert abs(d.mean()) < 5 * se
    assert vn.mean() < vp.mean()
