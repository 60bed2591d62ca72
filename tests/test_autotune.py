"""The wave autotuner's host logic (cpt/autotune.py): its samples-per-wave rule is the
renderer's (checked against the library's own scratch sizing), candidate generation
within the wave capacity and a memory budget, selection, and the result cache."""
import pytest

import cpt
from cpt import autotune
from cpt.device import make_params

W, H, SPP = 320, 200, 16
PIXELS = W * H


def scratch(wave, sort):
    return cpt.render_scratch_bytes(make_params(W, H, SPP, 0, 3, 3.0, True, 0, cpt.ACCUM_KAHAN,
                                                wave_paths=wave, ray_sort=bool(sort)))


def test_samples_per_wave_is_the_renderers_rule():
    # the library sizes a wave's scratch by its samples per pixel: waves that the rule maps
    # to the same count need the same bytes, and more samples need more
    by_count = {}
    for wave in (1, PIXELS - 1, PIXELS, PIXELS + 1, 2 * PIXELS - 1, 2 * PIXELS, 3 * PIXELS, 5 * PIXELS,
                 16 * PIXELS, 40 * PIXELS):
        by_count.setdefault(autotune.samples_per_wave(wave, PIXELS, SPP), set()).add(scratch(wave, 0))
    assert all(len(v) == 1 for v in by_count.values())
    sizes = [next(iter(by_count[k])) for k in sorted(by_count)]
    assert sizes == sorted(sizes) and len(set(sizes)) == len(sizes)
    assert sorted(by_count) == [1, 2, 3, 5, 16]


def test_candidates_cover_powers_of_two_and_spp():
    c = autotune.candidates(PIXELS, SPP)
    assert c == [(s * PIXELS, 0) for s in (1, 2, 4, 8, 16)] + [(16 * PIXELS, 1)]
    assert autotune.candidates(PIXELS, 6, try_sort=False) == [(s * PIXELS, 0) for s in (1, 2, 4, 6)]
    assert autotune.candidates(PIXELS, 1) == [(PIXELS, 0), (PIXELS, 1)]


def test_candidates_respect_budget_and_capacity():
    budget = scratch(4 * PIXELS, 0)
    c = autotune.candidates(PIXELS, SPP, scratch, budget)
    assert [w for w, s in c if s == 0] == [PIXELS, 2 * PIXELS, 4 * PIXELS]
    assert all(scratch(w, s) <= budget for w, s in c)
    big = 1 << 29  # 2^29 pixels: four samples would pass the renderer's 2^31-path wave capacity
    assert [w for w, s in autotune.candidates(big, 8, try_sort=False)] == [big, 2 * big]
    with pytest.raises(ValueError):
        autotune.candidates(PIXELS, SPP, scratch, 1024)
    with pytest.raises(ValueError):
        autotune.candidates(0, SPP)


def test_tune_keeps_the_fastest_and_the_first_of_ties():
    times = {(1, 0): 5.0, (2, 0): 3.0, (4, 0): 3.0, (4, 1): 4.0}
    seen = []

    def frame(wave, sort):
        seen.append((wave, sort))
        return times[(wave, sort)]

    r = autotune.tune(frame, list(times))
    assert (r.wave_paths, r.ray_sort, r.ms) == (2, 0, 3.0)
    assert seen == list(times) and len(r.table) == 4
    with pytest.raises(ValueError):
        autotune.tune(lambda w, s: float("nan"), [(1, 0)])
    with pytest.raises(ValueError):
        autotune.tune(frame, [])


def test_cache_round_trip(tmp_path):
    path = str(tmp_path / "tune.json")
    key = autotune.workload_key("B200", PIXELS, SPP, 5, 123456)
    cache = autotune.TuneCache(path)
    assert cache.get(key) is None
    r = autotune.tune(lambda w, s: 1.0 + s, autotune.candidates(PIXELS, 2))
    cache.put(key, r)
    again = autotune.TuneCache(path).get(key)
    assert again == r and again.wave_paths == PIXELS and again.ray_sort == 0
    assert sorted(p.name for p in tmp_path.iterdir()) == ["tune.json"]


def test_launch_shape_stage():
    base = autotune.TuneResult(4 * PIXELS, 0, 10.0)
    c = autotune.launch_candidates(base, refills=(0, 24, 24, 16), blocks=(0, 6))
    assert c == [(4 * PIXELS, 0, 0, 0, 0), (4 * PIXELS, 0, 24, 0, 0), (4 * PIXELS, 0, 16, 0, 0),
                 (4 * PIXELS, 0, 0, 6, 0), (4 * PIXELS, 0, 0, 0, 2)]
    times = {(24, 0, 0): 7.0, (16, 0, 0): 8.0, (0, 6, 0): 7.0, (0, 0, 2): 7.5}
    r = autotune.tune(lambda w, s, rl, b, n: times.get((rl, b, n), 9.0), c)
    assert (r.refill_lanes, r.blocks_per_sm, r.wave_lanes, r.ms) == (24, 0, 0, 7.0)
    assert r.table[0] == {"wave_paths": 4 * PIXELS, "ray_sort": 0, "refill_lanes": 0, "blocks_per_sm": 0,
                          "wave_lanes": 0, "ms": 9.0}
    r2 = autotune.tune(lambda w, s, rl, b, n: 5.0 if n == 2 else 9.0, c)
    assert r2.wave_lanes == 2
    with pytest.raises(ValueError):
        autotune.launch_candidates(base, refills=(40,))
    with pytest.raises(ValueError):
        autotune.launch_candidates(base, lanes=(3,))
    with pytest.raises(ValueError):
        autotune.tune(lambda *a: 1.0, [(1, 0, 0)])
    # the renderer accepts every candidate's fields (scratch sizes do not depend on them)
    p = make_params(W, H, SPP, 0, 3, 3.0, True, 0, cpt.ACCUM_KAHAN, wave_paths=4 * PIXELS, refill_lanes=24,
                    traverse_blocks_per_sm=6)
    assert cpt.render_scratch_bytes(p) == scratch(4 * PIXELS, 0)
