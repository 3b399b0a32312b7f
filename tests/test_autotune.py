"""Autotuner choice and cache logic, with a fake timer (no GPU)."""
import json

import zigtrace_b200 as zt
from zigtrace_b200 import autotune, scenes


def test_choose_picks_fastest_and_caches(tmp_path, monkeypatch):
    monkeypatch.setenv("ZT_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    cost = {(1, 64, 0): 3.0, (1, 128, 0): 1.0, (1, 256, 0): 2.0, (2, 128, 0): 9.0}
    calls = []

    def timer(fn, reps):
        calls.append(reps)
        return fn()

    best, ms, cached = autotune.choose("k", list(cost), lambda c: cost[c], reps=3, timer=timer)
    assert best == (1, 128, 0) and not cached and calls == [3] * 4
    data = json.loads((tmp_path / "tune.json").read_text())
    assert data["k"]["best"] == [1, 128, 0] and len(data["k"]["ms"]) == 4
    best2, _, cached2 = autotune.choose("k", list(cost), lambda c: 1 / 0, timer=timer)
    assert best2 == (1, 128, 0) and cached2 and len(calls) == 4
    best3, _, cached3 = autotune.choose("k", list(cost), lambda c: cost[c], use_cache=False, timer=timer)
    assert best3 == (1, 128, 0) and not cached3


def test_candidates_cover_modes_blocks_and_queue_capacities():
    modes = {m for m, _, _ in autotune.SINGLE_CANDIDATES}
    assert modes == {zt.MODE_MEGAKERNEL, zt.MODE_MEGAKERNEL_REGEN, zt.MODE_WAVEFRONT, zt.MODE_WAVEFRONT_SORTED}
    caps = {c for m, _, c in autotune.SINGLE_CANDIDATES if m == zt.MODE_WAVEFRONT}
    assert len(caps) >= 3 and 0 in caps
    assert {b for m, b, _ in autotune.SINGLE_CANDIDATES if m == zt.MODE_MEGAKERNEL} == {64, 128, 256}
    assert (autotune.PLAIN, 0, zt.MODE_MEGAKERNEL) in autotune.BATCH_CANDIDATES
    assert {o for b, o, _ in autotune.BATCH_CANDIDATES if b != autotune.PLAIN} == {0, 1}
    assert {m for _, _, m in autotune.BATCH_CANDIDATES} == {zt.MODE_MEGAKERNEL, zt.MODE_MEGAKERNEL_REGEN}


def test_scene_class_keys(native_lib):
    s = scenes.cornell().build()
    k = autotune.scene_class(s, zt.Options(256, 256, 64, 16))
    assert k == "prims1e1|planes0|lights1|px1e5|spp64|depth16|nee1|prec0"
    assert autotune.scene_class(s, zt.Options(256, 256, 64, 16), precision=1).endswith("|prec1")
    c2 = autotune.scene_class(scenes.random_spheres().build(), scenes.SPHERES_OPTIONS)
    c3 = autotune.scene_class(scenes.triangle_heavy(nx=100, nz=50).build(), scenes.TRIANGLE_HEAVY_OPTIONS)
    assert len({k, c2, c3}) == 3 and "planes1" in c2 and "lights0" in c2
    wl = scenes.batch_workload(count=4)
    for sc, _ in wl:
        sc.build()
    bk = autotune.batch_class([s for s, _ in wl], [o for _, o in wl])
    assert bk.startswith("batch|n4|")


def test_sphere_field_has_exact_count():
    for n in (16, 17, 1000, 19999):
        s = scenes.sphere_field(n, n)
        assert s.primitive_count() == n + 1  # + ground plane
