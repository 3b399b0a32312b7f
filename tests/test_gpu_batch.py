"""The batched form and the autotuner on the GPU: every pixel of a batched
render equals the single render of the same scene and options (bit-exact),
for every block size and order, and across graph replays."""
import numpy as np
import pytest

import kat_scenes as K
import oracle as O
import zigtrace_b200 as zt
from zigtrace_b200 import autotune, scenes

pytestmark = pytest.mark.gpu


def mixed_batch():
    items = [(scenes.cornell(), zt.Options(64, 48, 4, 16, seed=1)),
             (K.demo_scene(), zt.Options(24, 16, 8, 8)),
             (K.glass_scene(), zt.Options(40, 23, 4, 16, seed=5)),
             (K.lit_room(), zt.Options(33, 17, 8, 6, light_sampling=False))]
    items += scenes.batch_workload(count=12, spp=2, max_depth=16)
    for s, _ in items:
        s.build()
    return items


def test_render_batch_equals_single_renders():
    items = mixed_batch()
    got = zt.render_batch([s for s, _ in items], [o for _, o in items])
    for (s, o), img in zip(items, got):
        assert img.pixels.tobytes() == zt.render(s, o).pixels.tobytes()
    s, o = items[0]
    assert got[0].pixels.tobytes() == O.OracleScene.from_scene(s).render(o.width, o.height, o.spp, o.max_depth,
                                                                         seed=o.seed).tobytes()


@pytest.mark.parametrize("mode", [zt.MODE_MEGAKERNEL, zt.MODE_MEGAKERNEL_REGEN])
@pytest.mark.parametrize("block_size", [64, 128, 256])
@pytest.mark.parametrize("order", [0, 1])
def test_batch_object_all_configs_and_replay(block_size, order, mode):
    import torch
    items = mixed_batch()
    want = [zt.render(s, o).pixels for s, o in items]
    outs = [torch.full((o.width * o.height * 3,), -1.0, dtype=torch.float64, device="cuda") for _, o in items]
    b = zt.Batch([s for s, _ in items], [o for _, o in items], [t.data_ptr() for t in outs],
                 zt.GpuConfig(mode=mode, block_size=block_size), order=order)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # replay the captured graph
        for t in outs:
            t.fill_(-1.0)
        b.launch(stream)
        torch.cuda.synchronize()
        for t, w in zip(outs, want):
            assert t.cpu().numpy().reshape(-1, 3).tobytes() == w.tobytes()
    b.close()


def test_autotuned_configs_render_identical_pixels(tmp_path, monkeypatch):
    monkeypatch.setenv("ZT_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    scene = scenes.random_spheres().build()
    o = zt.Options(160, 90, 2, 50)
    want = zt.render(scene, o).pixels
    for mode, bs, cap in autotune.SINGLE_CANDIDATES:
        got = zt.render(scene, o, zt.GpuConfig(mode=mode, block_size=bs, queue_capacity=cap)).pixels
        assert got.tobytes() == want.tobytes()
    cfg, ms, cached = autotune.tune_render(scene, o, reps=1)
    assert (cfg.mode, cfg.block_size, cfg.queue_capacity) in autotune.SINGLE_CANDIDATES
    assert not cached and len(ms) == len(autotune.SINGLE_CANDIDATES)
    assert zt.render(scene, o, cfg).pixels.tobytes() == want.tobytes()
    fcfg, _, _ = autotune.tune_render(scene, o, reps=1, precision=zt.PRECISION_FAST)  # its own cache entry
    assert fcfg.precision == zt.PRECISION_FAST
    items = mixed_batch()
    bcfg, order, ms, cached = autotune.tune_batch([s for s, _ in items], [o for _, o in items], reps=1)
    assert not cached and len(ms) == len(autotune.BATCH_CANDIDATES) and order in (0, 1, autotune.PLAIN)
    got = zt.render_batch([s for s, _ in items], [o for _, o in items], bcfg)
    for (s, o), img in zip(items, got):
        assert img.pixels.tobytes() == zt.render(s, o).pixels.tobytes()
    assert autotune.tune_batch([s for s, _ in items], [o for _, o in items], reps=1)[3]  # cached now


def test_batch_rejects_bad_arguments():
    s = scenes.cornell().build()
    with pytest.raises(zt.ZigtraceError) as ei:
        zt.render_batch([s], [zt.Options(8, 8, 0, 4)])
    assert ei.value.name == "InvalidOptions"
    with pytest.raises(zt.ZigtraceError):
        zt.render_batch([s], [zt.Options(8, 8, 1, 4)], zt.GpuConfig(block_size=96))
    with pytest.raises(zt.ZigtraceError):
        zt.render_batch([s], [zt.Options(8, 8, 1, 4)], zt.GpuConfig(mode=zt.MODE_WAVEFRONT))


def test_batch_without_lights_matches_oracle():
    """A batch in which no render samples lights runs the kernel instance
    built without light sampling: sphere fields (no emitters) and lit fuzz
    scenes with light_sampling off."""
    items = scenes.batch_workload(count=6, spp=2, max_depth=16)
    items += [(K.fuzz_scene(k), zt.Options(24, 16, 3, 12, seed=k, light_sampling=False)) for k in range(3)]
    for s, _ in items:
        s.build()
    got = zt.render_batch([s for s, _ in items], [o for _, o in items])
    for (s, o), img in zip(items, got):
        if o.width * o.height > 64 * 64:
            continue
        want = O.OracleScene.from_scene(s).render(o.width, o.height, o.spp, o.max_depth, seed=o.seed,
                                                  light_sampling=o.light_sampling)
        assert img.pixels.tobytes() == want.tobytes()
    for (s, o), img in zip(items, got):
        assert img.pixels.tobytes() == zt.render(s, o).pixels.tobytes()
