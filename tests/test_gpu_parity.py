"""GPU parity with the oracle (run with -m gpu on a B200).

Bar: bit-exact.  The device computes the reference's f64 arithmetic with the
same operation order and no FMA contraction, so RNG draws, first-hit
primitive ids, path lengths and every f64 pixel must equal the oracle's.
Small cases compare whole images; the full-size workloads compare a random
subset of pixels re-rendered by the oracle (pixels are independent: each
owns its RNG stream, render.zig:135), plus size-independent properties.
"""
import numpy as np
import pytest

import kat_scenes as K
import oracle as O
import zigtrace_b200 as zt
from zigtrace_b200 import scenes

pytestmark = pytest.mark.gpu
MODES = [pytest.param(zt.MODE_MEGAKERNEL, id="mega"), pytest.param(zt.MODE_WAVEFRONT, id="wavefront"),
         pytest.param(zt.MODE_MEGAKERNEL_REGEN, id="regen"), pytest.param(zt.MODE_WAVEFRONT_SORTED, id="wf_sorted")]

DEBUG_CASES = {
    "demo": (K.demo_scene, dict(width=48, height=32, max_depth=8)),
    "glass": (K.glass_scene, dict(width=64, height=36, max_depth=16)),
    "lamps": (K.lamp_scene, dict(width=64, height=36, max_depth=12)),
    "lit_room": (K.lit_room, dict(width=48, height=32, max_depth=6)),
    "cornell": (scenes.cornell, dict(width=128, height=128, max_depth=16)),
    "spheres": (scenes.random_spheres, dict(width=160, height=90, max_depth=50)),
    "coincident": (lambda: K.random_shapes(7, 300), dict(width=64, height=64, max_depth=8)),
}


@pytest.mark.parametrize("name", sorted(DEBUG_CASES))
def test_first_hit_ids_and_path_lengths_bit_exact(name):
    build, o = DEBUG_CASES[name]
    scene = build()
    if name == "coincident":
        scene.camera = zt.CameraConfig(look_from=(0, 0, 30), look_at=(0, 0, 0), vfov=50)
    if name == "lamps":
        scene.camera = zt.CameraConfig(look_from=(0, 2.5, 8), look_at=(0, 1.5, 0), vfov=50)
    scene.build()
    fp, pl = zt.render_debug(scene, zt.Options(o["width"], o["height"], 1, o["max_depth"]))
    ofp, opl = O.OracleScene.from_scene(scene).render_debug(o["width"], o["height"], o["max_depth"])
    assert (fp == ofp).all()
    assert (pl == opl).all()
    assert (fp >= 0).sum() > 0


def test_rng_streams_bit_exact_many_pixels():
    got = zt.rng_streams(12345, 0, 100_000, 4)
    for i in (0, 1, 2, 777, 65535, 99_999):
        assert [int(x) for x in got[i]] == [int(x) for x in O.Rng.for_stream(12345, i).next_n(4)]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("spp,light_sampling", [(4, True), (4, False)])
def test_cornell_small_bit_exact(spp, light_sampling, mode):
    scene = scenes.cornell().build()
    img = zt.render(scene, zt.Options(64, 64, spp, 16, light_sampling=light_sampling), zt.GpuConfig(mode)).pixels
    want = O.OracleScene.from_scene(scene).render(64, 64, spp, 16, light_sampling=light_sampling)
    assert img.tobytes() == want.tobytes()


@pytest.mark.parametrize("mode", MODES)
def test_cornell_full_size_bit_exact(mode):
    """The Cornell workload at its full size: 256x256, 64 spp, depth 16."""
    scene = scenes.cornell().build()
    o = scenes.CORNELL_OPTIONS
    img = zt.render(scene, o, zt.GpuConfig(mode)).pixels
    want = O.OracleScene.from_scene(scene).render(o.width, o.height, o.spp, o.max_depth)
    assert img.tobytes() == want.tobytes()


def _subset_check(scene, o: zt.Options, n_pixels: int, mode: int, seed: int = 0):
    img = zt.render(scene, o, zt.GpuConfig(mode)).pixels
    rng = np.random.default_rng(seed)
    pix = np.unique(rng.integers(0, o.width * o.height, n_pixels)).astype(np.uint64)
    want = O.OracleScene.from_scene(scene).render_pixels(o.width, o.height, o.spp, o.max_depth, pix, seed=o.seed,
                                                         light_sampling=o.light_sampling)
    assert img[pix.astype(np.int64)].tobytes() == want.tobytes()
    assert np.isfinite(img).all()
    return img


@pytest.mark.parametrize("mode", MODES)
def test_random_spheres_full_size_subset_bit_exact(mode):
    """1280x720, 16 spp, depth 50; 3000 random pixels re-rendered by the oracle."""
    scene = scenes.random_spheres().build()
    img = _subset_check(scene, scenes.SPHERES_OPTIONS, 3000, mode)
    assert img.mean() > 0.1


@pytest.mark.parametrize("mode", MODES)
def test_triangle_heavy_subset_bit_exact(mode):
    """The 1M-triangle scene at full resolution, 4 spp; 400 oracle pixels."""
    scene = scenes.triangle_heavy().build()
    o = zt.Options(1920, 1080, 4, 16)
    _subset_check(scene, o, 400, mode)


@pytest.mark.parametrize("mode", MODES)
def test_triangle_heavy_benchmark_config_subset_bit_exact(mode):
    """The benchmark configuration itself (1920x1080, 64 spp, depth 16, BVH
    built on the device); 150 oracle pixels."""
    scene = scenes.triangle_heavy().build(device=True)
    assert scene.built_on_device
    _subset_check(scene, scenes.TRIANGLE_HEAVY_OPTIONS, 150, mode, seed=3)


@pytest.mark.parametrize("mode", MODES)
def test_render_is_deterministic_and_seed_dependent(mode):
    scene = scenes.random_spheres().build()
    o = zt.Options(320, 180, 4, 50, seed=7)
    g = zt.GpuConfig(mode)
    a = zt.render(scene, o, g).pixels
    b = zt.render(scene, o, g).pixels
    assert a.tobytes() == b.tobytes()
    c = zt.render(scene, zt.Options(320, 180, 4, 50, seed=8), g).pixels
    assert a.tobytes() != c.tobytes()


@pytest.mark.parametrize("mode", MODES)
def test_render_device_on_torch_stream_matches_host_render(mode):
    import torch
    scene = scenes.cornell().build()
    o = zt.Options(96, 64, 2, 16)
    want = zt.render(scene, o).pixels
    scene.upload()
    out = torch.empty(96 * 64 * 3, dtype=torch.float64, device="cuda")
    for _ in range(2):  # the second launch reuses the cached graph
        out.fill_(-1.0)
        zt.render_device(scene, o, out.data_ptr(), torch.cuda.current_stream().cuda_stream, zt.GpuConfig(mode))
    torch.cuda.synchronize()
    assert out.cpu().numpy().reshape(-1, 3).tobytes() == want.tobytes()


def test_row_bands_reassemble_the_image():
    from zigtrace_b200 import sharding
    scene = scenes.random_spheres().build()
    o = zt.Options(200, 113, 3, 50, seed=4)
    full = zt.render(scene, o).pixels
    bands = sharding.row_bands(o.height, 3, np.linspace(1, 3, o.height))
    parts = [sharding.render_rows(scene, o, a, b) for a, b in bands]
    assert np.concatenate(parts).tobytes() == full.tobytes()
    with pytest.raises(zt.ZigtraceError):
        sharding.render_rows(scene, o, 50, 40)


def test_row_bands_of_a_closed_scene_reassemble_the_image():
    """Cornell box: AUTO and zt_render_rows take the regeneration kernel."""
    from zigtrace_b200 import sharding
    scene = scenes.cornell().build()
    o = zt.Options(96, 71, 3, 16, seed=9)
    full = zt.render(scene, o).pixels
    assert full.tobytes() == O.OracleScene.from_scene(scene).render(96, 71, 3, 16, seed=9).tobytes()
    parts = [sharding.render_rows(scene, o, a, b) for a, b in sharding.row_bands(o.height, 4)]
    assert np.concatenate(parts).tobytes() == full.tobytes()


def test_render_sharded_over_nccl_single_rank():
    import os
    import socket
    import torch
    import torch.distributed as dist
    from zigtrace_b200 import sharding
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        scene = scenes.cornell().build()
        o = zt.Options(64, 40, 2, 16)
        scene.upload()
        img = sharding.render_sharded(scene, o)  # band rendered into the gather buffer on the device
        assert img.tobytes() == zt.render(scene, o).pixels.tobytes()
        dev = sharding.render_sharded(scene, o, as_numpy=False)
        assert dev.is_cuda and dev.cpu().numpy().tobytes() == img.tobytes()
        fast = sharding.render_sharded(scene, o, gpu=zt.GpuConfig(precision=zt.PRECISION_FAST))
        assert (fast == img).all(axis=1).mean() > 0.99  # the fast walk: nearly every pixel identical
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode", [zt.MODE_MEGAKERNEL, zt.MODE_MEGAKERNEL_REGEN])
def test_device_row_bands_reassemble_the_image(mode):
    import torch
    scene = scenes.random_spheres().build()
    scene.upload()
    o = zt.Options(200, 113, 3, 50, seed=4)
    full = zt.render(scene, o).pixels
    bands = [(0, 1), (1, 40), (40, 113)]
    out = torch.full((o.width * o.height * 3,), -1.0, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    for a, b in bands:
        zt.render_rows_device(scene, o, a, b, out.data_ptr() + 8 * a * o.width * 3, st, zt.GpuConfig(mode))
    torch.cuda.synchronize()
    assert out.cpu().numpy().reshape(-1, 3).tobytes() == full.tobytes()
    with pytest.raises(zt.ZigtraceError):
        zt.render_rows_device(scene, o, 50, 40, out.data_ptr(), st)
    with pytest.raises(zt.ZigtraceError):
        zt.render_rows_device(scene, o, 0, 10, out.data_ptr(), st, zt.GpuConfig(zt.MODE_WAVEFRONT))


@pytest.mark.parametrize("mode", MODES)
def test_edge_options(mode):
    scene = K.demo_scene().build()
    g = zt.GpuConfig(mode)
    assert (zt.render(scene, zt.Options(5, 3, 2, 0), g).pixels == 0).all()  # max_depth 0: loop never runs
    one = zt.render(scene, zt.Options(1, 1, 3, 8), g).pixels
    want = O.OracleScene.from_scene(scene).render(1, 1, 3, 8)
    assert one.tobytes() == want.tobytes()
    odd = zt.render(scene, zt.Options(37, 23, 3, 8, seed=2**64 - 1), g).pixels
    want = O.OracleScene.from_scene(scene).render(37, 23, 3, 8, seed=2**64 - 1)
    assert odd.tobytes() == want.tobytes()
    with pytest.raises(zt.ZigtraceError) as ei:
        zt.render(scene, zt.Options(0, 4, 1, 1))
    assert ei.value.name == "InvalidOptions"


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("seed", range(8))
def test_fuzz_scenes_bit_exact(seed, mode):
    """Random scenes with every shape, material and light kind, lens
    sampling and both backgrounds: whole image against the oracle."""
    scene = K.fuzz_scene(seed).build()
    o = zt.Options(32, 20, 3, 12, seed=seed)
    img = zt.render(scene, o, zt.GpuConfig(mode)).pixels
    want = O.OracleScene.from_scene(scene).render(32, 20, 3, 12, seed=seed)
    assert img.tobytes() == want.tobytes()


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("seed", range(3))
def test_fuzz_scenes_without_light_sampling_bit_exact(seed, mode):
    scene = K.fuzz_scene(seed).build()
    o = zt.Options(32, 20, 3, 12, seed=seed, light_sampling=False)
    img = zt.render(scene, o, zt.GpuConfig(mode)).pixels
    want = O.OracleScene.from_scene(scene).render(32, 20, 3, 12, seed=seed, light_sampling=False)
    assert img.tobytes() == want.tobytes()


def test_wavefront_iteration_bound_returns_timeout():
    """The wavefront loop runs on the device under an iteration bound; lowered
    below what the render needs, the bound ends the loop and the call returns
    ZT_ERR_TIMEOUT instead of hanging; the next render at the default bound
    is bit-exact again."""
    from zigtrace_b200 import _native as N
    scene = scenes.cornell().build()
    o = zt.Options(64, 64, 4, 16)
    g = zt.GpuConfig(zt.MODE_WAVEFRONT)
    N.check(N.lib().zt_set_wavefront_iteration_limit(3))
    try:
        with pytest.raises(zt.ZigtraceError) as ei:
            zt.render(scene, o, g)
        assert ei.value.name == "Timeout" and "iteration bound" in str(ei.value)
    finally:
        N.check(N.lib().zt_set_wavefront_iteration_limit(0))
    want = O.OracleScene.from_scene(scene).render(64, 64, 4, 16)
    assert zt.render(scene, o, g).pixels.tobytes() == want.tobytes()
