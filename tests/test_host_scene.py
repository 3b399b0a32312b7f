"""Host-side parity of the product library (no GPU needed): the uploaded BVH,
emitter table and encode path must equal the oracle's restatement of the
reference node for node and byte for byte."""
import numpy as np
import pytest

import kat_scenes as K
import oracle as O
import zigtrace_b200 as zt
from zigtrace_b200 import Material, scenes, sphere


def assert_same_build(scene: zt.Scene):
    scene.build()
    os_ = O.OracleScene.from_scene(scene)
    n1, i1 = scene.bvh()
    n2, i2 = os_.bvh()
    assert n1.tobytes() == n2.tobytes()
    assert (i1 == i2).all()
    l1, c1, t1 = scene.lights()
    l2, c2, t2 = os_.lights()
    assert l1.tobytes() == l2.tobytes() and c1.tobytes() == c2.tobytes() and t1 == t2
    assert scene.bvh_depth() == os_.bvh_depth()


@pytest.mark.parametrize("n", [1, 2, 3, 7, 50, 400, 2000])
def test_bvh_and_lights_match_oracle_random(native_lib, n):
    assert_same_build(K.random_shapes(n, n))


@pytest.mark.parametrize("builder", [K.demo_scene, K.lit_room, K.lamp_scene, K.glass_scene, K.empty_scene,
                                     scenes.cornell, scenes.random_spheres])
def test_bvh_and_lights_match_oracle_scenes(native_lib, builder):
    assert_same_build(builder())


def test_bvh_matches_oracle_coincident_and_degenerate(native_lib):
    # coincident centroids -> median split (bvh.zig:197-209), and zero-area
    # boxes (radius-0 spheres on a line) -> findSplit returns null
    s = zt.Scene()
    m = s.add_material(Material.lambertian((1, 1, 1)))
    for i in range(40):
        s.add(sphere((0, 0, 0), 1 + i * 0.01, m))
    for i in range(37):
        s.add(sphere((float(i % 7), 0, 0), 0.0, m))
    assert_same_build(s)


def test_bvh_matches_oracle_triangle_heavy_slice(native_lib):
    assert_same_build(scenes.triangle_heavy(nx=120, nz=60, n_ico=3, ico_subdiv=2, n_lights=8))


def test_build_rejects_undefined_material(native_lib):
    s = zt.Scene()
    s.add(sphere((0, 0, 0), 1, 3))
    with pytest.raises(zt.ZigtraceError) as ei:
        s.build()
    assert ei.value.name == "InvalidArgument"


def test_render_before_build_is_an_error(native_lib):
    with pytest.raises(zt.ZigtraceError) as ei:
        zt.render(zt.Scene(), zt.Options(4, 4, 1, 1))
    assert ei.value.name == "NotBuilt"


def test_to_rgb8_matches_oracle_encode(native_lib):
    rng = np.random.default_rng(0)
    px = np.concatenate([rng.uniform(-1, 4, (200, 3)), [[np.nan, 0.5, 1e9]]])
    img = zt.Image(len(px), 1, px)
    for tm, k in (("none", 0), ("reinhard", 1), ("aces", 2)):
        for gamma, exposure in ((2.2, 1.0), (1.0, 1.0), (2.4, 0.7)):
            got = img.to_rgb8(zt.Output(tonemap=tm, gamma=gamma, exposure=exposure))
            want = [O.encode(k, gamma, exposure, float(v)) for v in px.reshape(-1)]
            assert list(got) == want


def test_encode_kats_on_product(native_lib):  # image.zig:103-112
    img = zt.Image(4, 1, np.array([[-1, 7, 0.5], [np.nan, 0.5, 0.5], [0, 0, 0], [1, 1, 1]], np.float64))
    lin = img.to_rgb8(zt.Output(gamma=1.0))
    assert list(lin[:4]) == [0, 255, 128, 0]
    assert img.to_rgb8(zt.Output(gamma=2.2))[4] == 186


def test_write_ppm(native_lib):  # image.zig:114-126
    import io
    img = zt.Image(2, 1, np.array([[1.0, 0, 0], [0, 0, 1.0]]))
    buf = io.BytesIO()
    zt.write_ppm(buf, 2, 1, img.to_rgb8())
    assert buf.getvalue() == b"P6\n2 1\n255\n\xff\x00\x00\x00\x00\xff"


def test_device_build_falls_back_to_the_host_tree_without_a_gpu(native_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present: the device build is checked by the gpu tests")
    import kat_scenes as K
    dev = K.random_shapes(3, 500).build(device=True)
    host = K.random_shapes(3, 500).build()
    assert not dev.built_on_device
    (dn, di), (hn, hi) = dev.bvh(), host.bvh()
    assert dn.tobytes() == hn.tobytes() and di.tobytes() == hi.tobytes()


def test_device_entry_points_fail_loudly_without_a_gpu(native_lib):
    """No CPU fallback: on a machine without a usable GPU every rendering
    entry point returns a CUDA error instead of computing on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from zigtrace_b200 import scenes
    s = scenes.cornell().build()
    o = zt.Options(8, 8, 1, 4)
    from zigtrace_b200 import sharding
    fast = zt.GpuConfig(precision=zt.PRECISION_FAST)
    calls = [lambda: zt.render(s, o), lambda: zt.render_rgb8(s, o), lambda: zt.render_png(s, o),
             lambda: zt.forward(s, o), lambda: zt.render_batch([s], [o]), lambda: zt.render(s, o, fast),
             lambda: zt.render_batch([s], [o], fast), lambda: sharding.render_rows(s, o, 0, 4),
             lambda: zt.render(s, o, zt.GpuConfig(zt.MODE_WAVEFRONT_SORTED))]
    for call in calls:
        with pytest.raises(zt.ZigtraceError) as ei:
            call()
        assert ei.value.name == "CudaError"
    # device-resident calls need an uploaded scene: rejected before any device work
    with pytest.raises(zt.ZigtraceError) as ei:
        zt.render_rows_device(s, o, 0, 4, 1 << 20, 0)
    assert ei.value.name in ("CudaError", "InvalidArgument")
