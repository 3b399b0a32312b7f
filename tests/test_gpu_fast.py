"""The fast traversal (ZT_PRECISION_FAST) on the GPU against the oracle.

Bar: the statistical one for renders that are not bit-identical to the
reference algorithm (oracle/agreement.py) -- per-channel relative RMSE below
1e-3 against the oracle's image at the same seed and mean luminance within 3
Monte Carlo standard errors (from the oracle's per-pixel second moment).  The
fast walk reaches every BVH leaf the f64 walk reaches, so paths differ only
where a closest hit is decided by a tie or a grazing box test: the tests
also require nearly every pixel to be bit-identical to the oracle's.
Renders the float records cannot serve (a camera beyond their coordinate
range) and single renders of scenes under 64 bounded primitives take the
exact walk and must then be bit-identical; the scenes of the statistical
tests carry an extra 320-triangle icosphere to stay above that size.
"""
import numpy as np
import pytest

import kat_scenes as K
import oracle as O
import zigtrace_b200 as zt
from oracle.agreement import image_agreement
from zigtrace_b200 import scenes

pytestmark = pytest.mark.gpu

FAST = zt.GpuConfig(precision=zt.PRECISION_FAST)
MODES = [pytest.param(zt.MODE_MEGAKERNEL, id="mega"), pytest.param(zt.MODE_MEGAKERNEL_REGEN, id="regen")]
FAST_MIN_PRIMITIVES = 64  # single renders of smaller scenes take the exact walk


def _denser(scene, center, radius, material=0, seed=0):
    """Adds a 320-triangle icosphere so that a single render of the scene
    takes the fast walk (at least 64 bounded primitives)."""
    verts, faces = scenes.icosphere(2)
    v = np.asarray(verts) * radius + np.asarray(center, float)
    f = np.asarray(faces)
    scene.add_triangles(v[f[:, 0]], v[f[:, 1]], v[f[:, 2]], material)
    assert scene.primitive_count() - 1 >= FAST_MIN_PRIMITIVES
    return scene


def cornell_dense():
    s = scenes.cornell()
    return _denser(s, (400, 330, 200), 60.0, material=2)


def fuzz_dense(seed):
    s = K.fuzz_scene(seed)
    return _denser(s, (1.5, 0.6, -3.5), 0.5, material=0)


def _whole(scene, o, cfg):
    img = zt.render(scene, o, cfg).pixels
    want, m2 = O.OracleScene.from_scene(scene).render_moments(o.width, o.height, o.spp, o.max_depth, seed=o.seed,
                                                              light_sampling=o.light_sampling)
    return image_agreement(img, want, m2, o.spp)


def _subset(scene, o, cfg, n, seed):
    img = zt.render(scene, o, cfg).pixels
    rng = np.random.default_rng(seed)
    pix = np.unique(rng.integers(0, o.width * o.height, n)).astype(np.uint64)
    want, m2 = O.OracleScene.from_scene(scene).render_pixels_moments(o.width, o.height, o.spp, o.max_depth, pix,
                                                                     seed=o.seed, light_sampling=o.light_sampling)
    return image_agreement(img[pix.astype(np.int64)], want, m2, o.spp)


@pytest.mark.parametrize("mode", MODES)
def test_cornell_full_size(mode):
    a = _whole(cornell_dense().build(), scenes.CORNELL_OPTIONS, zt.GpuConfig(mode, precision=zt.PRECISION_FAST))
    assert a["ok"], a
    assert a["identical_pixels"] > 0.99, a


def test_random_spheres_full_size_subset():
    """1280x720, 16 spp, depth 50: the ground plane outside the BVH, thin lens."""
    a = _subset(scenes.random_spheres().build(), scenes.SPHERES_OPTIONS, FAST, 20000, seed=1)
    assert a["ok"], a
    assert a["identical_pixels"] > 0.99, a


def test_triangle_heavy_benchmark_config_subset():
    """The benchmark configuration: 1920x1080, 64 spp, depth 16, 1M triangles."""
    a = _subset(scenes.triangle_heavy().build(device=True), scenes.TRIANGLE_HEAVY_OPTIONS, FAST, 6000, seed=2)
    assert a["ok"], a
    assert a["identical_pixels"] > 0.99, a


@pytest.mark.parametrize("seed", range(8))
def test_fuzz_scenes(seed):
    """Every shape, material and light kind, lens sampling, both backgrounds."""
    scene = fuzz_dense(seed).build()
    a = _whole(scene, zt.Options(64, 48, 16, 12, seed=seed), FAST)
    assert a["ok"], a
    assert a["identical_pixels"] > 0.98, a


def test_light_sampling_off_and_batch():
    scene = cornell_dense().build()
    o = zt.Options(96, 96, 8, 16, light_sampling=False)
    a = _whole(scene, o, FAST)
    assert a["ok"], a
    items = scenes.batch_workload(count=12, seed=5)
    scs, opts = [s.build() for s, _ in items], [o for _, o in items]
    imgs = zt.render_batch(scs, opts, FAST)
    for s, o, img in zip(scs, opts, imgs):
        want, m2 = O.OracleScene.from_scene(s).render_moments(o.width, o.height, o.spp, o.max_depth, seed=o.seed)
        a = image_agreement(img.pixels, want, m2, o.spp)
        assert a["ok"] and a["identical_pixels"] > 0.99, a


def test_camera_outside_the_float_range_renders_exact():
    """A camera farther than 1e7 from the origin is outside the range the
    float test handles: the render falls back to the f64 walk and is
    bit-identical to the oracle."""
    far = cornell_dense()
    far.camera = zt.CameraConfig(look_from=(278, 278, -2e7), look_at=(278, 278, 0), vfov=0.01)
    far.build()
    o = zt.Options(64, 64, 4, 8)
    assert zt.render(far, o, FAST).pixels.tobytes() == O.OracleScene.from_scene(far).render(64, 64, 4, 8).tobytes()


def test_small_scene_single_render_is_exact():
    """Below 64 bounded primitives a single render takes the exact walk: the
    fast precision then gives the oracle's pixels bit for bit."""
    scene = scenes.cornell().build()
    o = zt.Options(64, 64, 4, 16)
    want = O.OracleScene.from_scene(scene).render(64, 64, 4, 16)
    assert zt.render(scene, o, FAST).pixels.tobytes() == want.tobytes()


def test_fast_is_deterministic():
    scene = scenes.random_spheres().build()
    o = zt.Options(320, 180, 4, 50, seed=7)
    assert zt.render(scene, o, FAST).pixels.tobytes() == zt.render(scene, o, FAST).pixels.tobytes()
