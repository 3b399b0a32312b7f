"""The reference's integrator tests (src/render.zig:188-403), run on the CPU
oracle and on the GPU path with the same tolerances as the reference."""
import math

import numpy as np
import pytest

import kat_scenes as K
from backends import GpuBackend, OracleBackend

import zigtrace_b200 as zt

BACKENDS = [pytest.param(OracleBackend(), id="oracle"),
            pytest.param(GpuBackend(zt.MODE_MEGAKERNEL), id="gpu-mega", marks=pytest.mark.gpu),
            pytest.param(GpuBackend(zt.MODE_WAVEFRONT), id="gpu-wavefront", marks=pytest.mark.gpu),
            pytest.param(GpuBackend(zt.MODE_MEGAKERNEL_REGEN), id="gpu-regen", marks=pytest.mark.gpu),
            pytest.param(GpuBackend(zt.MODE_WAVEFRONT_SORTED), id="gpu-wf-sorted", marks=pytest.mark.gpu)]


@pytest.mark.parametrize("be", BACKENDS)
def test_empty_scene_renders_background_exactly(be):  # render.zig:188-196
    img = be.render(K.empty_scene(), **K.kat_options())
    assert np.allclose(img, [0.25, 0.5, 0.75], atol=1e-12, rtol=0)


@pytest.mark.parametrize("be", BACKENDS)
def test_thread_count_invariance_and_seed_dependence(be):  # render.zig:211-228
    single = be.render(K.demo_scene(), **K.kat_options())
    multi = be.render(K.demo_scene(), **K.kat_options(threads=4))
    assert single.tobytes() == multi.tobytes()
    reseeded = be.render(K.demo_scene(), **K.kat_options(threads=4, seed=99))
    assert single.tobytes() != reseeded.tobytes()


@pytest.mark.parametrize("be", BACKENDS)
def test_diffuse_sphere_under_uniform_sky_reflects_albedo(be):  # render.zig:230-243
    img = be.render(K.albedo_sphere(), **K.kat_options())
    assert np.allclose(img, [0.5, 0.25, 0.125], atol=1e-12, rtol=0)


@pytest.mark.parametrize("be", BACKENDS)
def test_white_furnace_conserves_energy(be):  # render.zig:245-267
    img = be.render(K.furnace(), **K.kat_options(max_depth=64, spp=32))
    assert np.allclose(img.mean(axis=0), [1, 1, 1], atol=0.03, rtol=0)


@pytest.mark.parametrize("be", BACKENDS)
def test_emitters_are_seen_directly(be):  # render.zig:269-280
    img = be.render(K.emitter_scene(), **K.kat_options())
    assert (img == np.array([2, 1, 0.5])).all()


@pytest.mark.parametrize("be", BACKENDS)
def test_rejects_degenerate_options(be):  # render.zig:282-288
    with pytest.raises((ValueError, RuntimeError)) as ei:
        be.render(K.demo_scene(), **K.kat_options(spp=0))
    assert "InvalidOptions" in str(ei.value)
    with pytest.raises((ValueError, RuntimeError)):
        be.render(K.demo_scene(), **K.kat_options(tile_size=0))


def _stats(v):
    x = v[:, 0]
    mean = x.sum() / len(x)
    return mean, (x * x).sum() / len(x) - mean * mean


@pytest.mark.parametrize("be", BACKENDS)
def test_sphere_light_irradiance_closed_form(be):  # render.zig:313-325
    scene = K.lamp_over_floor(1)
    expected = 0.5 * 2.0 / 9.0
    with_nee, _ = _stats(be.mean_radiance(scene, (0, 1, 0), (0, -1, 0), 1, 20000, 2, True))
    without, _ = _stats(be.mean_radiance(scene, (0, 1, 0), (0, -1, 0), 2, 40000, 2, False))
    assert math.isclose(with_nee, expected, rel_tol=0.02)
    assert math.isclose(without, expected, rel_tol=0.06)


@pytest.mark.parametrize("be", BACKENDS)
def test_light_sampling_slashes_variance(be):  # render.zig:327-337
    scene = K.lamp_over_floor(0.2)
    mw, vw = _stats(be.mean_radiance(scene, (0, 1, 0), (0, -1, 0), 3, 5000, 2, True))
    _, vo = _stats(be.mean_radiance(scene, (0, 1, 0), (0, -1, 0), 3, 5000, 2, False))
    assert vw * 10 < vo
    assert math.isclose(mw, 0.5 * 2.0 * 0.04 / 9.0, rel_tol=0.02)


@pytest.mark.parametrize("be", BACKENDS)
def test_emitters_seen_through_a_mirror_are_not_weighted(be):  # render.zig:339-355
    import oracle as O
    scene = K.mirror_lamp()
    d = np.array([1.0, -1.0, 0.0])
    d = d * (1.0 / math.sqrt(d @ d))
    state = O.Rng.init(9).s.copy()
    for nee in (True, False):
        c = be.trace_with(scene, (0, 4, 0), d, state, 4, nee)
        assert np.allclose(c, [3, 2, 1], atol=1e-9, rtol=0)


@pytest.mark.parametrize("be", BACKENDS)
def test_shadowed_lights_add_nothing(be):  # render.zig:357-369
    m, _ = _stats(be.mean_radiance(K.shadowed_lamp(), (0, 1, 0), (0, -1, 0), 4, 2000, 2, True))
    assert m < 0.5 * 2.0 / 9.0 * 0.6


@pytest.mark.parametrize("be", BACKENDS)
def test_light_sampling_and_plain_path_tracing_agree(be):  # render.zig:371-403
    scene = K.lit_room()
    w = be.render(scene, **K.kat_options(spp=256, max_depth=6, threads=2))
    o = be.render(scene, **K.kat_options(spp=1024, max_depth=6, threads=2, light_sampling=False))
    mw, mo = w.sum(axis=0), o.sum(axis=0)
    assert mw.max() > 0
    assert np.all(np.abs(mw - mo) <= 0.05 * mo.max())
