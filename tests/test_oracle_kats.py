"""The reference's component tests restated against the CPU oracle.

Each test cites the Zig test it restates and keeps its tolerance.  Together
with the RNG golden vectors these pin the oracle, which then checks the GPU.
"""
import math

import numpy as np
import pytest

import kat_scenes as K
import oracle as O
import zigtrace_b200 as zt
from zigtrace_b200 import Material, sphere, triangle, plane


def norm(v):
    v = np.asarray(v, np.float64)
    return v * (1.0 / math.sqrt(v @ v))


# ------------------------------------------------------------------ rng ----
def test_same_seed_same_sequence():  # rng.zig:92-99
    a, b = O.Rng.init(42), O.Rng.init(42)
    assert (a.next_n(100) == b.next_n(100)).all()
    c = O.Rng.init(43)
    assert a.next_n(1)[0] != c.next_n(1)[0]


def test_streams_differ():  # rng.zig:101-105
    assert O.Rng.for_stream(7, 0).next_n(1)[0] != O.Rng.for_stream(7, 1).next_n(1)[0]


def test_float_range_and_mean():  # rng.zig:107-117
    f = O.Rng.init(1).float_n(100_000)
    assert (f >= 0).all() and (f < 1).all()
    assert abs(f.sum() / len(f) - 0.5) <= 0.01


def test_below_stays_in_range():  # rng.zig:119-124
    r = O.Rng.init(9)
    counts = np.zeros(5, int)
    for _ in range(10_000):
        counts[r.below(5)] += 1
    assert ((counts > 1700) & (counts < 2300)).all()


def test_sampling_domains():  # rng.zig:126-138
    r = O.Rng.init(3)
    mean = np.zeros(3)
    for _ in range(20_000):
        u = r.unit_vector()
        assert abs(math.sqrt(u @ u) - 1) <= 1e-9
        mean += u
        s = r.in_unit_sphere()
        assert s @ s < 1
        d = r.in_unit_disk()
        assert d @ d < 1 and d[2] == 0
    assert math.sqrt((mean / 20_000) @ (mean / 20_000)) < 0.03


def test_sincos_and_pow5_accuracy():
    """The project's sin/cos stay within 2 ulp of libm on [0, 2pi); pow5 is
    std.math.pow's x*((x*x)*(x*x)) with pow(1,5)=1, pow(0,5)=0."""
    xs = np.linspace(0, 2 * math.pi, 20001)[:-1]
    for x in xs:
        s, c = O.sincos(float(x))
        assert abs(s - math.sin(x)) <= 2 * math.ulp(max(abs(math.sin(x)), 1e-300)) + 1e-300 or abs(s - math.sin(x)) < 1e-16
        assert abs(c - math.cos(x)) <= 2 * math.ulp(abs(math.cos(x))) or abs(c - math.cos(x)) < 1e-16
    for x in (0.0, 0.3, 0.5, 1.0, 1.7, 2.0):
        assert O.pow5(x) == x * ((x * x) * (x * x))
        assert math.isclose(O.pow5(x), x ** 5, rel_tol=4e-16)


# ----------------------------------------------------------------- aabb ----
def test_slab_hit():  # aabb.zig:104-117
    lo, hi = (-1, -1, -1), (1, 1, 1)
    assert abs(O.aabb_hit(lo, hi, (0, 0, -5), (0, 0, 1), 0, 100) - 4) <= 1e-12
    assert O.aabb_hit(lo, hi, (0, 0, -5), (0, 0, 1), 0, 3) is None
    assert O.aabb_hit(lo, hi, (2, 0, -5), (0, 0, 1), 0, 100) is None
    assert O.aabb_hit(lo, hi, (0, 0, 0), norm((1, 1, 0)), 0, 100) is not None


# ------------------------------------------------------------- geometry ----
def test_sphere_hit_from_outside_and_inside():  # geometry.zig:266-283
    s = sphere((0, 0, -5), 1, 3)
    h = O.shape_intersect(s, (0, 0, 0), (0, 0, -1), 1e-4, 100)
    assert abs(h["t"] - 4) <= 1e-12 and h["front_face"] == 1
    assert np.allclose(h["normal"], (0, 0, 1), atol=1e-12) and h["material"] == 3
    hi = O.shape_intersect(s, (0, 0, -5), (0, 0, -1), 1e-4, 100)
    assert abs(hi["t"] - 1) <= 1e-12 and hi["front_face"] == 0
    assert np.allclose(hi["normal"], (0, 0, 1), atol=1e-12)
    assert O.shape_intersect(s, (0, 2, 0), (0, 0, -1), 1e-4, 100) is None


def test_negative_radius_flips_the_normal():  # geometry.zig:285-292
    s = sphere((0, 0, 0), -1, 0)
    h = O.shape_intersect(s, (0, 0, 5), (0, 0, -1), 1e-4, 100)
    assert abs(h["t"] - 4) <= 1e-12 and h["front_face"] == 0


def test_plane_hit():  # geometry.zig:294-307
    p = plane((0, 0, 0), (0, 1, 0), 0)
    h = O.shape_intersect(p, (0, 2, 0), (1, -1, 0), 1e-4, 100)
    assert abs(h["t"] - 2) <= 1e-12 and np.allclose(h["point"], (2, 0, 0), atol=1e-12)
    assert O.shape_intersect(p, (0, 2, 0), (1, 0, 0), 1e-4, 100) is None
    hb = O.shape_intersect(p, (0, -1, 0), (0, 1, 0), 1e-4, 100)
    assert hb["front_face"] == 0 and (hb["normal"] == (0, -1, 0)).all()


def test_triangle_hit_and_edges():  # geometry.zig:309-323
    tri = triangle((-1, -1, -3), (1, -1, -3), (0, 1, -3), 0)
    h = O.shape_intersect(tri, (0, 0, 0), (0, 0, -1), 1e-4, 100)
    assert abs(h["t"] - 3) <= 1e-12 and np.allclose(h["normal"], (0, 0, 1), atol=1e-12)
    assert O.shape_intersect(tri, (0.9, 0.9, 0), (0, 0, -1), 1e-4, 100) is None
    assert O.shape_intersect(tri, (0, 0, 0), (0, 0, 1), 1e-4, 100) is None


def test_intersect_all_picks_the_closest():  # geometry.zig:325-334
    shapes = np.array([sphere((0, 0, -10), 1, 0), sphere((0, 0, -4), 1, 1), plane((0, 0, -20), (0, 0, 1), 2)])
    assert O.intersect_all(shapes, (0, 0, 0), (0, 0, -1), 1e-4, 1e9)["material"] == 1


def test_scene_routes_planes_and_finds_closest_hit():  # scene.zig:233-250
    s = zt.Scene()
    m = s.add_material(Material.lambertian((1, 1, 1)))
    s.add(sphere((0, 0, -5), 1, m))
    s.add(plane((0, 0, -3), (0, 0, 1), m))
    s.add_quad((-1, -1, -2), (2, 0, 0), (0, 0.5, 0), m)
    os_ = O.OracleScene.from_scene(s)
    c = os_.counts()
    assert c["bounded"] == 3 and c["planes"] == 1
    assert abs(os_.intersect((0, 0, 0), (0, 0, -1), 1e-4, 1e9)["t"] - 3) <= 1e-12
    hq = os_.intersect((0, -0.75, 0), (0, 0, -1), 1e-4, 1e9)
    assert abs(hq["t"] - 2) <= 1e-12 and hq["front_face"] == 1


def test_sky_background_gradient():  # scene.zig:252-257
    bg = zt.Background.sky((1, 1, 1), (0, 0, 0)).record()
    assert (O.background_radiance(bg, (1, 0, 0)) == 1).all()
    assert (O.background_radiance(bg, (0, 3, 0)) == 0).all()
    assert (O.background_radiance(bg, (0, -1, 0)) == 1).all()


# ------------------------------------------------------------------ bvh ----
def random_rays(rng, shapes, n):
    """expectMatchesBruteForce's ray mix (bvh.zig:291-301)."""
    cents = []
    for s in shapes:
        if s["kind"] == zt.SPHERE:
            cents.append(s["p"][:3])
        else:
            p = s["p"].reshape(3, 3)
            lo, hi = p.min(0), p.max(0)
            cents.append((lo + hi) * 0.5)
    for _ in range(n):
        o = rng.uniform(-15, 15, 3)
        if rng.random() < 0.8:
            d = cents[rng.integers(len(cents))] + rng.uniform(-0.5, 0.5, 3) - o
            yield o, norm(d)
        else:
            yield o, norm(rng.normal(size=3))


def expect_matches_brute_force(scene, rng, rays):
    os_ = O.OracleScene.from_scene(scene)
    shapes = scene.shapes
    hits = 0
    for o, d in random_rays(rng, shapes, rays):
        want = O.intersect_all(shapes, o, d, 1e-6, 1e9)
        got = os_.intersect(o, d, 1e-6, 1e9)
        assert (want is None) == (got is None)
        if want is not None:
            hits += 1
            assert want["t"] == got["t"] and want["material"] == got["material"]
    assert hits > 0
    if len(shapes) >= 7:
        assert hits > rays // 4


@pytest.mark.parametrize("n", [1, 2, 3, 7, 50, 400])
def test_bvh_agrees_with_brute_force(n):  # bvh.zig:316-325
    expect_matches_brute_force(K.random_shapes(2026 + n, n), np.random.default_rng(n), 3000)


def test_bvh_structure_is_valid():  # bvh.zig:327-354
    scene = K.random_shapes(11, 257)
    nodes, idx = O.OracleScene.from_scene(scene).bvh()
    seen = np.zeros(257, bool)
    for nd in nodes:
        if nd["count"] == 0:
            for c in (nd["first"], nd["first"] + 1):
                cb = nodes[c]
                assert (np.minimum(cb["bmin"], nd["bmin"]) == nd["bmin"]).all()
                assert (np.maximum(cb["bmax"], nd["bmax"]) == nd["bmax"]).all()
            continue
        for i in idx[nd["first"]:nd["first"] + nd["count"]]:
            assert not seen[i]
            seen[i] = True
    assert seen.all()
    assert O.OracleScene.from_scene(scene).bvh_depth() < 30
    assert len(nodes) <= 2 * 257 - 1


def test_bvh_handles_coincident_primitives_and_empty_input():  # bvh.zig:356-367
    s = zt.Scene()
    for i in range(40):
        m = s.add_material(Material.lambertian((1, 1, 1)))
        s.add(sphere((0, 0, 0), 1 + i * 0.01, m))
    expect_matches_brute_force(s, np.random.default_rng(5), 500)
    empty = O.OracleScene.from_scene(zt.Scene())
    assert empty.intersect((0, 0, 0), (1, 0, 0), 0, 1e9) is None


# ------------------------------------------------------------- material ----
def test_lambertian_scatters_into_hemisphere_with_albedo():  # material.zig:84-99
    rng = O.Rng.init(5)
    m = Material.lambertian((0.2, 0.4, 0.6))
    h = O.make_hit(front_face=True)
    total = 0.0
    for _ in range(20_000):
        att, _, d = O.material_scatter(m, (0, -1, 0), h, rng)
        assert (att == (0.2, 0.4, 0.6)).all()
        c = d @ (0, 1, 0)
        assert c >= -1e-9
        total += c
    assert abs(total / 20_000 - 2 / 3) <= 0.01


def test_perfect_metal_mirrors():  # material.zig:101-107
    _, _, d = O.material_scatter(Material.metal((1, 1, 1)), (1, -1, 0), O.make_hit(), O.Rng.init(1))
    assert np.allclose(d, norm((1, 1, 0)), atol=1e-12)


def test_dielectric_with_unit_ior_passes_straight_through():  # material.zig:109-118
    rng = O.Rng.init(2)
    d0 = norm((0.3, -1, 0.1))
    for _ in range(100):
        att, _, d = O.material_scatter(Material.dielectric(1.0), d0, O.make_hit(), rng)
        assert np.allclose(d, d0, atol=1e-12) and (att == 1).all()


def test_total_internal_reflection():  # material.zig:120-127
    d0 = norm((1, -0.2, 0))
    _, _, d = O.material_scatter(Material.dielectric(1.5), d0, O.make_hit(front_face=False), O.Rng.init(3))
    assert np.allclose(d, d0 - 2 * (d0 @ (0, 1, 0)) * np.array([0, 1, 0]), atol=1e-12)


def test_schlick_endpoints():  # material.zig:129-132
    assert abs(O.schlick(1.0, 1.0 / 1.5) - 0.04) <= 1e-12
    assert abs(O.schlick(0.0, 1.0 / 1.5) - 1.0) <= 1e-12


def test_emissive_emits_only_from_the_front_and_never_scatters():  # material.zig:134-142
    m = Material.emissive((4, 4, 4))
    assert (O.material_emitted(m, O.make_hit(front_face=True)) == 4).all()
    assert (O.material_emitted(m, O.make_hit(front_face=False)) == 0).all()
    assert O.material_scatter(m, (0, -1, 0), O.make_hit(), O.Rng.init(4)) is None
    assert (O.material_emitted(Material.lambertian((1, 1, 1)), O.make_hit()) == 0).all()


# --------------------------------------------------------------- lights ----
def test_only_bounded_emissive_shapes_become_lights():  # light.zig:358-369
    lights, cdf, total = O.OracleScene.from_scene(K.lamp_scene()).lights()
    assert len(lights) == 3
    sphere_weight = 4 * math.pi * 0.25
    assert abs(lights[0]["weight"] - sphere_weight) <= 1e-12
    assert abs(total - (sphere_weight + 4 * 2.0)) <= 1e-12


def test_scene_without_emitters_never_samples():  # light.zig:371-380
    s = zt.Scene()
    m = s.add_material(Material.lambertian((1, 1, 1)))
    s.add(sphere((0, 0, 0), 1, m))
    os_ = O.OracleScene.from_scene(s)
    assert os_.counts()["lights"] == 0
    assert os_.lights_sample((0, 5, 0), O.Rng.init(1)) is None


def test_planes_bubbles_and_dark_emitters_are_not_sampled():  # light.zig:382-392
    s = zt.Scene()
    lamp = s.add_material(Material.emissive((1, 1, 1)))
    dark = s.add_material(Material.emissive((0, 0, 0)))
    s.add(plane((0, 0, 0), (0, 1, 0), lamp))
    s.add(sphere((0, 2, 0), -1, lamp))
    s.add(sphere((0, 5, 0), 1, dark))
    assert O.OracleScene.from_scene(s).counts()["lights"] == 0


def test_samples_land_on_emitters_with_consistent_pdfs():  # light.zig:394-414
    os_ = O.OracleScene.from_scene(K.lamp_scene())
    mats = K.lamp_scene().materials
    rng = O.Rng.init(7)
    origin = (0.5, 0.2, 0.3)
    got = 0
    for _ in range(2000):
        s = os_.lights_sample(origin, rng)
        if s is None:
            continue
        got += 1
        assert abs(math.sqrt(s["dir"] @ s["dir"]) - 1) <= 1e-9
        hit = os_.intersect(origin, s["dir"], 1e-6, math.inf)
        assert math.isclose(s["distance"], hit["t"], rel_tol=1e-6)
        assert mats[hit["material"]]["kind"] == zt.EMISSIVE
        assert hit["front_face"] == 1
        assert math.isclose(s["pdf"], os_.pdf_hit(origin, hit), rel_tol=1e-6)
    assert got > 1500


def test_reciprocal_pdf_matches_sphere_solid_angle():  # light.zig:416-430
    s = zt.Scene()
    lamp = s.add_material(Material.emissive((1, 1, 1)))
    s.add(sphere((0, 0, -4), 1, lamp))
    os_ = O.OracleScene.from_scene(s)
    rng = O.Rng.init(11)
    total = sum(1 / os_.lights_sample((0, 0, 0), rng)["pdf"] for _ in range(20000))
    cos_max = math.sqrt(1 - 1.0 / 16.0)
    assert math.isclose(2 * math.pi * (1 - cos_max), total / 20000, rel_tol=1e-9)


def test_reciprocal_pdf_matches_triangle_solid_angle():  # light.zig:432-459
    s = zt.Scene()
    lamp = s.add_material(Material.emissive((1, 1, 1)))
    tri = triangle((-1, 2, -1), (1.5, 2, -1), (0, 2, 1.5), lamp)
    s.add(tri)
    os_ = O.OracleScene.from_scene(s)
    rng = O.Rng.init(21)
    total = sum(1 / os_.lights_sample((0, 0, 0), rng)["pdf"] for _ in range(40000))
    hits = 0
    trials = 400_000
    for _ in range(trials):
        if O.shape_intersect(tri, (0, 0, 0), rng.unit_vector(), 1e-9, 1e9) is not None:
            hits += 1
    brute = 4 * math.pi * hits / trials
    assert math.isclose(brute, total / 40000, rel_tol=0.03)


def test_back_facing_triangle_and_enclosing_sphere_light_nothing():  # light.zig:461-478
    s = zt.Scene()
    lamp = s.add_material(Material.emissive((1, 1, 1)))
    s.add(triangle((-1, 0, -1), (-1, 0, 1), (1, 0, 0), lamp))
    os_ = O.OracleScene.from_scene(s)
    rng = O.Rng.init(3)
    assert os_.lights_sample((0, -2, 0), rng) is None
    assert os_.lights_sample((0, 2, 0), rng) is not None
    inside = zt.Scene()
    l2 = inside.add_material(Material.emissive((1, 1, 1)))
    inside.add(sphere((0, 0, 0), 2, l2))
    assert O.OracleScene.from_scene(inside).lights_sample((0, 0, 0), rng) is None


def test_lights_are_picked_in_proportion_to_power():  # light.zig:480-494
    s = zt.Scene()
    weak = s.add_material(Material.emissive((1, 1, 1)))
    strong = s.add_material(Material.emissive((3, 3, 3)))
    s.add(sphere((-5, 0, 0), 1, weak))
    s.add(sphere((5, 0, 0), 1, strong))
    os_ = O.OracleScene.from_scene(s)
    rng = O.Rng.init(5)
    right = sum(1 for _ in range(20000) if os_.lights_sample((0, 0, 0), rng)["dir"][0] > 0)
    assert abs(right / 20000 - 0.75) <= 0.015


# --------------------------------------------------------------- camera ----
def test_centre_ray_points_at_look_at():  # camera.zig:72-78
    cfg = zt.CameraConfig(look_from=(1, 2, 3), look_at=(4, 2, -1)).record()
    cam = O.camera_init(cfg, 16.0 / 9.0)
    o, d = O.camera_ray(cam, 0.5, 0.5, O.Rng.init(0))
    assert np.allclose(d, norm((3, 0, -4)), atol=1e-12) and (o == (1, 2, 3)).all()


def test_image_orientation_and_field_of_view():  # camera.zig:80-88
    cam = O.camera_init(zt.CameraConfig(vfov=90).record(), 1.0)
    rng = O.Rng.init(0)
    _, tl = O.camera_ray(cam, 0, 0, rng)
    assert tl[0] < 0 and tl[1] > 0
    _, top = O.camera_ray(cam, 0.5, 0, rng)
    assert abs(math.degrees(math.atan2(top[1], -top[2])) - 45) <= 1e-9


def test_depth_of_field_rays_converge_on_focus_plane():  # camera.zig:90-108
    cfg = zt.CameraConfig(look_from=(0, 0, 5), look_at=(0, 0, 0), aperture=0.8, focus_dist=5).record()
    cam = O.camera_init(cfg, 1.5)
    rng = O.Rng.init(9)
    spread = 0.0
    for _ in range(200):
        o, d = O.camera_ray(cam, 0.5, 0.5, rng)
        spread += abs(o[0]) + abs(o[1])
        hit = o + d * ((0 - o[2]) / d[2])
        assert np.allclose(hit, 0, atol=1e-9)
        assert math.sqrt((o - (0, 0, 5)) @ (o - (0, 0, 5))) <= 0.4 + 1e-12
    assert spread > 0


# -------------------------------------------------- differentiable form ----
def test_detached_forward_is_the_render_at_own_colors_and_linear_in_emission():
    from zigtrace_b200 import scenes
    scene, target = scenes.cornell_diff()
    os_ = O.OracleScene.from_scene(scene)
    theta = np.array([m["color"] for m in scene.materials])
    base = os_.render_params(20, 20, 2, 8, theta)
    assert base.tobytes() == os_.render(20, 20, 2, 8, threads=2).tobytes()
    doubled = theta.copy()
    doubled[32:] *= 2.0  # every term carries exactly one emitter radiance
    assert np.allclose(os_.render_params(20, 20, 2, 8, doubled), 2 * base, rtol=1e-12, atol=1e-15)


# ---------------------------------------------------------------- image ----
def test_tone_mapping_curves():  # image.zig:85-101
    assert O.tonemap(1, 1.0) == 0.5 and O.tonemap(0, -3.0) == 0
    assert abs(O.tonemap(2, 0)) <= 1e-12 and O.tonemap(2, 100) > 0.99
    for k in (0, 1, 2):
        xs = np.arange(0, 4, 0.05)
        ys = [O.tonemap(k, float(x)) for x in xs]
        assert all(b >= a for a, b in zip(ys, ys[1:]))


def test_encode_applies_gamma_and_clamps():  # image.zig:103-112
    assert O.encode(0, 1.0, 1.0, -1) == 0 and O.encode(0, 1.0, 1.0, 7) == 255
    assert O.encode(0, 1.0, 1.0, 0.5) == 128 and O.encode(0, 1.0, 1.0, float("nan")) == 0
    assert O.encode(0, 2.2, 1.0, 0.5) == 186
