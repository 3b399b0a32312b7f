"""The reference's test scenes, restated with the Scene API.

Each builder cites the test it comes from; ``kat_options`` is
testOptions (src/render.zig:184-186).
"""
from __future__ import annotations

import numpy as np

import zigtrace_b200 as zt
from zigtrace_b200 import Background, CameraConfig, Material, Scene, plane, sphere, triangle


def kat_options(**kw) -> dict:
    o = dict(width=24, height=16, spp=8, max_depth=8, tile_size=5)
    o.update(kw)
    return o


def empty_scene() -> Scene:  # render.zig:188-196
    s = Scene()
    s.background = Background.solid((0.25, 0.5, 0.75))
    return s


def demo_scene() -> Scene:  # render.zig:198-209
    s = Scene()
    ground = s.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    glass = s.add_material(Material.dielectric(1.5))
    gold = s.add_material(Material.metal((0.8, 0.6, 0.2), 0.2))
    lamp = s.add_material(Material.emissive((3, 3, 3)))
    s.add(plane((0, -1, 0), (0, 1, 0), ground))
    s.add(sphere((-1, 0, -3), 1, glass))
    s.add(sphere((1, 0, -3), 1, gold))
    s.add(sphere((0, 2, -4), 0.5, lamp))
    s.camera = CameraConfig(look_from=(0, 0.5, 1), look_at=(0, 0, -3), aperture=0.1)
    return s


def albedo_sphere() -> Scene:  # render.zig:230-243
    s = Scene()
    s.background = Background.solid((1, 1, 1))
    m = s.add_material(Material.lambertian((0.5, 0.25, 0.125)))
    s.add(sphere((0, 0, -3), 1, m))
    s.camera = CameraConfig(vfov=10)
    return s


def furnace() -> Scene:  # render.zig:245-267
    s = Scene()
    s.background = Background.solid((1, 1, 1))
    glass = s.add_material(Material.dielectric(1.5))
    white = s.add_material(Material.lambertian((1, 1, 1)))
    s.add(sphere((0, 0, -3), 1, glass))
    s.add(sphere((0, 0, -3), 0.5, white))
    return s


def emitter_scene() -> Scene:  # render.zig:269-280
    s = Scene()
    s.background = Background.solid((0, 0, 0))
    lamp = s.add_material(Material.emissive((2, 1, 0.5)))
    s.add(sphere((0, 0, -2), 1, lamp))
    s.camera = CameraConfig(vfov=20)
    return s


def lamp_over_floor(radius: float) -> Scene:  # render.zig:304-311
    s = Scene()
    s.background = Background.solid((0, 0, 0))
    floor = s.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    lamp = s.add_material(Material.emissive((2, 2, 2)))
    s.add(plane((0, 0, 0), (0, 1, 0), floor))
    s.add(sphere((0, 3, 0), radius, lamp))
    return s


def mirror_lamp() -> Scene:  # render.zig:339-355
    s = Scene()
    s.background = Background.solid((0, 0, 0))
    mirror = s.add_material(Material.metal((1, 1, 1), 0))
    lamp = s.add_material(Material.emissive((3, 2, 1)))
    s.add(plane((0, 0, 0), (0, 1, 0), mirror))
    s.add(sphere((8, 4, 0), 1, lamp))
    return s


def shadowed_lamp() -> Scene:  # render.zig:357-369
    s = lamp_over_floor(1)
    blocker = s.add_material(Material.lambertian((0, 0, 0)))
    s.add(sphere((0, 1.8, 0), 0.6, blocker))
    return s


def lit_room() -> Scene:  # render.zig:371-403
    s = Scene()
    s.background = Background.solid((0, 0, 0))
    wall = s.add_material(Material.lambertian((0.7, 0.6, 0.5)))
    lamp = s.add_material(Material.emissive((6, 6, 6)))
    ball = s.add_material(Material.lambertian((0.2, 0.5, 0.8)))
    s.add(plane((0, 0, 0), (0, 1, 0), wall))
    s.add_quad((-5, 0, -8), (10, 0, 0), (0, 6, 0), wall)
    s.add_quad((-1, 4, -4), (2, 0, 0), (0, 0, 2), lamp)
    s.add(sphere((0, 1, -3), 1, ball))
    s.camera = CameraConfig(look_from=(0, 2, 3), look_at=(0, 1.5, -3), vfov=60)
    return s


def lamp_scene() -> Scene:  # light.zig:346-356
    s = Scene()
    white = s.add_material(Material.lambertian((1, 1, 1)))
    dim = s.add_material(Material.emissive((1, 1, 1)))
    bright = s.add_material(Material.emissive((4, 4, 4)))
    s.add(plane((0, 0, 0), (0, 1, 0), white))
    s.add(sphere((0, 3, 0), 0.5, dim))
    s.add_quad((2, 2.5, -1), (1, 0, 0), (0, 0, 2), bright)
    s.add(sphere((-3, 1, 0), 1, white))
    return s


def glass_scene() -> Scene:
    """The example glass scene's content (examples/glass.txt): bubble,
    water, copper, mirror tetrahedron, small emitter, sky light, DOF."""
    s = Scene()
    s.background = Background.sky((1, 1, 1), (0.45, 0.65, 1.0))
    floor = s.add_material(Material.lambertian((0.55, 0.55, 0.5)))
    glass = s.add_material(Material.dielectric(1.5))
    water = s.add_material(Material.dielectric(1.33))
    copper = s.add_material(Material.metal((0.95, 0.64, 0.54), 0.25))
    mirror = s.add_material(Material.metal((0.95, 0.95, 0.95), 0.0))
    blue = s.add_material(Material.lambertian((0.1, 0.2, 0.6)))
    warm = s.add_material(Material.emissive((6, 3.5, 1.5)))
    s.add(plane((0, 0, 0), (0, 1, 0), floor))
    s.add(sphere((0, 0.6, 0), 0.6, glass))
    s.add(sphere((0, 0.6, 0), -0.55, glass))
    s.add(sphere((-1.35, 0.45, -0.4), 0.45, copper))
    s.add(sphere((1.35, 0.45, -0.4), 0.45, blue))
    s.add(sphere((0.6, 0.18, 1.0), 0.18, water))
    s.add(sphere((-0.7, 0.15, 1.1), 0.15, warm))
    s.add(triangle((-0.6, 0, -2.2), (0.6, 0, -2.2), (0, 0, -1.2), mirror))
    s.add(triangle((-0.6, 0, -2.2), (0, 1.2, -1.9), (0.6, 0, -2.2), mirror))
    s.add(triangle((0.6, 0, -2.2), (0, 1.2, -1.9), (0, 0, -1.2), mirror))
    s.add(triangle((0, 0, -1.2), (0, 1.2, -1.9), (-0.6, 0, -2.2), mirror))
    s.camera = CameraConfig(look_from=(0, 1.2, 4.5), look_at=(0, 0.6, 0), vfov=35, aperture=0.12, focus_dist=4.4)
    return s


def random_shapes(rng_seed: int, n: int) -> Scene:
    """randomScene of bvh.zig:272-289 (spheres and triangles, one material
    per shape), generated with numpy instead of the reference's Rng."""
    rng = np.random.default_rng(rng_seed)
    s = Scene()
    for i in range(n):
        s.add_material(Material.lambertian((0.5, 0.5, 0.5)))
        if rng.random() < 0.5:
            s.add(sphere(rng.uniform(-10, 10, 3), rng.uniform(0.05, 1.5), i))
        else:
            c = rng.uniform(-10, 10, 3)
            s.add(triangle(c + rng.uniform(-2, 2, 3), c + rng.uniform(-2, 2, 3), c + rng.uniform(-2, 2, 3), i))
    return s


def golden_cases() -> dict:
    """Small fixed renders whose oracle digests are frozen in images.json."""
    from zigtrace_b200 import scenes
    return {
        "demo_24x16_8spp": (demo_scene(), kat_options()),
        "demo_24x16_8spp_seed99": (demo_scene(), kat_options(seed=99)),
        "lit_room_24x16_16spp_nonee": (lit_room(), kat_options(spp=16, max_depth=6, light_sampling=False)),
        "lit_room_24x16_16spp": (lit_room(), kat_options(spp=16, max_depth=6)),
        "glass_32x18_8spp": (glass_scene(), dict(width=32, height=18, spp=8, max_depth=16)),
        "lamps_32x18_8spp": (lamp_scene(), dict(width=32, height=18, spp=8, max_depth=12)),
        "cornell_32x32_8spp": (scenes.cornell(), dict(width=32, height=32, spp=8, max_depth=16)),
        "spheres_64x36_2spp": (scenes.random_spheres(), dict(width=64, height=36, spp=2, max_depth=50)),
    }


def fuzz_scene(seed: int) -> Scene:
    """A random scene exercising every shape, material and light kind:
    spheres (some with negative radius), triangles, quads, a plane, all four
    materials (metal with and without fuzz, glass), emissive spheres and
    quads as lights, a sky or a solid background, and a thin-lens camera."""
    rng = np.random.default_rng(10_000 + seed)
    s = Scene()
    mats = [s.add_material(Material.lambertian(rng.uniform(0.1, 0.9, 3))),
            s.add_material(Material.metal(rng.uniform(0.3, 1.0, 3), float(rng.choice([0.0, rng.uniform(0, 1)])))),
            s.add_material(Material.dielectric(float(rng.uniform(1.2, 2.0)))),
            s.add_material(Material.emissive(rng.uniform(1, 12, 3))),
            s.add_material(Material.lambertian(rng.uniform(0.1, 0.9, 3)))]
    s.add(plane((0, float(rng.uniform(-1.5, -0.5)), 0), (0, 1, 0), mats[4]))
    for _ in range(int(rng.integers(4, 12))):
        c = rng.uniform([-3, -1, -5], [3, 2, -1])
        r = float(rng.uniform(0.2, 0.8)) * (-1 if rng.random() < 0.15 else 1)
        s.add(sphere(c, r, int(rng.choice(mats))))
    for _ in range(int(rng.integers(2, 8))):
        c = rng.uniform([-3, -1, -5], [3, 2, -1])
        s.add(triangle(c, c + rng.uniform(-1, 1, 3), c + rng.uniform(-1, 1, 3), int(rng.choice(mats[:3]))))
    s.add_quad(rng.uniform([-1, 2.5, -3], [0, 3, -2]), (1.0, 0, 0), (0, 0, 1.0), mats[3])
    s.add(sphere(rng.uniform([-2, 2, -4], [2, 3, -2]), float(rng.uniform(0.1, 0.4)), mats[3]))
    s.background = Background.sky((1, 1, 1), (0.5, 0.7, 1.0)) if rng.random() < 0.5 else \
        Background.solid(rng.uniform(0, 0.2, 3))
    s.camera = CameraConfig(look_from=(float(rng.uniform(-1, 1)), 0.5, 3), look_at=(0, 0.2, -3), vfov=50,
                            aperture=float(rng.choice([0.0, 0.1])), focus_dist=5.0)
    return s
