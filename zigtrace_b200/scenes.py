"""Seeded synthetic workloads, built through the public Scene API.

No public benchmark suite or dataset is involved: each workload is generated
procedurally from a fixed seed, with the shapes, sizes and value
distributions of the configurations the renderer is measured on.

- ``cornell``: the Cornell box of examples/cornell.txt (five Lambertian
  walls, a 130x105 one-sided ceiling light of radiance 15, a glass sphere
  r=90 and a metal sphere with fuzz 0), black background; 256x256, 64 spp,
  depth 16.
- ``random_spheres``: ground plane, three r=1 spheres and about 320 r=0.2
  spheres on a jittered 18x18 grid over [-11, 11]^2 (80% Lambertian with
  albedo U*U, 15% metal albedo U(0.5,1) fuzz U(0,0.5), 5% glass), sky
  background, thin lens (aperture 0.1, focus 10); 1280x720, 16 spp, depth 50.
- ``triangle_heavy``: a 1000x500-cell heightfield (2 triangles per cell,
  fBm heights) plus 20 icospheres at subdivision 3, Lambertian/metal mix,
  64 small emissive quads of radiance U(5,20), black background;
  1920x1080, 64 spp, depth 16.
"""
from __future__ import annotations

import math
from typing import Tuple

import numpy as np

from .api import Background, CameraConfig, Material, Options, Scene, plane, sphere


# ------------------------------------------------------------- Cornell ----
def cornell(metal_fuzz: float = 0.0) -> Scene:
    """Cornell box, geometry of examples/cornell.txt:15-23."""
    s = Scene()
    s.background = Background.solid((0.0, 0.0, 0.0))
    red = s.add_material(Material.lambertian((0.65, 0.05, 0.05)))
    green = s.add_material(Material.lambertian((0.12, 0.45, 0.15)))
    white = s.add_material(Material.lambertian((0.73, 0.73, 0.73)))
    light = s.add_material(Material.emissive((15.0, 15.0, 15.0)))
    glass = s.add_material(Material.dielectric(1.5))
    steel = s.add_material(Material.metal((0.85, 0.85, 0.88), metal_fuzz))
    s.add_quad((555, 0, 0), (0, 555, 0), (0, 0, 555), red)
    s.add_quad((0, 0, 0), (0, 555, 0), (0, 0, 555), green)
    s.add_quad((343, 554, 332), (-130, 0, 0), (0, 0, -105), light)  # faces down
    s.add_quad((0, 0, 0), (555, 0, 0), (0, 0, 555), white)  # floor
    s.add_quad((555, 555, 555), (-555, 0, 0), (0, 0, -555), white)  # ceiling
    s.add_quad((0, 0, 555), (555, 0, 0), (0, 555, 0), white)  # back wall
    s.add(sphere((190, 90, 190), 90, glass))
    s.add(sphere((380, 120, 360), 120, steel))
    s.camera = CameraConfig(look_from=(278, 278, -800), look_at=(278, 278, 0), vfov=40)
    return s


CORNELL_OPTIONS = Options(width=256, height=256, spp=64, max_depth=16, seed=0)


# ------------------------------------------------------ random spheres ----
def random_spheres(seed: int = 0, grid: int = 18, extent: float = 11.0) -> Scene:
    """Ground plane + 3 big spheres + jittered grid of r=0.2 spheres."""
    rng = np.random.default_rng(seed)
    s = Scene()
    s.background = Background.sky((1.0, 1.0, 1.0), (0.5, 0.7, 1.0))
    ground = s.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    s.add(plane((0.0, 0.0, 0.0), (0.0, 1.0, 0.0), ground))
    glass = s.add_material(Material.dielectric(1.5))
    brown = s.add_material(Material.lambertian((0.4, 0.2, 0.1)))
    polished = s.add_material(Material.metal((0.7, 0.6, 0.5), 0.0))
    big = [((0.0, 1.0, 0.0), glass), ((-4.0, 1.0, 0.0), brown), ((4.0, 1.0, 0.0), polished)]
    for c, m in big:
        s.add(sphere(c, 1.0, m))
    cell = 2.0 * extent / grid
    for i in range(grid):
        for j in range(grid):
            jx, jz, choose = rng.random(), rng.random(), rng.random()
            cx = -extent + (i + 0.05 + 0.9 * jx) * cell
            cz = -extent + (j + 0.05 + 0.9 * jz) * cell
            if any(math.hypot(cx - c[0], cz - c[2]) < 1.2 for c, _ in big):
                continue
            if choose < 0.8:
                albedo = tuple(float(a) for a in rng.random(3) * rng.random(3))
                m = s.add_material(Material.lambertian(albedo))
            elif choose < 0.95:
                albedo = tuple(float(a) for a in rng.uniform(0.5, 1.0, 3))
                m = s.add_material(Material.metal(albedo, float(rng.uniform(0.0, 0.5))))
            else:
                m = glass
            s.add(sphere((cx, 0.2, cz), 0.2, m))
    s.camera = CameraConfig(look_from=(13, 2, 3), look_at=(0, 0, 0), vfov=20, aperture=0.1, focus_dist=10.0)
    return s


SPHERES_OPTIONS = Options(width=1280, height=720, spp=16, max_depth=50, seed=0)


# ------------------------------------------------------ triangle heavy ----
def _value_noise(x: np.ndarray, z: np.ndarray, rng: np.random.Generator, freq: float) -> np.ndarray:
    """Smoothly interpolated lattice noise in [-1, 1]."""
    n = int(math.ceil(freq)) + 2
    lattice = rng.uniform(-1.0, 1.0, (n + 1, n + 1))
    gx, gz = x * freq, z * freq
    ix, iz = np.floor(gx).astype(np.int64), np.floor(gz).astype(np.int64)
    fx, fz = gx - ix, gz - iz
    sx, sz = fx * fx * (3 - 2 * fx), fz * fz * (3 - 2 * fz)
    ix %= n
    iz %= n
    a = lattice[ix, iz] * (1 - sx) + lattice[ix + 1, iz] * sx
    b = lattice[ix, iz + 1] * (1 - sx) + lattice[ix + 1, iz + 1] * sx
    return a * (1 - sz) + b * sz


def heightfield(nx: int, nz: int, size_x: float, size_z: float, seed: int, octaves: int = 6,
                amplitude: float = 3.0) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(nx+1)x(nz+1) vertex grid with fBm heights; returns triangle corner
    arrays v0, v1, v2 (2 per cell, front face up)."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(-size_x / 2, size_x / 2, nx + 1)
    zs = np.linspace(-size_z / 2, size_z / 2, nz + 1)
    X, Z = np.meshgrid(xs, zs, indexing="ij")
    u, v = (X - xs[0]) / size_x, (Z - zs[0]) / size_z
    H = np.zeros_like(X)
    amp, freq = amplitude, 4.0
    for _ in range(octaves):
        H += amp * _value_noise(u, v, rng, freq)
        amp *= 0.5
        freq *= 2.0
    P = np.stack([X, H, Z], axis=-1)
    p00, p10 = P[:-1, :-1].reshape(-1, 3), P[1:, :-1].reshape(-1, 3)
    p01, p11 = P[:-1, 1:].reshape(-1, 3), P[1:, 1:].reshape(-1, 3)
    v0 = np.concatenate([p00, p00])
    v1 = np.concatenate([p01, p11])
    v2 = np.concatenate([p11, p10])
    return v0, v1, v2, H


def icosphere(subdivisions: int) -> Tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: (vertices, faces) with outward (counter-clockwise)
    winding; 20 * 4^subdivisions faces."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [tuple(c / math.sqrt(1 + t * t) for c in v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache = {}
        new_faces = []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = np.add(verts[a], verts[b]) / 2.0
                m = m / np.linalg.norm(m)
                verts.append(tuple(m))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            new_faces += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = new_faces
    return np.array(verts, np.float64), np.array(faces, np.int64)


def triangle_heavy(seed: int = 0, nx: int = 1000, nz: int = 500, n_ico: int = 20, ico_subdiv: int = 3,
                   n_lights: int = 64) -> Scene:
    """Heightfield + icospheres + small emissive quads, black background."""
    rng = np.random.default_rng(seed + 1000)
    size_x, size_z = 100.0, 50.0
    s = Scene()
    s.background = Background.solid((0.0, 0.0, 0.0))
    terrain = s.add_material(Material.lambertian((0.45, 0.5, 0.4)))
    v0, v1, v2, H = heightfield(nx, nz, size_x, size_z, seed)
    s.add_triangles(v0, v1, v2, terrain)

    def height_at(x, z):
        i = int(round((x + size_x / 2) / size_x * nx))
        j = int(round((z + size_z / 2) / size_z * nz))
        return float(H[min(max(i, 0), nx), min(max(j, 0), nz)])

    verts, faces = icosphere(ico_subdiv)
    for k in range(n_ico):
        cx, cz = rng.uniform(-0.4 * size_x, 0.4 * size_x), rng.uniform(-0.4 * size_z, 0.4 * size_z)
        r = rng.uniform(1.0, 3.0)
        cy = height_at(cx, cz) + r * 0.8
        if rng.random() < 0.5:
            m = s.add_material(Material.lambertian(tuple(float(a) for a in rng.uniform(0.2, 0.9, 3))))
        else:
            m = s.add_material(Material.metal(tuple(float(a) for a in rng.uniform(0.5, 1.0, 3)),
                                              float(rng.uniform(0.0, 0.3))))
        P = verts * r + np.array([cx, cy, cz])
        s.add_triangles(P[faces[:, 0]], P[faces[:, 1]], P[faces[:, 2]], m)
    for k in range(n_lights):
        cx, cz = rng.uniform(-0.45 * size_x, 0.45 * size_x), rng.uniform(-0.45 * size_z, 0.45 * size_z)
        y = height_at(cx, cz) + rng.uniform(4.0, 8.0)
        m = s.add_material(Material.emissive(tuple([float(rng.uniform(5.0, 20.0))] * 3)))
        w = rng.uniform(0.6, 1.5)
        # corner, u, v with u x v pointing down (-y): faces the terrain
        s.add_quad((cx - w / 2, y, cz - w / 2), (w, 0, 0), (0, 0, w), m)
    s.camera = CameraConfig(look_from=(0.0, 22.0, 48.0), look_at=(0.0, 0.0, 0.0), vfov=55)
    return s


TRIANGLE_HEAVY_OPTIONS = Options(width=1920, height=1080, spp=64, max_depth=16, seed=0)


# ----------------------------------------------------- differentiable form ----
def cornell_diff(seed: int = 0, perturb: float = 0.2):
    """Cornell-style box for the differentiable form: 32 Lambertian materials
    (floor and back wall 3x3 patches, side walls and ceiling 2x2, two
    spheres) with albedos U(0.1, 0.9) and 4 emissive quads under the ceiling
    with radiance U(2, 20) per channel.  Returns (scene, target_colors): the
    target is every colour scaled by U(1 - perturb, 1 + perturb)."""
    rng = np.random.default_rng(seed + 500)
    s = Scene()
    s.background = Background.solid((0.0, 0.0, 0.0))
    ids = iter(range(32))
    for _ in range(32):
        s.add_material(Material.lambertian(tuple(float(a) for a in rng.uniform(0.1, 0.9, 3))))
    L = 555.0

    def patches(origin, u, v, nu, nv):
        for a in range(nu):
            for b in range(nv):
                corner = [origin[k] + u[k] * a / nu + v[k] * b / nv for k in range(3)]
                s.add_quad(corner, [c / nu for c in u], [c / nv for c in v], next(ids))

    patches((0, 0, 0), (L, 0, 0), (0, 0, L), 3, 3)      # floor
    patches((0, 0, L), (L, 0, 0), (0, L, 0), 3, 3)      # back wall
    patches((L, 0, 0), (0, L, 0), (0, 0, L), 2, 2)      # x = 555 wall
    patches((0, 0, 0), (0, L, 0), (0, 0, L), 2, 2)      # x = 0 wall
    patches((0, L, 0), (L, 0, 0), (0, 0, L), 2, 2)      # ceiling
    s.add(sphere((185.0, 100.0, 200.0), 100.0, next(ids)))
    s.add(sphere((380.0, 80.0, 380.0), 80.0, next(ids)))
    for cx, cz in ((160.0, 160.0), (395.0, 160.0), (160.0, 395.0), (395.0, 395.0)):
        m = s.add_material(Material.emissive(tuple(float(a) for a in rng.uniform(2.0, 20.0, 3))))
        s.add_quad((cx - 50.0, 554.0, cz - 40.0), (100.0, 0.0, 0.0), (0.0, 0.0, 80.0), m)  # faces down
    s.camera = CameraConfig(look_from=(278, 278, -800), look_at=(278, 278, 0), vfov=40)
    colors = np.array([m["color"] for m in s.materials])
    target = colors * rng.uniform(1.0 - perturb, 1.0 + perturb, colors.shape)
    return s, target


DIFF_OPTIONS = Options(width=512, height=512, spp=64, max_depth=16, seed=0)


# --------------------------------------------------------- batched form ----
def sphere_field(seed: int, n: int) -> Scene:
    """Ground plane + exactly n r=0.2 spheres on a jittered grid sized to n
    (spacing as in random_spheres), 80/15/5 Lambertian/metal/glass, sky
    background, thin-lens camera framing the field."""
    from .api import LAMBERTIAN, METAL, DIELECTRIC
    from . import _native as N
    rng = np.random.default_rng(seed)
    g = int(math.ceil(math.sqrt(n)))
    cell = 22.0 / 18.0
    extent = g * cell / 2.0
    cells = rng.permutation(g * g)[:n]
    i, j = cells // g, cells % g
    cx = -extent + (i + 0.05 + 0.9 * rng.random(n)) * cell
    cz = -extent + (j + 0.05 + 0.9 * rng.random(n)) * cell
    choose = rng.random(n)
    s = Scene()
    s.background = Background.sky((1.0, 1.0, 1.0), (0.5, 0.7, 1.0))
    ground = s.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    s.add(plane((0.0, 0.0, 0.0), (0.0, 1.0, 0.0), ground))
    mats = np.zeros(n, N.MATERIAL_DTYPE)
    lam, met = choose < 0.8, (choose >= 0.8) & (choose < 0.95)
    gl = ~(lam | met)
    mats["kind"] = np.where(lam, LAMBERTIAN, np.where(met, METAL, DIELECTRIC))
    mats["color"][lam] = rng.random((int(lam.sum()), 3)) * rng.random((int(lam.sum()), 3))
    mats["color"][met] = rng.uniform(0.5, 1.0, (int(met.sum()), 3))
    mats["param"][met] = rng.uniform(0.0, 0.5, int(met.sum()))
    mats["param"][gl] = 1.5
    first = s.add_materials(mats)
    s.add_spheres(np.stack([cx, np.full(n, 0.2), cz], axis=1), np.full(n, 0.2), first + np.arange(n))
    k = max(extent / 11.0, 0.25)
    s.camera = CameraConfig(look_from=(13 * k, 2 * k, 3 * k), look_at=(0, 0, 0), vfov=20, aperture=0.1 * k,
                            focus_dist=10.0 * k)
    return s


BATCH_RESOLUTIONS = ((64, 64), (128, 128), (256, 256), (512, 288))


def batch_workload(count: int = 256, seed: int = 0, spp: int = 16, max_depth: int = 16):
    """The batched form's renders: scene k is a sphere field from its own
    seed with a sphere count log-uniform in [16, 20000] and a resolution drawn
    from BATCH_RESOLUTIONS; returns [(scene, Options)]."""
    rng = np.random.default_rng(seed + 77)
    out = []
    for k in range(count):
        n = int(math.floor(math.exp(rng.uniform(math.log(16), math.log(20000)))))
        w, h = BATCH_RESOLUTIONS[int(rng.integers(len(BATCH_RESOLUTIONS)))]
        out.append((sphere_field(seed + k, n), Options(width=w, height=h, spp=spp, max_depth=max_depth, seed=0)))
    return out

WORKLOADS = {
    "cornell": (cornell, CORNELL_OPTIONS),
    "random_spheres": (random_spheres, SPHERES_OPTIONS),
    "triangle_heavy": (triangle_heavy, TRIANGLE_HEAVY_OPTIONS),
}
