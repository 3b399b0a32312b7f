"""ctypes wrapper of the CPU oracle (oracle/zt_oracle.c).

TEST INFRASTRUCTURE ONLY: the C restatement of the reference renderer that
the tests, the smoke check and the benchmark's CPU-baseline leg use as the
checker.  The product package never imports this module.

Scenes are described with the same structured arrays as the product's C ABI
(materials, shapes in insertion order, camera config, background), so one
description feeds both.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libzt_oracle.so"

V3 = C.c_double * 3
STATS_FIELDS = ("samples", "ext_rays", "shadow_rays", "node_pops", "slab_tests", "sphere_tests", "tri_tests",
                "plane_tests", "hits", "nee_samples", "pdfhit_calls", "pdfhit_light_tests", "rng_draws")
HIT_DTYPE = np.dtype([("t", "<f8"), ("point", "<f8", (3,)), ("normal", "<f8", (3,)), ("front_face", "<u4"),
                      ("material", "<u4"), ("prim", "<i4"), ("pad", "<i4")])
NODE_DTYPE = np.dtype([("bmin", "<f8", (3,)), ("bmax", "<f8", (3,)), ("first", "<u4"), ("count", "<u4")])
SHAPE_DTYPE = np.dtype([("kind", "<u4"), ("material", "<u4"), ("p", "<f8", (9,))])
LIGHT_DTYPE = np.dtype([("shape", SHAPE_DTYPE), ("radiance", "<f8", (3,)), ("weight", "<f8")])
CAMERA_DTYPE = np.dtype([("origin", "<f8", (3,)), ("upper_left", "<f8", (3,)), ("horizontal", "<f8", (3,)),
                         ("vertical", "<f8", (3,)), ("u", "<f8", (3,)), ("v", "<f8", (3,)),
                         ("lens_radius", "<f8")])
OPTIONS_DTYPE = np.dtype([("width", "<u8"), ("height", "<u8"), ("spp", "<u8"), ("max_depth", "<u8"),
                          ("threads", "<u8"), ("seed", "<u8"), ("tile_size", "<u8"),
                          ("light_sampling", "<u4"), ("reserved", "<u4")])

_lib = None


def build() -> Path:
    """Compiles the oracle with its Makefile if needed."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(LIB_PATH))
        _lib.ozt_scene_bounded_count.restype = C.c_size_t
        _lib.ozt_scene_plane_count.restype = C.c_size_t
        _lib.ozt_scene_node_count.restype = C.c_size_t
        _lib.ozt_scene_light_count.restype = C.c_size_t
        _lib.ozt_bvh_depth.restype = C.c_size_t
        _lib.ozt_lights_pdf_hit.restype = C.c_double
        _lib.ozt_schlick.restype = C.c_double
        _lib.ozt_schlick.argtypes = [C.c_double, C.c_double]
        _lib.ozt_tonemap.restype = C.c_double
        _lib.ozt_tonemap.argtypes = [C.c_int, C.c_double]
        _lib.ozt_encode.restype = C.c_uint8
        _lib.ozt_encode.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double]
        _lib.ozt_rng_below.restype = C.c_uint64
        _lib.ozt_rng_below.argtypes = [C.c_void_p, C.c_uint64]
        _lib.ozt_pow5.restype = C.c_double
        _lib.ozt_pow5.argtypes = [C.c_double]
        _lib.ozt_sincos.argtypes = [C.c_double, C.c_void_p, C.c_void_p]
        _lib.ozt_aabb_hit.argtypes = [C.c_void_p] * 4 + [C.c_double, C.c_double, C.c_void_p]
        _lib.ozt_scene_intersect.argtypes = [C.c_void_p] * 3 + [C.c_double, C.c_double, C.c_void_p]
        _lib.ozt_shape_intersect.argtypes = [C.c_void_p] * 3 + [C.c_double, C.c_double, C.c_void_p]
        _lib.ozt_intersect_all.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_double,
                                           C.c_double, C.c_void_p]
        _lib.ozt_trace_with.argtypes = [C.c_void_p] * 4 + [C.c_uint64, C.c_int, C.c_void_p]
        _lib.ozt_camera_init.argtypes = [C.c_void_p, C.c_double, C.c_void_p]
        _lib.ozt_camera_ray.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.ozt_rng_init.argtypes = [C.c_uint64, C.c_void_p]
        _lib.ozt_rng_for_stream.argtypes = [C.c_uint64, C.c_uint64, C.c_void_p]
        _lib.ozt_rng_next_n.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p]
        _lib.ozt_rng_float_n.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p]
        _lib.ozt_render_pixels.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                           C.c_void_p]
        _lib.ozt_scene_create.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p,
                                          C.c_int, C.c_void_p]
        for name in ("ozt_scene_free", "ozt_scene_bounded_count", "ozt_scene_plane_count", "ozt_scene_node_count",
                     "ozt_scene_light_count", "ozt_bvh_depth"):
            getattr(_lib, name).argtypes = [C.c_void_p]
        _lib.ozt_scene_nodes.argtypes = [C.c_void_p, C.c_void_p]
        _lib.ozt_scene_indices.argtypes = [C.c_void_p, C.c_void_p]
        _lib.ozt_scene_lights.argtypes = [C.c_void_p] * 4
        _lib.ozt_render.argtypes = [C.c_void_p] * 4
        _lib.ozt_render_moments.argtypes = [C.c_void_p] * 4
        _lib.ozt_render_pixels_moments.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                                   C.c_void_p]
        _lib.ozt_render_debug.argtypes = [C.c_void_p] * 4
        _lib.ozt_render_params.argtypes = [C.c_void_p] * 4
        _lib.ozt_lights_sample.argtypes = [C.c_void_p] * 7
        _lib.ozt_lights_pdf_hit.argtypes = [C.c_void_p] * 3
        _lib.ozt_material_emitted.argtypes = [C.c_void_p] * 3
        _lib.ozt_material_scatter.argtypes = [C.c_void_p] * 8
        _lib.ozt_background_radiance.argtypes = [C.c_void_p] * 3
        for name in ("ozt_rng_unit_vector", "ozt_rng_in_unit_sphere", "ozt_rng_in_unit_disk"):
            getattr(_lib, name).argtypes = [C.c_void_p, C.c_void_p]
    return _lib


def _p(a: np.ndarray) -> C.c_void_p:
    """Pointer to the array's data that keeps the array alive for the call."""
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


def v3(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, np.float64).reshape(3))


# ------------------------------------------------------------------ RNG ----
class Rng:
    """Rng state (4 x u64), src/rng.zig:10-88."""

    def __init__(self, state):
        self.s = np.ascontiguousarray(np.asarray(state, np.uint64).reshape(4))

    @staticmethod
    def init(seed: int) -> "Rng":
        s = np.zeros(4, np.uint64)
        lib().ozt_rng_init(seed, _p(s))
        return Rng(s)

    @staticmethod
    def for_stream(seed: int, stream: int) -> "Rng":
        s = np.zeros(4, np.uint64)
        lib().ozt_rng_for_stream(seed, stream, _p(s))
        return Rng(s)

    def next_n(self, n: int) -> np.ndarray:
        out = np.zeros(n, np.uint64)
        lib().ozt_rng_next_n(_p(self.s), n, _p(out))
        return out

    def float_n(self, n: int) -> np.ndarray:
        out = np.zeros(n, np.float64)
        lib().ozt_rng_float_n(_p(self.s), n, _p(out))
        return out

    def below(self, n: int) -> int:
        return int(lib().ozt_rng_below(_p(self.s), n))

    def _vec(self, fn) -> np.ndarray:
        out = np.zeros(3)
        getattr(lib(), fn)(_p(self.s), _p(out))
        return out

    def unit_vector(self):
        return self._vec("ozt_rng_unit_vector")

    def in_unit_sphere(self):
        return self._vec("ozt_rng_in_unit_sphere")

    def in_unit_disk(self):
        return self._vec("ozt_rng_in_unit_disk")


# ---------------------------------------------------------------- Scene ----
class OracleScene:
    """Scene.init/add/build (src/scene.zig:53-96) in the oracle."""

    def __init__(self, materials: np.ndarray, shapes: np.ndarray, camera: np.ndarray, background: np.ndarray,
                 build: bool = True):
        self.materials = np.ascontiguousarray(materials)
        self.shapes = np.ascontiguousarray(shapes)
        self.camera_cfg = np.ascontiguousarray(camera)
        self.background = np.ascontiguousarray(background)
        h = C.c_void_p()
        rc = lib().ozt_scene_create(_p(self.materials), len(self.materials), _p(self.shapes), len(self.shapes),
                                    _p(self.camera_cfg), _p(self.background), int(build), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"ozt_scene_create failed: {rc}")
        self.h = h

    @staticmethod
    def from_scene(scene, build: bool = True) -> "OracleScene":
        """From a zigtrace_b200.Scene (same array layouts)."""
        return OracleScene(scene.materials, scene.shapes, scene.camera.record(), scene.background.record(),
                           build)

    def __del__(self):
        if getattr(self, "h", None):
            lib().ozt_scene_free(self.h)
            self.h = None

    # -- inspection
    def counts(self):
        L = lib()
        return dict(bounded=L.ozt_scene_bounded_count(self.h), planes=L.ozt_scene_plane_count(self.h),
                    nodes=L.ozt_scene_node_count(self.h), lights=L.ozt_scene_light_count(self.h))

    def bvh(self):
        c = self.counts()
        nodes = np.zeros(c["nodes"], NODE_DTYPE)
        idx = np.zeros(c["bounded"], np.uint32)
        lib().ozt_scene_nodes(self.h, _p(nodes))
        lib().ozt_scene_indices(self.h, _p(idx))
        return nodes, idx

    def bvh_depth(self) -> int:
        return int(lib().ozt_bvh_depth(self.h))

    def lights(self):
        n = self.counts()["lights"]
        lights = np.zeros(n, LIGHT_DTYPE)
        cdf = np.zeros(n)
        total = C.c_double()
        lib().ozt_scene_lights(self.h, _p(lights), _p(cdf), C.byref(total))
        return lights, cdf, total.value

    # -- rendering
    @staticmethod
    def options(width, height, spp, max_depth, threads=1, seed=0, tile_size=16, light_sampling=True):
        o = np.zeros(1, OPTIONS_DTYPE)
        o["width"], o["height"], o["spp"], o["max_depth"] = width, height, spp, max_depth
        o["threads"], o["seed"], o["tile_size"], o["light_sampling"] = threads, seed, tile_size, int(light_sampling)
        return o

    def render(self, width, height, spp, max_depth, threads=None, seed=0, tile_size=16, light_sampling=True,
               stats: bool = False):
        threads = threads or os.cpu_count() or 1
        o = self.options(width, height, spp, max_depth, threads, seed, tile_size, light_sampling)
        out = np.zeros(width * height * 3)
        st = (C.c_uint64 * len(STATS_FIELDS))()
        rc = lib().ozt_render(self.h, _p(o), _p(out), st if stats else None)
        if rc != 0:
            raise ValueError("InvalidOptions")
        img = out.reshape(height * width, 3)
        if stats:
            return img, dict(zip(STATS_FIELDS, list(st)))
        return img

    def render_moments(self, width, height, spp, max_depth, threads=None, seed=0, light_sampling=True):
        """The image and, per pixel, the mean squared sample luminance."""
        threads = threads or os.cpu_count() or 1
        o = self.options(width, height, spp, max_depth, threads, seed, 16, light_sampling)
        out = np.zeros(width * height * 3)
        m2 = np.zeros(width * height)
        if lib().ozt_render_moments(self.h, _p(o), _p(out), _p(m2)) != 0:
            raise ValueError("InvalidOptions")
        return out.reshape(height * width, 3), m2

    def render_pixels_moments(self, width, height, spp, max_depth, pixels, threads=None, seed=0,
                              light_sampling=True):
        """render_pixels plus each listed pixel's mean squared sample luminance."""
        threads = threads or os.cpu_count() or 1
        o = self.options(width, height, spp, max_depth, threads, seed, 16, light_sampling)
        pix = np.ascontiguousarray(pixels, np.uint64)
        out = np.zeros(len(pix) * 3)
        m2 = np.zeros(len(pix))
        if lib().ozt_render_pixels_moments(self.h, _p(o), _p(pix), len(pix), _p(out), _p(m2)) != 0:
            raise ValueError("InvalidOptions")
        return out.reshape(len(pix), 3), m2

    def render_pixels(self, width, height, spp, max_depth, pixels, threads=None, seed=0, light_sampling=True,
                      stats: bool = False):
        threads = threads or os.cpu_count() or 1
        o = self.options(width, height, spp, max_depth, threads, seed, 16, light_sampling)
        pix = np.ascontiguousarray(np.asarray(pixels, np.uint64))
        out = np.zeros(len(pix) * 3)
        st = (C.c_uint64 * len(STATS_FIELDS))()
        rc = lib().ozt_render_pixels(self.h, _p(o), _p(pix), len(pix), _p(out), st if stats else None)
        if rc != 0:
            raise ValueError("InvalidOptions")
        if stats:
            return out.reshape(-1, 3), dict(zip(STATS_FIELDS, list(st)))
        return out.reshape(-1, 3)

    def render_params(self, width, height, spp, max_depth, theta, seed=0, light_sampling=True):
        """Detached-sampling forward of the differentiable form (theta: n_materials x 3)."""
        o = self.options(width, height, spp, max_depth, 1, seed, 16, light_sampling)
        th = np.ascontiguousarray(np.asarray(theta, np.float64).reshape(-1))
        out = np.zeros(width * height * 3)
        lib().ozt_render_params(self.h, _p(o), _p(th), _p(out))
        return out.reshape(-1, 3)

    def render_debug(self, width, height, max_depth, seed=0, light_sampling=True):
        o = self.options(width, height, 1, max_depth, 1, seed, 16, light_sampling)
        fp = np.zeros(width * height, np.int32)
        pl = np.zeros(width * height, np.uint32)
        lib().ozt_render_debug(self.h, _p(o), _p(fp), _p(pl))
        return fp, pl

    def trace_with(self, origin, direction, rng: Rng, max_depth: int, light_sampling: bool = True):
        out = np.zeros(3)
        lib().ozt_trace_with(self.h, _p(v3(origin)), _p(v3(direction)), _p(rng.s), max_depth, int(light_sampling),
                             _p(out))
        return out

    def intersect(self, origin, direction, tmin, tmax) -> Optional[np.void]:
        h = np.zeros(1, HIT_DTYPE)
        ok = lib().ozt_scene_intersect(self.h, _p(v3(origin)), _p(v3(direction)), tmin, tmax, _p(h))
        return h[0] if ok else None

    def lights_sample(self, origin, rng: Rng):
        d, r = np.zeros(3), np.zeros(3)
        dist, pdf = C.c_double(), C.c_double()
        ok = lib().ozt_lights_sample(self.h, _p(v3(origin)), _p(rng.s), _p(d), C.byref(dist), _p(r), C.byref(pdf))
        if not ok:
            return None
        return dict(dir=d, distance=dist.value, radiance=r, pdf=pdf.value)

    def pdf_hit(self, origin, hit: np.void) -> float:
        h = np.array([hit], HIT_DTYPE)
        return float(lib().ozt_lights_pdf_hit(self.h, _p(v3(origin)), _p(h)))


# -------------------------------------------------------- free functions ----
def shape_intersect(shape: np.void, origin, direction, tmin, tmax):
    s = np.array([shape], SHAPE_DTYPE)
    h = np.zeros(1, HIT_DTYPE)
    ok = lib().ozt_shape_intersect(_p(s), _p(v3(origin)), _p(v3(direction)), tmin, tmax, _p(h))
    return h[0] if ok else None


def intersect_all(shapes: np.ndarray, origin, direction, tmin, tmax):
    s = np.ascontiguousarray(shapes, SHAPE_DTYPE)
    h = np.zeros(1, HIT_DTYPE)
    ok = lib().ozt_intersect_all(_p(s), len(s), _p(v3(origin)), _p(v3(direction)), tmin, tmax, _p(h))
    return h[0] if ok else None


def material_scatter(material: np.void, in_dir, hit: np.void, rng: Rng):
    m = np.array([material])
    h = np.array([hit], HIT_DTYPE)
    att, o, d = np.zeros(3), np.zeros(3), np.zeros(3)
    ok = lib().ozt_material_scatter(_p(m), _p(np.zeros(3)), _p(v3(in_dir)), _p(h), _p(rng.s), _p(att), _p(o), _p(d))
    return (att, o, d) if ok else None


def material_emitted(material: np.void, hit: np.void):
    m = np.array([material])
    h = np.array([hit], HIT_DTYPE)
    out = np.zeros(3)
    lib().ozt_material_emitted(_p(m), _p(h), _p(out))
    return out


def make_hit(t=1.0, point=(0, 0, 0), normal=(0, 1, 0), front_face=True, material=0) -> np.void:
    h = np.zeros(1, HIT_DTYPE)
    h["t"], h["point"], h["normal"], h["front_face"], h["material"] = t, point, normal, int(front_face), material
    return h[0]


def schlick(cosine: float, eta: float) -> float:
    return float(lib().ozt_schlick(cosine, eta))


def camera_init(camera_cfg: np.ndarray, aspect: float) -> np.ndarray:
    out = np.zeros(1, CAMERA_DTYPE)
    lib().ozt_camera_init(_p(np.ascontiguousarray(camera_cfg)), aspect, _p(out))
    return out[0]


def camera_ray(cam: np.void, s: float, t: float, rng: Rng):
    c = np.array([cam], CAMERA_DTYPE)
    o, d = np.zeros(3), np.zeros(3)
    lib().ozt_camera_ray(_p(c), s, t, _p(rng.s), _p(o), _p(d))
    return o, d


def background_radiance(background: np.ndarray, direction) -> np.ndarray:
    out = np.zeros(3)
    lib().ozt_background_radiance(_p(np.ascontiguousarray(background)), _p(v3(direction)), _p(out))
    return out


def aabb_hit(bmin, bmax, origin, direction, tmin, tmax):
    t = C.c_double()
    ok = lib().ozt_aabb_hit(_p(v3(bmin)), _p(v3(bmax)), _p(v3(origin)), _p(v3(direction)), tmin, tmax, C.byref(t))
    return t.value if ok else None


def tonemap(kind: int, c: float) -> float:
    return float(lib().ozt_tonemap(kind, c))


def encode(kind: int, gamma: float, exposure: float, linear: float) -> int:
    return int(lib().ozt_encode(kind, gamma, exposure, linear))


def sincos(x: float):
    s, c = C.c_double(), C.c_double()
    lib().ozt_sincos(x, C.byref(s), C.byref(c))
    return s.value, c.value


def pow5(x: float) -> float:
    return float(lib().ozt_pow5(x))
