"""Host-side mirror of zigtrace's library API (src/root.zig:2-17).

Names and argument meanings follow the reference: ``Scene`` with
``add_material`` / ``add`` / ``add_quad`` / ``build`` (src/scene.zig:53-96),
``Options`` (src/render.zig:12-23), ``render(scene, options) -> Image``
(src/render.zig:152), ``Image.to_rgb8(Output)`` (src/image.zig:65-73) and
``write_ppm`` (src/image.zig:77-81).  Rendering runs on the GPU through the
C ABI; errors surface as ``ZigtraceError`` whose ``name`` is the reference's
Zig error name (``InvalidOptions``, ``OutOfMemory``, ...).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _native as N
from ._native import ZigtraceError

Vec = Sequence[float]

LAMBERTIAN, METAL, DIELECTRIC, EMISSIVE = 0, 1, 2, 3
SPHERE, TRIANGLE, PLANE = 0, 1, 2
MODE_AUTO, MODE_MEGAKERNEL, MODE_WAVEFRONT, MODE_MEGAKERNEL_REGEN, MODE_WAVEFRONT_SORTED = 0, 1, 2, 3, 4
PRECISION_EXACT, PRECISION_FAST = 0, 1


# ---------------------------------------------------------------- Material --
class Material:
    """Material union, src/material.zig:15-24."""

    @staticmethod
    def _rec(kind: int, color: Vec, param: float) -> np.void:
        r = np.zeros((), N.MATERIAL_DTYPE)
        r["kind"] = kind
        r["color"] = color
        r["param"] = param
        return r

    @staticmethod
    def lambertian(albedo: Vec) -> np.void:
        return Material._rec(LAMBERTIAN, albedo, 0.0)

    @staticmethod
    def metal(albedo: Vec, fuzz: float = 0.0) -> np.void:
        return Material._rec(METAL, albedo, fuzz)

    @staticmethod
    def dielectric(ior: float) -> np.void:
        return Material._rec(DIELECTRIC, (0.0, 0.0, 0.0), ior)

    @staticmethod
    def emissive(color: Vec) -> np.void:
        return Material._rec(EMISSIVE, color, 0.0)


# ------------------------------------------------------------------- Shape --
def sphere(center: Vec, radius: float, material: int) -> np.void:
    """Sphere, src/geometry.zig:32-58 (negative radius = inward normals)."""
    r = np.zeros((), N.SHAPE_DTYPE)
    r["kind"], r["material"] = SPHERE, material
    r["p"][:4] = (*center, radius)
    return r


def triangle(v0: Vec, v1: Vec, v2: Vec, material: int) -> np.void:
    """Triangle, src/geometry.zig:76-104."""
    r = np.zeros((), N.SHAPE_DTYPE)
    r["kind"], r["material"] = TRIANGLE, material
    r["p"][:] = (*v0, *v1, *v2)
    return r


def plane(point: Vec, normal: Vec, material: int) -> np.void:
    """Infinite plane with unit normal, src/geometry.zig:60-74."""
    r = np.zeros((), N.SHAPE_DTYPE)
    r["kind"], r["material"] = PLANE, material
    r["p"][:6] = (*point, *normal)
    return r


# ------------------------------------------------------------ Scene parts --
@dataclass
class CameraConfig:
    """CameraConfig, src/camera.zig:8-18."""
    look_from: Vec = (0.0, 0.0, 0.0)
    look_at: Vec = (0.0, 0.0, -1.0)
    up: Vec = (0.0, 1.0, 0.0)
    vfov: float = 60.0
    aperture: float = 0.0
    focus_dist: Optional[float] = None

    def record(self) -> np.ndarray:
        r = np.zeros(1, N.CAMERA_DTYPE)
        r["look_from"], r["look_at"], r["up"] = self.look_from, self.look_at, self.up
        r["vfov"], r["aperture"] = self.vfov, self.aperture
        if self.focus_dist is not None:
            r["focus_dist"], r["has_focus_dist"] = self.focus_dist, 1
        return r


@dataclass
class Background:
    """Background union, src/scene.zig:15-28."""
    kind: int = 1
    a: Vec = (1.0, 1.0, 1.0)
    b: Vec = (0.5, 0.7, 1.0)

    @staticmethod
    def solid(color: Vec) -> "Background":
        return Background(0, tuple(color), (0.0, 0.0, 0.0))

    @staticmethod
    def sky(horizon: Vec, zenith: Vec) -> "Background":
        return Background(1, tuple(horizon), tuple(zenith))

    def record(self) -> np.ndarray:
        r = np.zeros(1, N.BACKGROUND_DTYPE)
        r["kind"], r["a"], r["b"] = self.kind, self.a, self.b
        return r


@dataclass
class Settings:
    """Scene render settings, src/scene.zig:30-37."""
    width: int = 400
    height: int = 225
    spp: int = 32
    max_depth: int = 16


@dataclass
class Options:
    """render.Options, src/render.zig:12-23."""
    width: int
    height: int
    spp: int
    max_depth: int
    threads: int = 1
    seed: int = 0
    tile_size: int = 16
    light_sampling: bool = True

    def record(self) -> np.ndarray:
        r = np.zeros(1, N.OPTIONS_DTYPE)
        for k in ("width", "height", "spp", "max_depth", "threads", "seed", "tile_size"):
            v = int(getattr(self, k))
            if v < 0:
                raise ZigtraceError(-1, f"{k} must be non-negative")
            r[k] = v
        r["light_sampling"] = 1 if self.light_sampling else 0
        return r


@dataclass
class GpuConfig:
    """Device execution choices (zt_gpu_config); zeros mean defaults.
    ``precision``: PRECISION_EXACT (bit-identical to the CPU oracle's restatement of the reference
    algorithm) or PRECISION_FAST (single-precision conservative BVH boxes,
    f64 everything else)."""
    mode: int = MODE_AUTO
    block_size: int = 0
    queue_capacity: int = 0
    precision: int = 0

    def record(self) -> np.ndarray:
        r = np.zeros(1, N.GPU_CONFIG_DTYPE)
        r["mode"], r["block_size"], r["queue_capacity"] = self.mode, self.block_size, self.queue_capacity
        r["precision"] = self.precision
        return r


# ------------------------------------------------------------------- Scene --
class Scene:
    """Scene container, src/scene.zig:40-121.

    Shapes are kept in insertion order as a structured array (the layout of
    ``zt_shape``); ``build`` hands them to the native library, which routes
    planes outside the BVH, builds the binned-SAH BVH and the emitter table on
    the host exactly as the reference does.
    """

    def __init__(self) -> None:
        self._mats: list = []
        self._chunks: list = []
        self._n_shapes = 0
        self.camera = CameraConfig()
        self.background = Background()
        self.settings = Settings()
        self._handle: Optional[C.c_void_p] = None

    # -- construction (scene.zig:57-88)
    def add_material(self, m: np.void) -> int:
        self._mats.append(np.array(m, N.MATERIAL_DTYPE))
        self._invalidate()
        return len(self._mats) - 1

    def add_materials(self, mats: np.ndarray) -> int:
        """Vectorised Scene.addMaterial; returns the id of the first one."""
        first = len(self._mats)
        self._mats.extend(np.ascontiguousarray(mats, N.MATERIAL_DTYPE).reshape(-1))
        self._invalidate()
        return first

    def add(self, shape: np.void) -> None:
        self.add_shapes(np.array([shape], N.SHAPE_DTYPE))

    def add_shapes(self, shapes: np.ndarray) -> None:
        shapes = np.ascontiguousarray(shapes, N.SHAPE_DTYPE)
        if len(shapes):
            self._chunks.append(shapes)
            self._n_shapes += len(shapes)
        self._invalidate()

    def add_quad(self, corner: Vec, u: Vec, v: Vec, material: int) -> None:
        """Two triangles corner+a*u+b*v, front face on the u x v side
        (scene.zig:82-88)."""
        c = [float(x) for x in corner]
        u = [float(x) for x in u]
        v = [float(x) for x in v]
        p1 = [c[i] + u[i] for i in range(3)]
        p2 = [(c[i] + u[i]) + v[i] for i in range(3)]
        p3 = [c[i] + v[i] for i in range(3)]
        self.add_shapes(np.array([triangle(c, p1, p2, material), triangle(c, p2, p3, material)], N.SHAPE_DTYPE))

    def add_triangles(self, v0: np.ndarray, v1: np.ndarray, v2: np.ndarray, material) -> None:
        """Vectorised Scene.add of many triangles (rows of v0/v1/v2)."""
        n = len(v0)
        a = np.zeros(n, N.SHAPE_DTYPE)
        a["kind"] = TRIANGLE
        a["material"] = material
        a["p"][:, 0:3], a["p"][:, 3:6], a["p"][:, 6:9] = v0, v1, v2
        self.add_shapes(a)

    def add_spheres(self, centers: np.ndarray, radii: np.ndarray, materials) -> None:
        n = len(centers)
        a = np.zeros(n, N.SHAPE_DTYPE)
        a["kind"] = SPHERE
        a["material"] = materials
        a["p"][:, 0:3] = centers
        a["p"][:, 3] = radii
        self.add_shapes(a)

    # -- arrays in the C-ABI layout
    @property
    def materials(self) -> np.ndarray:
        return np.array(self._mats, N.MATERIAL_DTYPE).reshape(-1)

    @property
    def shapes(self) -> np.ndarray:
        if not self._chunks:
            return np.zeros(0, N.SHAPE_DTYPE)
        if len(self._chunks) > 1:
            self._chunks = [np.concatenate(self._chunks)]
        return self._chunks[0]

    def primitive_count(self) -> int:
        return self._n_shapes

    # -- build (scene.zig:90-96)
    def build(self, device: bool = False) -> "Scene":
        """Scene.build.  device=True builds the BVH on the current CUDA
        device (the same tree; see zt_scene_build_device); ``built_on_device``
        and ``build_ms`` then report what happened."""
        lib = N.lib()
        self._invalidate()
        h = C.c_void_p()
        N.check(lib.zt_scene_create(C.byref(h)))
        self._handle = h
        mats = self.materials
        if len(mats):
            N.check(lib.zt_scene_add_materials(h, N.ptr(mats), len(mats), None))
        shapes = self.shapes
        if len(shapes):
            N.check(lib.zt_scene_add_shapes(h, N.ptr(shapes), len(shapes)))
        N.check(lib.zt_scene_set_camera(h, N.ptr(self.camera.record())))
        N.check(lib.zt_scene_set_background(h, N.ptr(self.background.record())))
        self.built_on_device, self.build_ms = False, None
        if device:
            used, ms = C.c_uint32(), C.c_double()
            N.check(lib.zt_scene_build_device(h, C.byref(used), C.byref(ms)))
            self.built_on_device = bool(used.value)
            self.build_ms = ms.value if used.value else None
        else:
            N.check(lib.zt_scene_build(h))
        return self

    def build_with_bvh(self, nodes: np.ndarray, indices: np.ndarray) -> "Scene":
        """Scene.build with a BVH built elsewhere -- the reference's own
        ``Bvh.build`` output (``nodes`` in the zt_bvh_node layout, ``indices``
        the shape permutation) -- used as given (zt_scene_set_bvh)."""
        lib = N.lib()
        self._invalidate()
        h = C.c_void_p()
        N.check(lib.zt_scene_create(C.byref(h)))
        self._handle = h
        mats = self.materials
        if len(mats):
            N.check(lib.zt_scene_add_materials(h, N.ptr(mats), len(mats), None))
        shapes = self.shapes
        if len(shapes):
            N.check(lib.zt_scene_add_shapes(h, N.ptr(shapes), len(shapes)))
        N.check(lib.zt_scene_set_camera(h, N.ptr(self.camera.record())))
        N.check(lib.zt_scene_set_background(h, N.ptr(self.background.record())))
        nodes = np.ascontiguousarray(nodes, N.BVH_NODE_DTYPE)
        indices = np.ascontiguousarray(indices, np.uint32)
        self.built_on_device, self.build_ms = False, None
        N.check(lib.zt_scene_set_bvh(h, N.ptr(nodes) if len(nodes) else None, len(nodes),
                                     N.ptr(indices) if len(indices) else None, len(indices)))
        return self

    @property
    def handle(self) -> C.c_void_p:
        if self._handle is None:
            raise ZigtraceError(-8, "scene is not built: call Scene.build() first")
        # camera/background may be edited after build: push the current ones
        lib = N.lib()
        N.check(lib.zt_scene_set_camera(self._handle, N.ptr(self.camera.record())))
        N.check(lib.zt_scene_set_background(self._handle, N.ptr(self.background.record())))
        return self._handle

    def _invalidate(self) -> None:
        if self._handle is not None:
            N.lib().zt_scene_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self._invalidate()
        except Exception:
            pass

    # -- inspection
    def counts(self) -> dict:
        vals = [C.c_uint64() for _ in range(5)]
        N.check(N.lib().zt_scene_counts(self.handle, *[C.byref(v) for v in vals]))
        return dict(zip(("materials", "bounded", "planes", "nodes", "lights"), (v.value for v in vals)))

    def bvh(self):
        c = self.counts()
        nodes = np.zeros(c["nodes"], N.BVH_NODE_DTYPE)
        idx = np.zeros(c["bounded"], np.uint32)
        N.check(N.lib().zt_scene_bvh(self.handle, N.ptr(nodes), N.ptr(idx)))
        return nodes, idx

    def bvh_depth(self) -> int:
        d = C.c_uint64()
        N.check(N.lib().zt_scene_bvh_depth(self.handle, C.byref(d)))
        return d.value

    def lights(self):
        c = self.counts()
        lights = np.zeros(c["lights"], N.LIGHT_DTYPE)
        cdf = np.zeros(c["lights"], np.float64)
        total = C.c_double()
        N.check(N.lib().zt_scene_lights(self.handle, N.ptr(lights), N.ptr(cdf), C.byref(total)))
        return lights, cdf, total.value

    def upload(self) -> None:
        N.check(N.lib().zt_scene_upload(self.handle))

    def release_device(self) -> None:
        if self._handle is not None:
            N.check(N.lib().zt_scene_release_device(self._handle))

    def set_primal_cache_limit(self, max_bytes: int) -> None:
        """Largest per-sample primal cache ``forward`` may keep for
        ``backward`` (0 keeps none; the backward then traces the primal)."""
        N.check(N.lib().zt_scene_set_primal_cache_limit(self.handle, int(max_bytes)))

    def staging_bytes(self) -> int:
        """Bytes one upload copies host-to-device (from pinned memory)."""
        b = C.c_uint64()
        N.check(N.lib().zt_scene_upload_bytes(self.handle, C.byref(b)))
        return b.value


# ------------------------------------------------------------------- Image --
TONEMAPS = {"none": 0, "reinhard": 1, "aces": 2}


@dataclass
class Output:
    """Output, src/image.zig:24-38."""
    tonemap: str = "none"
    gamma: float = 2.2
    exposure: float = 1.0


@dataclass
class Image:
    """HDR framebuffer, src/image.zig:40-74: ``pixels[y*width + x]`` RGB f64."""
    width: int
    height: int
    pixels: np.ndarray = field(repr=False)

    def get(self, x: int, y: int) -> np.ndarray:
        return self.pixels[y * self.width + x]

    def to_rgb8(self, out: Output = Output()) -> np.ndarray:
        px = np.ascontiguousarray(self.pixels, np.float64)
        rgb = np.zeros(self.width * self.height * 3, np.uint8)
        N.check(N.lib().zt_image_to_rgb8(N.ptr(px), self.width * self.height, TONEMAPS[out.tonemap],
                                         out.gamma, out.exposure, N.ptr(rgb)))
        return rgb


def png_size(width: int, height: int) -> int:
    """Bytes of the PNG file png.writePng writes (src/png.zig:10-58)."""
    n = C.c_uint64()
    N.check(N.lib().zt_png_size(width, height, C.byref(n)))
    return n.value


def encode_png(rgb: np.ndarray, width: int, height: int) -> bytes:
    """png.writePng (src/png.zig:10-58) on the host: 8-bit RGB, no filtering,
    stored DEFLATE blocks."""
    n = png_size(width, height)
    src = np.ascontiguousarray(np.asarray(rgb, np.uint8).reshape(-1))
    if src.size != width * height * 3:
        raise ZigtraceError(-5, "rgb must hold width*height*3 bytes")
    out = np.zeros(n, np.uint8)
    N.check(N.lib().zt_png_encode(N.ptr(src), width, height, N.ptr(out), n))
    return out.tobytes()


def write_png(f, width: int, height: int, rgb: np.ndarray) -> None:
    """png.writePng to a binary file object."""
    f.write(encode_png(rgb, width, height))


def image_to_rgb8_device(d_pixels: int, n_pixels: int, d_rgb_out: int, out: Output = Output(),
                         stream: int = 0) -> None:
    """Image.toRgb8 on the device between two device buffers (pointers as ints)."""
    N.check(N.lib().zt_image_to_rgb8_device(C.c_void_p(d_pixels), n_pixels, TONEMAPS[out.tonemap], out.gamma,
                                            out.exposure, C.c_void_p(d_rgb_out), C.c_void_p(stream)))


def encode_png_device(d_rgb: int, width: int, height: int, d_out: int, capacity: int, stream: int = 0) -> None:
    """png.writePng assembled on the device between two device buffers."""
    N.check(N.lib().zt_png_encode_device(C.c_void_p(d_rgb), width, height, C.c_void_p(d_out), capacity,
                                         C.c_void_p(stream)))


def write_ppm(f, width: int, height: int, rgb: np.ndarray) -> None:
    """Binary P6 PPM, src/image.zig:77-81."""
    assert rgb.size == width * height * 3
    f.write(f"P6\n{width} {height}\n255\n".encode())
    f.write(np.asarray(rgb, np.uint8).tobytes())


# ------------------------------------------------------------------ render --
def render(scene: Scene, opts: Options, gpu: Optional[GpuConfig] = None) -> Image:
    """render.render (src/render.zig:152-180) on the current CUDA device."""
    rec = opts.record()
    out = np.zeros(int(opts.width) * int(opts.height) * 3, np.float64)
    cfg = gpu.record() if gpu is not None else None
    N.check(N.lib().zt_render_ex(scene.handle, N.ptr(rec), N.ptr(cfg) if cfg is not None else None, N.ptr(out)))
    return Image(int(opts.width), int(opts.height), out.reshape(-1, 3))


def render_rgb8(scene: Scene, opts: Options, out: Output = Output(), gpu: Optional[GpuConfig] = None) -> np.ndarray:
    """render + Image.toRgb8 with both stages on the device (W*H*3 bytes)."""
    rec = opts.record()
    cfg = gpu.record() if gpu is not None else None
    rgb = np.zeros(int(opts.width) * int(opts.height) * 3, np.uint8)
    N.check(N.lib().zt_render_rgb8(scene.handle, N.ptr(rec), N.ptr(cfg) if cfg is not None else None,
                                   TONEMAPS[out.tonemap], out.gamma, out.exposure, N.ptr(rgb)))
    return rgb


def render_png(scene: Scene, opts: Options, out: Output = Output(), gpu: Optional[GpuConfig] = None) -> bytes:
    """render + Image.toRgb8 + png.writePng with every stage on the device:
    the bytes of the PNG file."""
    rec = opts.record()
    cfg = gpu.record() if gpu is not None else None
    n = png_size(int(opts.width), int(opts.height))
    buf = np.zeros(n, np.uint8)
    N.check(N.lib().zt_render_png(scene.handle, N.ptr(rec), N.ptr(cfg) if cfg is not None else None,
                                  TONEMAPS[out.tonemap], out.gamma, out.exposure, N.ptr(buf), n))
    return buf.tobytes()


def render_device(scene: Scene, opts: Options, d_out_ptr: int, stream_ptr: int,
                  gpu: Optional[GpuConfig] = None) -> None:
    """Enqueues a render into a device buffer on a CUDA stream (no sync)."""
    rec = opts.record()
    cfg = gpu.record() if gpu is not None else None
    N.check(N.lib().zt_render_device(scene.handle, N.ptr(rec), N.ptr(cfg) if cfg is not None else None,
                                     C.c_void_p(d_out_ptr), C.c_void_p(stream_ptr)))


def render_rows_device(scene: Scene, opts: Options, y0: int, y1: int, d_out_ptr: int, stream_ptr: int = 0,
                       gpu: Optional[GpuConfig] = None) -> None:
    """Enqueues rows [y0, y1) of the image into a device buffer of
    (y1 - y0) * width * 3 doubles on a CUDA stream (no sync)."""
    rec = opts.record()
    cfg = gpu.record() if gpu is not None else None
    N.check(N.lib().zt_render_rows_device(scene.handle, N.ptr(rec), int(y0), int(y1),
                                          N.ptr(cfg) if cfg is not None else None, C.c_void_p(d_out_ptr),
                                          C.c_void_p(stream_ptr)))


class Batch:
    """A prepared batch of renders (zt_batch): one persistent launch over all
    images, captured in a CUDA graph and replayed by ``launch``.  Outputs are
    device buffers given as integer addresses (e.g. ``tensor.data_ptr()``).
    order 1 puts the largest renders first."""

    def __init__(self, scenes, opts_list, d_out_ptrs, gpu: Optional[GpuConfig] = None, order: int = 1):
        n = len(scenes)
        assert n == len(opts_list) == len(d_out_ptrs) and n > 0
        self._scenes = list(scenes)  # keep the scenes (and their device copies) alive
        handles = (C.c_void_p * n)(*[s.handle.value for s in scenes])
        recs = np.concatenate([o.record() for o in opts_list])
        outs = (C.c_void_p * n)(*[int(p) for p in d_out_ptrs])
        cfg = gpu.record() if gpu is not None else None
        h = C.c_void_p()
        N.check(N.lib().zt_batch_create(handles, N.ptr(recs), n, outs, N.ptr(cfg) if cfg is not None else None,
                                        order, C.byref(h)))
        self._h = h

    def launch(self, stream_ptr: int = 0) -> None:
        N.check(N.lib().zt_batch_launch(self._h, C.c_void_p(stream_ptr)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            N.lib().zt_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def render_batch(scenes, opts_list, gpu: Optional[GpuConfig] = None):
    """Many renders in one persistent launch; returns one Image per render."""
    n = len(scenes)
    outs = [np.zeros(int(o.width) * int(o.height) * 3, np.float64) for o in opts_list]
    handles = (C.c_void_p * n)(*[s.handle.value for s in scenes])
    recs = np.concatenate([o.record() for o in opts_list])
    ptrs = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
    cfg = gpu.record() if gpu is not None else None
    N.check(N.lib().zt_render_batch(handles, N.ptr(recs), n, ptrs, N.ptr(cfg) if cfg is not None else None))
    return [Image(int(o.width), int(o.height), a.reshape(-1, 3)) for o, a in zip(opts_list, outs)]


# ------------------------------------------------------ differentiable form --
def _colors_arg(scene: Scene, colors):
    if colors is None:
        return None
    c = np.ascontiguousarray(np.asarray(colors, np.float64).reshape(-1))
    if c.size != 3 * len(scene.materials):
        raise ZigtraceError(-5, f"colors must hold 3 values per material ({3 * len(scene.materials)})")
    return c


def forward(scene: Scene, opts: Options, colors=None) -> Image:
    """Image at material colours `colors` (n_materials x 3) with the scene's
    own colours driving sampling (zt_forward); colors=None gives render()."""
    c = _colors_arg(scene, colors)
    out = np.zeros(int(opts.width) * int(opts.height) * 3, np.float64)
    N.check(N.lib().zt_forward(scene.handle, N.ptr(opts.record()), N.ptr(c) if c is not None else None, N.ptr(out)))
    return Image(int(opts.width), int(opts.height), out.reshape(-1, 3))


def backward(scene: Scene, opts: Options, d_image, colors=None) -> np.ndarray:
    """dL/dcolors (n_materials x 3) for dL/dimage (width*height x 3), by path
    replay (zt_backward)."""
    c = _colors_arg(scene, colors)
    g = np.ascontiguousarray(np.asarray(d_image, np.float64).reshape(-1))
    if g.size != int(opts.width) * int(opts.height) * 3:
        raise ZigtraceError(-5, "d_image must hold width*height*3 values")
    out = np.zeros(3 * len(scene.materials), np.float64)
    N.check(N.lib().zt_backward(scene.handle, N.ptr(opts.record()), N.ptr(c) if c is not None else None, N.ptr(g),
                                N.ptr(out)))
    return out.reshape(-1, 3)


def forward_rows(scene: Scene, opts: Options, y0: int, y1: int, colors=None) -> np.ndarray:
    """Rows [y0, y1) of forward()'s image ((y1-y0)*width x 3), zt_forward_rows."""
    c = _colors_arg(scene, colors)
    out = np.zeros(max(y1 - y0, 0) * int(opts.width) * 3 + 1, np.float64)  # the C ABI validates the band
    N.check(N.lib().zt_forward_rows(scene.handle, N.ptr(opts.record()), y0, y1, N.ptr(c) if c is not None else None,
                                    N.ptr(out)))
    return out[:-1].reshape(-1, 3)


def backward_rows(scene: Scene, opts: Options, y0: int, y1: int, d_band, colors=None) -> np.ndarray:
    """The share of dL/dcolors of image rows [y0, y1): d_band is dL/d(those
    rows) ((y1-y0)*width x 3); the shares of all bands sum to backward()'s."""
    c = _colors_arg(scene, colors)
    g = np.ascontiguousarray(np.asarray(d_band, np.float64).reshape(-1))
    if g.size != max(y1 - y0, 0) * int(opts.width) * 3:
        raise ZigtraceError(-5, "d_band must hold (y1-y0)*width*3 values")
    out = np.zeros(3 * len(scene.materials), np.float64)
    N.check(N.lib().zt_backward_rows(scene.handle, N.ptr(opts.record()), y0, y1, N.ptr(c) if c is not None else None,
                                     N.ptr(g if g.size else np.zeros(1)), N.ptr(out)))
    return out.reshape(-1, 3)


def set_colors(scene: Scene, colors) -> Scene:
    """Makes `colors` the scene's own material colours (they then also drive
    sampling) and rebuilds it."""
    c = np.asarray(colors, np.float64).reshape(-1, 3)
    mats = scene.materials.copy()
    mats["color"] = c
    scene._mats = list(mats)
    return scene.build()


def render_function():
    """torch.autograd.Function computing the image from material colours:
    ``img = render_function().apply(colors, scene, opts)`` with colors a
    float64 tensor (n_materials x 3); backward by path replay."""
    import torch

    class RenderFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, colors, scene, opts):
            ctx.scene, ctx.opts = scene, opts
            c = colors.detach().cpu().numpy()
            ctx.save_for_backward(colors)
            return torch.from_numpy(forward(scene, opts, c).pixels.copy()).to(colors.device)

        @staticmethod
        def backward(ctx, grad_image):
            (colors,) = ctx.saved_tensors
            g = backward(ctx.scene, ctx.opts, grad_image.detach().cpu().numpy(), colors.detach().cpu().numpy())
            return torch.from_numpy(g).to(colors.device), None, None

    return RenderFunction


def render_debug(scene: Scene, opts: Options):
    """First-sample primitive ids and path lengths per pixel (device)."""
    n = int(opts.width) * int(opts.height)
    fp = np.zeros(n, np.int32)
    pl = np.zeros(n, np.uint32)
    N.check(N.lib().zt_render_debug(scene.handle, N.ptr(opts.record()), N.ptr(fp), N.ptr(pl)))
    return fp, pl


def trace_paths(scene: Scene, origin: Vec, direction: Vec, rng_state: np.ndarray, n: int, max_depth: int,
                light_sampling: bool = True) -> np.ndarray:
    """render.traceWith n times along one ray with one RNG stream (the
    reference tests' meanRadiance loop), on the device.  ``rng_state`` (4
    uint64 words) is updated in place; returns (n, 3) radiance."""
    assert rng_state.dtype == np.uint64 and rng_state.shape == (4,) and rng_state.flags["C_CONTIGUOUS"]
    o = np.asarray(origin, np.float64).reshape(3).copy()
    d = np.asarray(direction, np.float64).reshape(3).copy()
    out = np.zeros(int(n) * 3, np.float64)
    N.check(N.lib().zt_trace_paths(scene.handle, N.ptr(o), N.ptr(d), N.ptr(rng_state), int(n), int(max_depth),
                                   1 if light_sampling else 0, N.ptr(out)))
    return out.reshape(-1, 3)


def rng_streams(seed: int, stream0: int, n_streams: int, n_draws: int) -> np.ndarray:
    """Rng.forStream + next() draws evaluated on the device."""
    out = np.zeros(n_streams * n_draws, np.uint64)
    N.check(N.lib().zt_rng_streams(seed, stream0, n_streams, n_draws, N.ptr(out)))
    return out.reshape(n_streams, n_draws)
