"""Scene loading from the line-oriented text format of src/scenefile.zig.

``parse(source)`` returns a built ``Scene`` (settings, camera, background,
named materials, spheres, planes, triangles and quads), or raises
``SceneFileError`` with the 1-based line number and the reference's message
(scenefile.zig:33-103).  Each non-blank line is one directive; ``#`` starts
a comment; materials are named and must be declared before shapes use them.
"""
from __future__ import annotations

import math
import re
from typing import Dict, List, Optional, Tuple

from .api import (Background, CameraConfig, Material, Scene, plane, sphere, triangle)

Vec = Tuple[float, float, float]


class SceneFileError(ValueError):
    """SyntaxError of scenefile.parse with its Diagnostic (line, message)."""

    def __init__(self, line: int, message: str):
        self.line = line
        self.message = message
        super().__init__(f"line {line}: {message}")


def _sub(a: Vec, b: Vec) -> Vec:
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def _cross(a: Vec, b: Vec) -> Vec:  # vec.zig cross
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def _near_zero(a: Vec) -> bool:  # vec.zig nearZero
    return abs(a[0]) < 1e-8 and abs(a[1]) < 1e-8 and abs(a[2]) < 1e-8


def _normalize(a: Vec) -> Vec:  # Vec3.normalize: scale by the reciprocal of the length
    inv = 1.0 / math.sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2])
    return (a[0] * inv, a[1] * inv, a[2] * inv)


class _Line:
    """LineParser, scenefile.zig:182-231."""

    def __init__(self, tokens: List[str], line: int):
        self.tokens = tokens
        self.pos = 0
        self.line = line

    def fail(self, message: str) -> SceneFileError:
        return SceneFileError(self.line, message)

    def peek(self) -> Optional[str]:
        return self.tokens[self.pos] if self.pos < len(self.tokens) else None

    def word(self) -> str:
        if self.pos >= len(self.tokens):
            raise self.fail("unexpected end of line")
        self.pos += 1
        return self.tokens[self.pos - 1]

    def number(self) -> float:
        tok = self.word()
        try:
            if not tok.isascii():
                raise ValueError(tok)
            body = tok.lstrip("+-")
            v = float.fromhex(tok) if body[:2].lower() == "0x" else float(tok)
        except ValueError:
            raise self.fail("expected a number") from None
        if not math.isfinite(v):
            raise self.fail("number must be finite")
        return v

    def positive_int(self) -> int:
        tok = self.word()
        try:
            if not tok.isascii():
                raise ValueError(tok)
            v = int(tok, 10)
        except ValueError:
            raise self.fail("expected a positive integer") from None
        if v <= 0:
            raise self.fail("expected a positive integer")
        return v

    def vec(self) -> Vec:
        return (self.number(), self.number(), self.number())

    def color(self) -> Vec:
        c = self.vec()
        if c[0] < 0 or c[1] < 0 or c[2] < 0:
            raise self.fail("colour components must be non-negative")
        return c

    def material_ref(self, names: Dict[str, int]) -> int:
        name = self.word()
        if name not in names:
            raise self.fail("undefined material")
        return names[name]

    def end(self) -> None:
        if self.pos < len(self.tokens):
            raise self.fail("unexpected extra tokens")


def _camera(p: _Line, scene: Scene) -> None:  # parseCamera, scenefile.zig:106-136
    cfg = scene.camera
    look_from, look_at, up = tuple(cfg.look_from), tuple(cfg.look_at), tuple(cfg.up)
    vfov, aperture, focus = cfg.vfov, cfg.aperture, cfg.focus_dist
    saw_from = saw_to = False
    while p.peek() is not None:
        key = p.word()
        if key == "from":
            look_from, saw_from = p.vec(), True
        elif key == "to":
            look_at, saw_to = p.vec(), True
        elif key == "up":
            up = p.vec()
        elif key == "fov":
            vfov = p.number()
            if not (0 < vfov < 180):
                raise p.fail("fov must be between 0 and 180 degrees")
        elif key == "aperture":
            aperture = p.number()
            if aperture < 0:
                raise p.fail("aperture must be non-negative")
        elif key == "focus":
            f = p.number()
            if not f > 0:
                raise p.fail("focus distance must be positive")
            focus = f
        else:
            raise p.fail("unknown camera parameter")
    if not saw_from or not saw_to:
        raise p.fail("camera needs 'from' and 'to'")
    view = _sub(look_from, look_at)
    if _near_zero(view):
        raise p.fail("camera 'from' and 'to' must differ")
    if _near_zero(_cross(up, view)):
        raise p.fail("camera 'up' is parallel to the view direction")
    scene.camera = CameraConfig(look_from=look_from, look_at=look_at, up=up, vfov=vfov, aperture=aperture,
                                focus_dist=focus)


def _material(p: _Line) -> object:  # parseMaterial, scenefile.zig:138-153
    kind = p.word()
    if kind == "lambertian":
        return Material.lambertian(p.color())
    if kind == "metal":
        albedo = p.color()
        fuzz = p.number() if p.peek() is not None else 0.0
        if fuzz < 0 or fuzz > 1:
            raise p.fail("metal fuzz must be in [0, 1]")
        return Material.metal(albedo, fuzz)
    if kind == "dielectric":
        ior = p.number()
        if not ior > 0:
            raise p.fail("index of refraction must be positive")
        return Material.dielectric(ior)
    if kind == "emissive":
        return Material.emissive(p.color())
    raise p.fail("unknown material type")


def parse(source: str, build: bool = True, device: bool = False) -> Scene:
    """scenefile.parse (scenefile.zig:35-103): the scene, built (on the
    device with device=True, zt_scene_build_device)."""
    scene = Scene()
    names: Dict[str, int] = {}
    for line_no, raw in enumerate(source.split("\n"), start=1):
        line = raw.split("#", 1)[0]
        p = _Line([t for t in re.split(r"[ \t\r]+", line) if t], line_no)  # tokenizeAny(" \t\r")
        keyword = p.peek()
        if keyword is None:
            continue
        p.word()
        if keyword == "image":
            scene.settings.width = p.positive_int()
            scene.settings.height = p.positive_int()
        elif keyword == "samples":
            scene.settings.spp = p.positive_int()
        elif keyword == "depth":
            scene.settings.max_depth = p.positive_int()
        elif keyword == "camera":
            _camera(p, scene)
        elif keyword == "background":
            kind = p.word()
            if kind == "color":
                scene.background = Background.solid(p.vec())
            elif kind == "sky":
                scene.background = Background.sky(p.vec(), p.vec())
            else:
                raise p.fail("background must be 'color' or 'sky'")
        elif keyword == "material":
            name = p.word()
            if name in names:
                raise p.fail("material already defined")
            names[name] = scene.add_material(_material(p))
        elif keyword == "sphere":
            center = p.vec()
            radius = p.number()
            if radius == 0:
                raise p.fail("sphere radius must be non-zero")
            scene.add(sphere(center, radius, p.material_ref(names)))
        elif keyword == "plane":
            point = p.vec()
            normal = p.vec()
            if _near_zero(normal):
                raise p.fail("plane normal must be non-zero")
            scene.add(plane(point, _normalize(normal), p.material_ref(names)))
        elif keyword == "triangle":
            v0, v1, v2 = p.vec(), p.vec(), p.vec()
            if _near_zero(_cross(_sub(v1, v0), _sub(v2, v0))):
                raise p.fail("degenerate triangle")
            scene.add(triangle(v0, v1, v2, p.material_ref(names)))
        elif keyword == "quad":
            corner, u, v = p.vec(), p.vec(), p.vec()
            if _near_zero(_cross(u, v)):
                raise p.fail("degenerate quad")
            scene.add_quad(corner, u, v, p.material_ref(names))
        else:
            raise p.fail("unknown directive")
        p.end()
    if build:
        scene.build(device=device)
    return scene


def load(path: str, build: bool = True, device: bool = False) -> Scene:
    """parse() of a file."""
    with open(path, "r", encoding="utf-8") as f:
        return parse(f.read(), build=build, device=device)
