"""Scene loading (src/scenefile.zig): the reference's own parser tests
(scenefile.zig:233-275) restated, plus a scene file rendered the same as
the scene built through the API."""
import numpy as np
import pytest

import zigtrace_b200 as zt
from zigtrace_b200 import scenefile


def test_parses_a_complete_scene():
    src = "\n".join([
        "# a test scene",
        "image 320 200",
        "samples 8",
        "depth 5",
        "camera from 0 1 5 to 0 0 0 fov 35 aperture 0.2 focus 4.5",
        "background color 0.1 0.2 0.3",
        "material ground lambertian 0.5 0.5 0.5",
        "material steel metal 0.8 0.8 0.8 0.1",
        "material glass dielectric 1.5   # trailing comment",
        "material lamp emissive 4 4 4",
        "",
        "sphere 0 1 0 1 glass",
        "plane 0 0 0  0 2 0 ground",
        "triangle -1 0 -1  1 0 -1  0 2 -1 steel",
        "quad -1 3 -1  2 0 0  0 0 2 lamp",
    ])
    scene = scenefile.parse(src)
    assert (scene.settings.width, scene.settings.height) == (320, 200)
    assert (scene.settings.spp, scene.settings.max_depth) == (8, 5)
    assert scene.camera.vfov == 35 and scene.camera.focus_dist == 4.5
    assert scene.background.kind == 0 and tuple(scene.background.a) == (0.1, 0.2, 0.3)
    mats = scene.materials
    assert len(mats) == 4 and mats[1]["param"] == 0.1
    c = scene.counts()
    assert c["bounded"] == 4 and c["planes"] == 1  # sphere, triangle, 2 quad halves; the plane
    planes = scene.shapes[scene.shapes["kind"] == zt.PLANE]
    assert tuple(planes[0]["p"][3:6]) == (0.0, 1.0, 0.0)
    assert c["nodes"] > 0


@pytest.mark.parametrize("src,line,msg", [
    ("image 10", 1, "unexpected end of line"),
    ("\n\nsphere 0 0 0 1 nope", 3, "undefined material"),
    ("material a lambertian 1 1 1\nmaterial a dielectric 1.5", 2, "material already defined"),
    ("frobnicate", 1, "unknown directive"),
    ("samples 0", 1, "expected a positive integer"),
    ("camera from 0 0 0 to 0 0 0", 1, "camera 'from' and 'to' must differ"),
    ("camera from 0 0 0", 1, "camera needs 'from' and 'to'"),
    ("material m metal 1 1 1 2", 1, "metal fuzz must be in [0, 1]"),
    ("material m lambertian 1 x 1", 1, "expected a number"),
    ("material m lambertian 1 1 1\ntriangle 0 0 0 1 1 1 2 2 2 m", 2, "degenerate triangle"),
    ("depth 3 4", 1, "unexpected extra tokens"),
    ("background gradient", 1, "background must be 'color' or 'sky'"),
])
def test_reports_errors_with_line_numbers(src, line, msg):
    with pytest.raises(scenefile.SceneFileError) as ei:
        scenefile.parse(src)
    assert ei.value.line == line and ei.value.message == msg


def test_more_diagnostics():
    for src, msg in [("sphere 0 0 0 1 m", "undefined material"),
                     ("material m lambertian 1 1 1\nsphere 0 0 0 0 m", "sphere radius must be non-zero"),
                     ("material m lambertian 1 1 1\nplane 0 0 0 0 0 0 m", "plane normal must be non-zero"),
                     ("material m lambertian 1 1 1\nquad 0 0 0 1 0 0 2 0 0 m", "degenerate quad"),
                     ("camera from 0 0 1 to 0 0 0 up 0 0 1", "camera 'up' is parallel to the view direction"),
                     ("camera from 0 0 1 to 0 0 0 fov 180", "fov must be between 0 and 180 degrees"),
                     ("material m lambertian -1 1 1", "colour components must be non-negative"),
                     ("material m dielectric 0", "index of refraction must be positive"),
                     ("material m plastic 1 1 1", "unknown material type"),
                     ("material m lambertian inf 1 1", "number must be finite"),
                     ("camera from 0 0 1 to 0 0 0 zoom 2", "unknown camera parameter")]:
        with pytest.raises(scenefile.SceneFileError) as ei:
            scenefile.parse(src)
        assert ei.value.message == msg, src


def test_file_scene_equals_api_scene(native_lib, tmp_path):
    src = """image 40 30
samples 2
depth 8
camera from 0 1.5 6 to 0 0.5 0 fov 45
background sky 1 1 1  0.5 0.7 1.0
material floor lambertian 0.6 0.6 0.5
material ball metal 0.9 0.8 0.7 0.2
material lamp emissive 6 6 5
plane 0 0 0  0 3 0 floor
sphere -0.8 0.6 0 0.6 ball
quad -0.5 2 -0.5  1 0 0  0 0 1 lamp
"""
    p = tmp_path / "s.txt"
    p.write_text(src)
    a = scenefile.load(str(p))
    b = zt.Scene()
    floor = b.add_material(zt.Material.lambertian((0.6, 0.6, 0.5)))
    ball = b.add_material(zt.Material.metal((0.9, 0.8, 0.7), 0.2))
    lamp = b.add_material(zt.Material.emissive((6, 6, 5)))
    b.add(zt.plane((0, 0, 0), (0, 1, 0), floor))
    b.add(zt.sphere((-0.8, 0.6, 0), 0.6, ball))
    b.add_quad((-0.5, 2, -0.5), (1, 0, 0), (0, 0, 1), lamp)
    b.camera = zt.CameraConfig(look_from=(0, 1.5, 6), look_at=(0, 0.5, 0), vfov=45)
    b.background = zt.Background.sky((1, 1, 1), (0.5, 0.7, 1.0))
    b.build()
    assert a.shapes.tobytes() == b.shapes.tobytes() and a.materials.tobytes() == b.materials.tobytes()
    (an, ai), (bn, bi) = a.bvh(), b.bvh()
    assert an.tobytes() == bn.tobytes() and ai.tobytes() == bi.tobytes()
