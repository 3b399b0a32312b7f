"""Device BVH build (zt_scene_build_device) against the host build.

The host build is pinned to the oracle node for node (test_host_scene); the
device build must give the same tree: every node's first/count, the
primitive permutation, and bounds equal as numbers (the sign of a zero may
differ: min/max of +0 and -0 may return either, which no traversal or split
decision distinguishes).  Renders of the two builds are bit-identical.
"""
import numpy as np
import pytest

import kat_scenes as K
import zigtrace_b200 as zt
from zigtrace_b200 import scenes

pytestmark = pytest.mark.gpu


def _pair(build):
    host = build().build()
    dev = build().build(device=True)
    return host, dev


def _same_tree(host, dev):
    hn, hi = host.bvh()
    dn, di = dev.bvh()
    assert len(hn) == len(dn)
    assert (hn["first"] == dn["first"]).all() and (hn["count"] == dn["count"]).all()
    assert (hn["bmin"] == dn["bmin"]).all() and (hn["bmax"] == dn["bmax"]).all()
    assert hi.tobytes() == di.tobytes()


CASES = {
    "cornell": scenes.cornell,                                   # 12 triangles + 2 spheres: one warp subtree
    "demo": K.demo_scene,
    "spheres": scenes.random_spheres,                            # ~320 spheres: large levels + warp subtrees
    "random_shapes_2000": lambda: K.random_shapes(3, 2000),
    "sphere_field_20000": lambda: scenes.sphere_field(5, 20000),
    "fuzz_0": lambda: K.fuzz_scene(0),
    "fuzz_1": lambda: K.fuzz_scene(1),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_device_build_equals_host_build(name):
    host, dev = _pair(CASES[name])
    assert dev.built_on_device
    _same_tree(host, dev)


def test_device_build_triangle_heavy_and_render():
    host, dev = _pair(scenes.triangle_heavy)
    assert dev.built_on_device and dev.build_ms is not None
    _same_tree(host, dev)
    o = zt.Options(320, 180, 2, 16)
    assert zt.render(dev, o).pixels.tobytes() == zt.render(host, o).pixels.tobytes()


def test_duplicate_primitives_fall_back_to_the_host():
    def dup():
        s = zt.Scene()
        m = s.add_material(zt.Material.lambertian((0.5, 0.5, 0.5)))
        for _ in range(40):  # 40 identical triangles: splitMedian at the root
            s.add(zt.triangle((0, 0, 0), (1, 0, 0), (0, 1, 0), m))
        s.add(zt.sphere((3, 0, 0), 0.5, m))
        return s
    host, dev = _pair(dup)
    assert not dev.built_on_device
    _same_tree(host, dev)


def test_device_build_of_tiny_and_empty_scenes():
    for build in (lambda: zt.Scene(), lambda: K.random_shapes(1, 1), lambda: K.random_shapes(2, 33)):
        host, dev = _pair(build)
        _same_tree(host, dev)
