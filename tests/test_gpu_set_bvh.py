"""Rendering from a BVH handed in through zt_scene_set_bvh (the reference's
own tree, used as given) on the GPU: bit-exact against the oracle, in every
single-scene mode; a tree whose leaves are too large for the fast
traversal's packed records renders exact under PRECISION_FAST."""
import numpy as np
import pytest

import kat_scenes as K
import oracle as O
import zigtrace_b200 as zt
from zigtrace_b200 import _native as N
from zigtrace_b200 import scenes

pytestmark = pytest.mark.gpu


def _as_abi(nodes):
    out = np.zeros(len(nodes), N.BVH_NODE_DTYPE)
    out["bmin"], out["bmax"] = nodes["bmin"], nodes["bmax"]
    out["first"], out["count"] = nodes["first"], nodes["count"]
    return out


@pytest.mark.parametrize("mode", [zt.MODE_MEGAKERNEL, zt.MODE_WAVEFRONT, zt.MODE_MEGAKERNEL_REGEN,
                                  zt.MODE_WAVEFRONT_SORTED])
@pytest.mark.parametrize("make,o", [(scenes.cornell, zt.Options(64, 64, 4, 16)),
                                    (lambda: K.fuzz_scene(5), zt.Options(48, 32, 8, 12, seed=5))])
def test_imported_tree_renders_bit_exact(make, o, mode):
    scene = make()
    os_ = O.OracleScene.from_scene(scene)
    nodes, idx = os_.bvh()
    scene.build_with_bvh(_as_abi(nodes), idx)
    img = zt.render(scene, o, zt.GpuConfig(mode)).pixels
    want = os_.render(o.width, o.height, o.spp, o.max_depth, seed=o.seed)
    assert img.tobytes() == want.tobytes()


def test_one_big_leaf_renders_exact_under_fast():
    """A tree that is a single leaf of 80 primitives: more than the 15 a
    packed fast record holds (and more than the 64 below which a single
    render takes the exact walk anyway), so PRECISION_FAST renders with the
    f64 walk; a tree of one leaf is also what Scene.intersect's brute-force
    loop tests (scene.zig:109-112)."""
    scene = scenes.cornell()
    n = scene.primitive_count()
    rng = np.random.default_rng(3)
    m = scene.add_material(zt.Material.lambertian((0.3, 0.6, 0.2)))
    c = rng.uniform(100, 450, (80 - n, 3))
    scene.add_triangles(c, c + rng.uniform(-40, 40, c.shape), c + rng.uniform(-40, 40, c.shape), m)
    n = scene.primitive_count()
    shapes = scene.shapes
    lo = np.minimum(np.minimum(shapes["p"][:, 0:3], shapes["p"][:, 3:6]), shapes["p"][:, 6:9])
    hi = np.maximum(np.maximum(shapes["p"][:, 0:3], shapes["p"][:, 3:6]), shapes["p"][:, 6:9])
    sph = shapes["kind"] == zt.SPHERE
    r = shapes["p"][:, 3:4]
    lo[sph] = shapes["p"][sph, 0:3] - np.abs(r[sph])
    hi[sph] = shapes["p"][sph, 0:3] + np.abs(r[sph])
    root = np.zeros(1, N.BVH_NODE_DTYPE)
    root["bmin"], root["bmax"] = lo.min(axis=0), hi.max(axis=0)
    root["first"], root["count"] = 0, n
    scene.build_with_bvh(root, np.arange(n, dtype=np.uint32))
    o = zt.Options(48, 48, 4, 8)
    fast = zt.render(scene, o, zt.GpuConfig(precision=zt.PRECISION_FAST)).pixels
    exact = zt.render(scene, o).pixels
    assert fast.tobytes() == exact.tobytes()
