"""zt_scene_set_bvh: a BVH built elsewhere (the reference's Bvh.build output,
bvh.zig:41-67) used as given.  CPU only: the oracle's own tree goes in
through the C ABI and comes back node for node; every malformed tree that
could make the device walk leave its arrays or its stack is rejected."""
import numpy as np
import pytest

import kat_scenes as K
import oracle as O
import zigtrace_b200 as zt
from zigtrace_b200 import _native as N
from zigtrace_b200 import scenes


def _as_abi(nodes):
    out = np.zeros(len(nodes), N.BVH_NODE_DTYPE)
    out["bmin"], out["bmax"] = nodes["bmin"], nodes["bmax"]
    out["first"], out["count"] = nodes["first"], nodes["count"]
    return out


@pytest.mark.parametrize("make", [scenes.cornell, scenes.random_spheres, lambda: K.fuzz_scene(3),
                                  lambda: K.random_shapes(7, 300)])
def test_oracle_tree_round_trips(native_lib, make):
    scene = make()
    onodes, oidx = O.OracleScene.from_scene(scene).bvh()
    imported = make().build_with_bvh(_as_abi(onodes), oidx)
    built = make().build()
    n1, i1 = imported.bvh()
    n2, i2 = built.bvh()
    assert n1.tobytes() == n2.tobytes() and i1.tobytes() == i2.tobytes()
    l1, c1, t1 = imported.lights()
    l2, c2, t2 = built.lights()
    assert l1.tobytes() == l2.tobytes() and c1.tobytes() == c2.tobytes() and t1 == t2
    assert imported.counts() == built.counts()


def test_empty_scene(native_lib):
    s = zt.Scene()
    m = s.add_material(zt.Material.lambertian((0.5, 0.5, 0.5)))
    s.add(zt.plane((0, 0, 0), (0, 1, 0), m))
    s.build_with_bvh(np.zeros(0, N.BVH_NODE_DTYPE), np.zeros(0, np.uint32))
    assert s.counts()["nodes"] == 0


def _base():
    scene = scenes.cornell()
    nodes, idx = O.OracleScene.from_scene(scene).bvh()
    return scene, _as_abi(nodes), idx.copy()


def _rejects(scene, nodes, idx, what):
    with pytest.raises(zt.ZigtraceError) as ei:
        scene.build_with_bvh(nodes, idx)
    assert ei.value.name == "InvalidArgument" and what in str(ei.value), str(ei.value)


def test_malformed_trees_are_rejected(native_lib):
    scene, nodes, idx = _base()
    interior = np.flatnonzero(nodes["count"] == 0)
    leaves = np.flatnonzero(nodes["count"] > 0)

    bad = idx.copy(); bad[0] = bad[1]
    _rejects(scene, nodes, bad, "permutation")
    bad = idx.copy(); bad[0] = 10_000
    _rejects(scene, nodes, bad, "permutation")
    _rejects(scene, nodes, idx[:-1], "one entry per bounded shape")
    _rejects(scene, nodes[:-1], idx, "node count")

    b = nodes.copy(); b["first"][interior[0]] += 1  # even child index
    _rejects(scene, b, idx, "in a pair")
    b = nodes.copy(); b["first"][interior[-1]] = len(nodes) - 1  # right child past the end
    _rejects(scene, b, idx, "in a pair")
    b = nodes.copy(); b["first"][0] = 1; b["first"][interior[1]] = 1  # two parents of the same pair
    _rejects(scene, b, idx, "")
    b = nodes.copy(); b["first"][leaves[0]] = len(idx) - 1; b["count"][leaves[0]] = 2  # past the last shape
    _rejects(scene, b, idx, "past the last shape")
    b = nodes.copy(); b["first"][leaves[1]] = b["first"][leaves[0]]  # two leaves share a position
    _rejects(scene, b, idx, "")
    # the scene is left unbuilt after a rejection
    with pytest.raises(zt.ZigtraceError) as ei:
        scene.bvh()
    assert ei.value.name == "NotBuilt"


def test_depth_beyond_64_is_rejected(native_lib):
    """A chain (each interior node: a one-shape leaf and the rest) of depth 65
    would overflow the traversal stack of max_depth + 2 entries."""
    n = 67
    s = zt.Scene()
    m = s.add_material(zt.Material.lambertian((0.5, 0.5, 0.5)))
    s.add_spheres(np.stack([np.arange(n, dtype=float), np.zeros(n), np.zeros(n)], 1), np.full(n, 0.4), m)

    def chain(depth):
        nodes = [(0, n)]  # (first, count) per node; bounds do not matter for the shape checks
        cur, pos = 0, 0
        for _ in range(depth):
            left = len(nodes)
            nodes[cur] = (left, 0)
            nodes.append((pos, 1))          # leaf with one shape
            nodes.append((pos + 1, n - pos - 1))
            pos += 1
            cur = left + 1
        a = np.zeros(len(nodes), N.BVH_NODE_DTYPE)
        a["first"] = [f for f, _ in nodes]
        a["count"] = [c for _, c in nodes]
        a["bmin"], a["bmax"] = -100.0, 100.0
        return a

    s.build_with_bvh(chain(64), np.arange(n, dtype=np.uint32))  # level 64 is the reference's deepest
    assert s.bvh_depth() == 65  # Bvh.depth counts levels (bvh.zig:128-137)
    with pytest.raises(zt.ZigtraceError) as ei:
        s.build_with_bvh(chain(65), np.arange(n, dtype=np.uint32))
    assert "deeper than 64" in str(ei.value)
