"""The fast traversal's float box test reaches every box the reference's f64
test reaches (zigtrace_b200/csrc/zt_fast.cuh, superset property), checked on
the CPU with the device arithmetic restated in NumPy: float records built as
in scene_host.cpp (bounds moved out by 2^-20 M per axis, then rounded out to
float), per-ray constants and slab test as in zt_fast.cuh (the FMA emulated
as a float64 product-sum rounded once to float32).  Rays aim at box corners,
edges and faces from near and far, including axis-parallel directions and
origins on box planes: the cases where rounding decides the f64 test."""
import numpy as np

import oracle as O
import zigtrace_b200 as zt

F32 = np.float32


def f64_slab(lo, hi, o, inv, tmin, tmax):
    """aabb.zig:68-83 as the device's compare-and-select form."""
    l = np.full(len(o), tmin)
    h = np.full(len(o), tmax)
    with np.errstate(invalid="ignore", over="ignore"):
        for a in range(3):
            t0 = (lo[:, a] - o[:, a]) * inv[:, a]
            t1 = (hi[:, a] - o[:, a]) * inv[:, a]
            sw = inv[:, a] < 0
            n = np.where(sw, t1, t0)
            f = np.where(sw, t0, t1)
            l = np.where(n > l, n, l)
            h = np.where(f < h, f, h)
    return ~(h < l)


def out_f32(x, up):
    f = x.astype(F32)
    if up:
        return np.where(f.astype(np.float64) < x, np.nextafter(f, F32(np.inf)), f)
    return np.where(f.astype(np.float64) > x, np.nextafter(f, F32(-np.inf)), f)


def fast_records(lo, hi, root_lo, root_hi):
    eps = np.ldexp(np.maximum(np.abs(root_lo), np.abs(root_hi)), -20)
    return out_f32(lo - eps, False), out_f32(hi + eps, True)


def fma32(a, b, c):
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(F32)


def f32_slab(lo32, hi32, o, d, tmin, tmax, rcp_ulps=None):
    """rcp_ulps: per-element -1/0/+1, the device reciprocal's error (it is
    within 1 ulp of the correctly rounded one)."""
    o32, d32 = o.astype(F32), d.astype(F32)
    om = np.abs(o32).max(axis=1)
    K = np.where(om > F32(1e7), F32(1e37) / om, F32(1e30)).astype(F32)
    with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
        inv = F32(1) / d32
        if rcp_ulps is not None:
            inv = np.where(rcp_ulps > 0, np.nextafter(inv, F32(np.inf)),
                           np.where(rcp_ulps < 0, np.nextafter(inv, F32(-np.inf)), inv)).astype(F32)
    inv = np.where(np.abs(inv) <= K[:, None], inv, np.copysign(K[:, None], inv)).astype(F32)
    n = (-o32 * inv).astype(F32)
    w = (np.abs(n) * F32(2.0 ** -20)).astype(F32)
    off_lo = np.where(inv >= 0, n - w, n + w).astype(F32)
    off_hi = np.where(inv >= 0, n + w, n - w).astype(F32)
    a = fma32(lo32, inv, off_lo)
    b = fma32(hi32, inv, off_hi)
    tmin32 = out_f32(np.full(len(o), tmin), False)
    tmax32 = out_f32(np.full(len(o), tmax), True)
    near = np.maximum(np.minimum(a, b).max(axis=1), tmin32)
    far = np.minimum(np.maximum(a, b).min(axis=1), tmax32)
    return near <= far, near


def _scene_boxes(seed):
    rng = np.random.default_rng(seed)
    s = zt.Scene()
    m = s.add_material(zt.Material.lambertian((0.5, 0.5, 0.5)))
    c = rng.uniform(-500, 500, (400, 3)) * np.array([1.0, 0.02, 0.5])
    s.add_triangles(c, c + rng.uniform(-3, 3, (400, 3)), c + rng.uniform(-3, 3, (400, 3)), m)
    s.add_spheres(rng.uniform(-200, 200, (50, 3)), rng.uniform(0.1, 5, 50), m)
    nodes, _ = O.OracleScene.from_scene(s).bvh()
    return nodes["bmin"], nodes["bmax"]


def _grazing_rays(lo, hi, rng, n):
    """Rays aimed at a point on a random box's surface (corner, edge or face)."""
    k = rng.integers(0, len(lo), n)
    u = rng.integers(0, 3, (n, 3))  # per axis: at lo, at hi, or inside
    frac = rng.random((n, 3))
    tgt = np.where(u == 0, lo[k], np.where(u == 1, hi[k], lo[k] + frac * (hi[k] - lo[k])))
    dist = 10.0 ** rng.uniform(-3, 4, n)
    d = rng.normal(size=(n, 3))
    axis_par = rng.random(n) < 0.2  # zero components
    d[axis_par, rng.integers(0, 3, axis_par.sum())] = 0.0
    d /= np.linalg.norm(d, axis=1)[:, None]
    o = tgt - d * dist[:, None]
    on_plane = rng.random(n) < 0.1  # origin exactly on one of the box's planes
    ax = rng.integers(0, 3, n)
    o[on_plane, ax[on_plane]] = lo[k[on_plane], ax[on_plane]]
    return k, o, d


def test_float_box_test_is_a_superset_of_the_f64_test():
    rng = np.random.default_rng(1)
    total_hits = 0
    for seed in range(3):
        lo, hi = _scene_boxes(seed)
        lo32, hi32 = fast_records(lo, hi, lo[0], hi[0])
        assert (lo32 <= lo).all() and (hi32 >= hi).all()
        k, o, d = _grazing_rays(lo, hi, rng, 200_000)
        # also random other boxes for every ray
        k = np.concatenate([k, rng.integers(0, len(lo), len(k))])
        o = np.concatenate([o, o])
        d = np.concatenate([d, d])
        with np.errstate(divide="ignore"):
            inv = 1.0 / d
        for tmin, tmax in ((1e-4, np.inf), (1e-4, 37.5), (0.0, 1e3)):
            hit64 = f64_slab(lo[k], hi[k], o, inv, tmin, tmax)
            hit32, near32 = f32_slab(lo32[k], hi32[k], o, d, tmin, tmax,
                                     rcp_ulps=rng.integers(-1, 2, size=(len(o), 3)))
            missed = hit64 & ~hit32
            assert not missed.any(), f"{missed.sum()} boxes reached by the f64 test but not the float test"
            total_hits += int(hit64.sum())
    assert total_hits > 100_000


def test_float_entry_distance_is_a_lower_bound():
    """Entry distances order the walk and prune it: the float one must not
    exceed the f64 one wherever the f64 test reaches the box."""
    rng = np.random.default_rng(2)
    lo, hi = _scene_boxes(7)
    lo32, hi32 = fast_records(lo, hi, lo[0], hi[0])
    k, o, d = _grazing_rays(lo, hi, rng, 200_000)
    with np.errstate(divide="ignore"):
        inv = 1.0 / d
    tmin = 1e-4
    hit64 = f64_slab(lo[k], hi[k], o, inv, tmin, np.inf)
    _, near32 = f32_slab(lo32[k], hi32[k], o, d, tmin, np.inf, rcp_ulps=rng.integers(-1, 2, size=(len(o), 3)))
    near64 = np.full(len(o), tmin)
    with np.errstate(invalid="ignore", over="ignore"):
        for a in range(3):
            t0 = (lo[k, a] - o[:, a]) * inv[:, a]
            t1 = (hi[k, a] - o[:, a]) * inv[:, a]
            n = np.where(inv[:, a] < 0, t1, t0)
            near64 = np.where(n > near64, n, near64)
    assert (near32[hit64].astype(np.float64) <= near64[hit64]).all()
