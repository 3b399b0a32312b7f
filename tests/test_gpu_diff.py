"""The differentiable form on the GPU: forward parity (bit-exact with the
plain render at the scene's own colours, and with the oracle's detached
forward at other colours), and the path-replay adjoint against central finite
differences with common random numbers, on the device and on the CPU
oracle.  Tolerance: the target is gradients within 2% of finite
differences; with detached sampling each sample is a polynomial in the
colours, so the adjoint and FD agree far closer and the tests use 1e-4
relative."""
import numpy as np
import pytest

import oracle as O
import zigtrace_b200 as zt
from zigtrace_b200 import scenes

pytestmark = pytest.mark.gpu


def small():
    scene, target = scenes.cornell_diff()
    scene.build()
    return scene, target, zt.Options(48, 48, 4, 8)


def test_forward_at_own_colors_is_the_render():
    scene, _, o = small()
    assert zt.forward(scene, o).pixels.tobytes() == zt.render(scene, o).pixels.tobytes()


def test_forward_at_other_colors_matches_oracle():
    scene, target, o = small()
    got = zt.forward(scene, o, target).pixels
    want = O.OracleScene.from_scene(scene).render_params(o.width, o.height, o.spp, o.max_depth, target)
    assert got.tobytes() == want.tobytes()


def _weights(o):
    return np.random.default_rng(4).uniform(-1, 1, (o.width * o.height, 3))


def _check(grad, fd, tol=1e-4):
    for (m, c), g in fd.items():
        assert abs(grad[m, c] - g) <= tol * max(abs(g), 1e-3), (m, c, grad[m, c], g)


PARAMS = [(0, 0), (4, 1), (13, 2), (30, 0), (32, 0), (34, 2)]  # albedos of patches/sphere, emitter radiances


def test_adjoint_matches_device_central_fd():
    scene, _, o = small()
    w = _weights(o)
    theta = np.array([m["color"] for m in scene.materials])
    grad = zt.backward(scene, o, w, theta)
    h = 1e-3
    fd = {}
    for m, c in PARAMS:
        tp, tm = theta.copy(), theta.copy()
        tp[m, c] += h
        tm[m, c] -= h
        lp = (zt.forward(scene, o, tp).pixels * w).sum()
        lm = (zt.forward(scene, o, tm).pixels * w).sum()
        fd[(m, c)] = (lp - lm) / (2 * h)
    _check(grad, fd)
    assert all(abs(v) > 0 for v in fd.values())


def test_adjoint_matches_cpu_oracle_fd():
    scene, _, _ = small()
    o = zt.Options(24, 24, 2, 8)
    w = _weights(o)
    theta = np.array([m["color"] for m in scene.materials])
    grad = zt.backward(scene, o, w, theta)
    os_ = O.OracleScene.from_scene(scene)
    h = 1e-3
    fd = {}
    for m, c in PARAMS[:4]:
        tp, tm = theta.copy(), theta.copy()
        tp[m, c] += h
        tm[m, c] -= h
        lp = (os_.render_params(o.width, o.height, o.spp, o.max_depth, tp) * w).sum()
        lm = (os_.render_params(o.width, o.height, o.spp, o.max_depth, tm) * w).sum()
        fd[(m, c)] = (lp - lm) / (2 * h)
    _check(grad, fd)


def test_autograd_function_and_descent_reduce_the_loss():
    import torch
    scene, target, o = small()
    target_img = torch.from_numpy(zt.forward(scene, o, target).pixels.copy())
    f = zt.render_function()
    start = np.array([m["color"] for m in scene.materials])
    albedo = torch.tensor(start[:32], dtype=torch.float64, requires_grad=True)
    radiance = torch.tensor(start[32:], dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([{"params": [albedo], "lr": 0.02}, {"params": [radiance], "lr": 0.5}])
    losses = []
    for _ in range(20):  # sampling stays at the scene's colours: common random numbers
        opt.zero_grad()
        img = f.apply(torch.cat([albedo, radiance]), scene, o)
        loss = ((img - target_img) ** 2).mean()
        loss.backward()
        assert torch.isfinite(albedo.grad).all() and torch.isfinite(radiance.grad).all()
        opt.step()
        with torch.no_grad():
            albedo.clamp_(0.01, 0.99)
            radiance.clamp_(min=0.0)
        losses.append(loss.item())
    assert losses[-1] < 0.3 * losses[0]


def test_row_bands_of_forward_and_backward():
    """zt_forward_rows bands concatenate to zt_forward's image bit for bit;
    zt_backward_rows shares sum to zt_backward's gradient (atomics: the last
    bits may differ), with and without the forward's primal cache."""
    scene, target, _ = small()
    o = zt.Options(64, 48, 4, 16)
    rng = np.random.default_rng(5)
    th = np.array([m["color"] for m in scene.materials]) * rng.uniform(0.9, 1.1, (len(scene.materials), 3))
    full = zt.forward(scene, o, th).pixels
    bands = [(0, 13), (13, 30), (30, 48)]
    parts = [zt.forward_rows(scene, o, a, b, th) for a, b in bands]
    assert np.concatenate(parts).tobytes() == full.tobytes()
    d = 2.0 * (full - 0.25)
    want = zt.backward(scene, o, d, th)
    for warm in (True, False):
        if warm:
            zt.forward(scene, o, th)  # cache covers every band
        else:
            zt.forward_rows(scene, o, 0, 5, th)  # cache of another band: recomputed
        got = sum(zt.backward_rows(scene, o, a, b, d[a * 64:b * 64], th) for a, b in bands)
        assert np.allclose(got, want, rtol=1e-10, atol=1e-12)


def test_sharded_forward_backward_over_nccl_single_rank():
    import os
    import socket
    import torch
    import torch.distributed as dist
    from zigtrace_b200 import sharding
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        scene, _, _ = small()
        o = zt.Options(48, 32, 2, 16)
        img = sharding.forward_sharded(scene, o)
        assert img.tobytes() == zt.forward(scene, o).pixels.tobytes()
        d = img - 0.1
        g = sharding.backward_sharded(scene, o, d)
        assert np.allclose(g, zt.backward(scene, o, d), rtol=1e-10, atol=1e-12)
        items = scenes.batch_workload(count=6, seed=3)
        imgs = sharding.render_batch_sharded([sc.build() for sc, _ in items], [op for _, op in items])
        for (sc, op), im in zip(items, imgs):
            assert im.tobytes() == zt.render(sc, op).pixels.tobytes()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("seed", range(3))
def test_forward_at_own_colors_on_fuzz_scenes(seed):
    import kat_scenes as K
    scene = K.fuzz_scene(seed).build()
    o = zt.Options(32, 20, 3, 12, seed=seed)
    assert zt.forward(scene, o).pixels.tobytes() == zt.render(scene, o).pixels.tobytes()


def test_backward_after_a_second_view_uses_its_own_primal():
    """Forward view A, forward view B, backward A: the primal kept by the last
    forward belongs to view B, so the backward of A must not reuse it; the
    gradient equals backward A computed with no cache at all."""
    scene, _, o = small()
    theta = np.array([m["color"] for m in scene.materials])
    w = _weights(o)
    view_a = scene.camera
    view_b = zt.CameraConfig(look_from=(300, 250, -700), look_at=(270, 270, 0), vfov=42)
    zt.forward(scene, o, theta)                      # A
    scene.camera = view_b
    zt.forward(scene, o, theta)                      # B: its primal replaces A's
    scene.camera = view_a
    warm = zt.backward(scene, o, w, theta)           # A again
    scene.set_primal_cache_limit(0)                  # no cache: the backward traces its own primal
    cold = zt.backward(scene, o, w, theta)
    tol = dict(rtol=1e-9, atol=1e-12 * np.abs(cold).max())  # atomics add in varying order
    np.testing.assert_allclose(warm, cold, **tol)
    scene.background = zt.Background.solid((0.2, 0.3, 0.4))  # the same for a background change
    scene.set_primal_cache_limit(1 << 30)
    zt.forward(scene, o, theta)
    scene.background = zt.Background.solid((0.0, 0.0, 0.0))
    np.testing.assert_allclose(zt.backward(scene, o, w, theta), cold, **tol)


def test_primal_cache_off_at_full_hd_matches_cached():
    """1920x1080x64 (3.2 GB of primal radiance, above the default 1 GiB cache
    limit, so the default backward recomputes the primal) against the same
    backward with the cache raised to hold it."""
    scene, target = scenes.cornell_diff()
    scene.build()
    o = zt.Options(1920, 1080, 64, 8)
    theta = np.array([m["color"] for m in scene.materials])
    w = np.random.default_rng(9).uniform(-1, 1, (o.width * o.height, 3))
    img = zt.forward(scene, o, theta).pixels
    recomputed = zt.backward(scene, o, w, theta)
    scene.set_primal_cache_limit(4 << 30)
    assert zt.forward(scene, o, theta).pixels.tobytes() == img.tobytes()
    cached = zt.backward(scene, o, w, theta)
    np.testing.assert_allclose(cached, recomputed, rtol=1e-9, atol=1e-12 * np.abs(recomputed).max())
    assert np.abs(cached).max() > 0
