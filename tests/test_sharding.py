"""Row sharding across ranks: band arithmetic, and a world-size-2 gloo run on
CPU whose bands are rendered by the oracle and gathered by render_sharded;
the gathered image must equal the one-process render bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from zigtrace_b200 import sharding


def test_row_bands_cover_every_row_once():
    for h in (1, 2, 7, 256, 1080):
        for world in (1, 2, 3, 8):
            bands = sharding.row_bands(h, world)
            assert len(bands) == world and bands[0][0] == 0 and bands[-1][1] == h
            assert all(a <= b for a, b in bands) and all(bands[i][1] == bands[i + 1][0] for i in range(world - 1))


def test_row_bands_balance_costs():
    costs = np.ones(100)
    costs[:20] = 10.0  # expensive top rows
    bands = sharding.row_bands(100, 2, costs)
    a = costs[bands[0][0]:bands[0][1]].sum()
    b = costs[bands[1][0]:bands[1][1]].sum()
    assert abs(a - b) <= 10.0 and bands[0][1] < 50
    with pytest.raises(ValueError):
        sharding.row_bands(10, 2, np.ones(9))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, result_path):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / "tests"))
    import torch.distributed as dist
    import oracle as O
    import kat_scenes as K
    from zigtrace_b200 import sharding as S

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    scene = K.demo_scene()
    opts = K.kat_options(width=30, height=17, spp=3)
    o = type("O", (), {"width": 30, "height": 17})()
    os_ = O.OracleScene.from_scene(scene)

    def band(_scene, _o, y0, y1):  # the oracle stands in for the GPU band render
        pix = np.arange(y0 * 30, y1 * 30, dtype=np.uint64)
        return os_.render_pixels(30, 17, opts["spp"], opts["max_depth"], pix, threads=1)

    img = S.render_sharded(scene, o, render_band=band, row_costs=np.linspace(1, 5, 17))
    if rank == 0:
        np.save(result_path, img)
    dist.destroy_process_group()


def test_render_sharded_gloo_world_2(tmp_path):
    import kat_scenes as K
    import oracle as O
    path = str(tmp_path / "img.npy")
    mp.spawn(_worker, args=(2, _free_port(), path), nprocs=2, join=True)
    got = np.load(path)
    o = K.kat_options(width=30, height=17, spp=3)
    want = O.OracleScene.from_scene(K.demo_scene()).render(o["width"], o["height"], o["spp"], o["max_depth"])
    assert got.tobytes() == want.tobytes()


def test_assign_batch_lpt():
    rng = np.random.default_rng(1)
    for world in (1, 2, 3, 8):
        costs = rng.exponential(1.0, 50)
        parts = sharding.assign_batch(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(50))
        loads = [costs[p].sum() if p else 0.0 for p in parts]
        assert max(loads) <= costs.sum() / world + costs.max() + 1e-9  # LPT bound
        assert parts == sharding.assign_batch(costs, world)  # deterministic
    assert sharding.assign_batch([1.0], 3) == [[0], [], []]


def _grad_worker(rank, world, port, result_path):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / "tests"))
    import torch.distributed as dist
    import kat_scenes as K
    from zigtrace_b200 import sharding as S

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    scene = K.demo_scene()
    o = type("O", (), {"width": 6, "height": 7})()
    d_image = np.arange(6 * 7 * 3, dtype=np.float64).reshape(-1, 3)
    n = 3 * len(scene.materials)

    def band(_scene, _o, y0, y1, d_band):  # a stand-in share: linear in the band's dL/dpixels
        assert d_band.shape == ((y1 - y0) * 6, 3)
        return np.arange(1, n + 1, dtype=np.float64) * d_band.sum()

    g = S.backward_sharded(scene, o, d_image, backward_band=band, row_costs=np.linspace(1, 3, 7))
    items = [(k, k + 1) for k in range(5)]
    imgs = S.render_batch_sharded([None] * 5, items, costs=[3, 1, 4, 1, 5],
                                  render_item=lambda _sc, wh: np.full((wh[0] * wh[1], 3), float(wh[0])))
    if rank == 0:
        np.save(result_path, np.concatenate([g.reshape(-1)] + [im.reshape(-1) for im in imgs]))
    dist.destroy_process_group()


def test_backward_and_batch_sharded_gloo_world_2(tmp_path):
    import kat_scenes as K
    path = str(tmp_path / "g.npy")
    mp.spawn(_grad_worker, args=(2, _free_port(), path), nprocs=2, join=True)
    got = np.load(path)
    n = 3 * len(K.demo_scene().materials)
    total = np.arange(6 * 7 * 3, dtype=np.float64).sum()
    assert np.allclose(got[:n], np.arange(1, n + 1) * total, rtol=0, atol=1e-9)
    want = np.concatenate([np.full((k * (k + 1), 3), float(k)).reshape(-1) for k in range(5)])
    assert got[n:].tobytes() == want.tobytes()
