"""One image across several GPUs, one process per GPU.

Pixels are independent (each owns its RNG stream, src/render.zig:135), so
rank r renders a contiguous band of image rows with zt_render_rows and the
bands are gathered with one all-gather over torch.distributed (NCCL on GPUs,
gloo on CPU).  The gathered image is bit-identical to a one-device render.
Bands can be balanced by a per-row cost estimate (e.g. the previous frame's
per-row times); without one they split the rows evenly.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .api import Options, Scene


def row_bands(height: int, world: int, row_costs: Optional[Sequence[float]] = None) -> List[Tuple[int, int]]:
    """Contiguous [y0, y1) bands, one per rank, covering every row once.
    With row_costs, each band holds about 1/world of the total cost."""
    if world < 1 or height < 1:
        raise ValueError("height and world must be positive")
    if row_costs is None:
        edges = [(height * r) // world for r in range(world + 1)]
    else:
        c = np.asarray(row_costs, np.float64)
        if c.shape != (height,) or (c < 0).any():
            raise ValueError("row_costs needs one non-negative value per row")
        cum = np.concatenate([[0.0], np.cumsum(c)])
        total = cum[-1]
        edges = [0]
        for r in range(1, world):
            y = int(np.searchsorted(cum, total * r / world, side="left")) if total > 0 else (height * r) // world
            edges.append(min(max(y, edges[-1]), height))
        edges.append(height)
    return [(edges[r], edges[r + 1]) for r in range(world)]


def render_rows(scene: Scene, opts: Options, y0: int, y1: int) -> np.ndarray:
    """Rows [y0, y1) of the image on the current device ((y1-y0)*width x 3)."""
    out = np.zeros(max(y1 - y0, 0) * int(opts.width) * 3 + 1, np.float64)  # the C ABI validates the band
    N.check(N.lib().zt_render_rows(scene.handle, N.ptr(opts.record()), y0, y1, N.ptr(out)))
    return out[:-1].reshape(-1, 3)


def render_sharded(scene: Scene, opts: Options, group=None,
                   render_band: Callable[[Scene, Options, int, int], np.ndarray] = render_rows,
                   row_costs: Optional[Sequence[float]] = None) -> np.ndarray:
    """Renders the image across the ranks of `group` and returns the whole
    (height*width x 3) image on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    bands = row_bands(int(opts.height), world, row_costs)
    y0, y1 = bands[rank]
    width = int(opts.width)
    mine = render_band(scene, opts, y0, y1) if y1 > y0 else np.zeros((0, 3))
    max_rows = max(b - a for a, b in bands)
    device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")
    buf = torch.zeros(max_rows * width * 3, dtype=torch.float64, device=device)
    if len(mine):
        buf[:mine.size] = torch.from_numpy(np.ascontiguousarray(mine).reshape(-1)).to(device)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    img = np.empty((int(opts.height) * width, 3), np.float64)
    for (a, b), part in zip(bands, parts):
        n = (b - a) * width
        img[a * width:b * width] = part[:n * 3].cpu().numpy().reshape(-1, 3)
    return img
