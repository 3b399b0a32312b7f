"""Work split across GPUs, one process per GPU.

Pixels are independent (each owns its RNG stream, src/render.zig:135), so
rank r renders a contiguous band of image rows straight into its slot of a
device buffer (zt_render_rows_device) and one all-gather over
torch.distributed (NCCL on GPUs, gloo on CPU) assembles the frame in device
memory.  The gathered image is bit-identical to a one-device render.
Bands can be balanced by a per-row cost estimate (e.g. the previous frame's
per-row times); without one they split the rows evenly.

The differentiable form splits the same way: each rank runs the forward and
the path-replay backward of its band (zt_forward_rows / zt_backward_rows)
and one all-reduce sums the gradient shares (3 values per material).  A
batch of renders is split by estimated cost, longest first onto the least
loaded rank (LPT), rendered as one batched launch per rank, and gathered
with one tensor all-gather on every rank.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .api import Options, Scene, backward_rows, forward_rows, render


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
    """Rows [y0, y1) of the image on the current device, into host memory
    ((y1-y0)*width x 3)."""
    out = np.zeros(max(y1 - y0, 0) * int(opts.width) * 3 + 1, np.float64)  # the C ABI validates the band
    N.check(N.lib().zt_render_rows(scene.handle, N.ptr(opts.record()), y0, y1, N.ptr(out)))
    return out[:-1].reshape(-1, 3)


def _device(group):
    import torch
    import torch.distributed as dist
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")


def _gather_padded(buf, world: int, group):
    """All-gather of equal-sized flat tensors into one (world * len) tensor:
    all_gather_into_tensor on NCCL, the list form elsewhere (gloo)."""
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        out = torch.empty(world * buf.numel(), dtype=buf.dtype, device=buf.device)
        dist.all_gather_into_tensor(out, buf, group=group)
        return out
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return torch.cat(parts)


def render_sharded(scene: Scene, opts: Options, group=None,
                   render_band: Optional[Callable[[Scene, Options, int, int], np.ndarray]] = None,
                   row_costs: Optional[Sequence[float]] = None, gpu=None, as_numpy: bool = True, stream=None):
    """Renders the image across the ranks of `group`; every rank gets the
    whole (height*width x 3) image.

    By default each rank renders its band on its GPU straight into its slot
    of the all-gather buffer (zt_render_rows_device) and one all-gather
    assembles the frame in device memory, with no host round trip; with
    as_numpy=False the image stays on the device (a torch tensor).
    `render_band` substitutes another band renderer returning host rows
    (the CPU tests use the oracle)."""
    import torch
    import torch.distributed as dist

    from .api import render_rows_device

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    height, width = int(opts.height), int(opts.width)
    bands = row_bands(height, world, row_costs)
    y0, y1 = bands[rank]
    max_rows = max(b - a for a, b in bands)
    device = _device(group)
    buf = torch.zeros(max_rows * width * 3, dtype=torch.float64, device=device)
    if y1 > y0:
        if render_band is not None:
            mine = np.ascontiguousarray(render_band(scene, opts, y0, y1), np.float64).reshape(-1)
            buf[:mine.size] = torch.from_numpy(mine).to(device)
        else:
            st = stream if stream is not None else torch.cuda.current_stream()
            render_rows_device(scene, opts, y0, y1, buf.data_ptr(), st.cuda_stream, gpu)
    gathered = _gather_padded(buf, world, group)
    stride = max_rows * width * 3
    img = torch.cat([gathered[r * stride:r * stride + (b - a) * width * 3] for r, (a, b) in enumerate(bands)])
    img = img.view(height * width, 3)
    return img.cpu().numpy() if as_numpy else img


def forward_sharded(scene: Scene, opts: Options, colors=None, group=None, row_costs=None,
                    forward_band: Optional[Callable] = None) -> np.ndarray:
    """forward() across the ranks of `group`: each rank's band by
    zt_forward_rows, gathered as render_sharded does."""
    band = forward_band or (lambda sc, o, y0, y1: forward_rows(sc, o, y0, y1, colors))
    return render_sharded(scene, opts, group, render_band=band, row_costs=row_costs)


def backward_sharded(scene: Scene, opts: Options, d_image, colors=None, group=None, row_costs=None,
                     backward_band: Optional[Callable] = None) -> np.ndarray:
    """backward() across the ranks of `group`: each rank computes the
    gradient share of its band of rows, then one all-reduce sums the shares
    (n_materials x 3 on every rank)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    width = int(opts.width)
    y0, y1 = row_bands(int(opts.height), world, row_costs)[rank]
    g = np.asarray(d_image, np.float64).reshape(-1, 3)
    band = backward_band or (lambda sc, o, a, b, d: backward_rows(sc, o, a, b, d, colors))
    n = 3 * len(scene.materials)
    share = band(scene, opts, y0, y1, g[y0 * width:y1 * width]) if y1 > y0 else np.zeros(n)
    device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")
    t = torch.from_numpy(np.ascontiguousarray(share, np.float64).reshape(-1).copy()).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy().reshape(-1, 3)


def assign_batch(costs: Sequence[float], world: int) -> List[List[int]]:
    """Longest-processing-time assignment: renders in decreasing cost (ties by
    index) each go to the rank with the least assigned cost so far (ties to
    the lower rank).  Returns the indices each rank renders, in input order."""
    if world < 1:
        raise ValueError("world must be positive")
    c = np.asarray(costs, np.float64)
    load = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(c)), key=lambda k: (-c[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += float(c[i])
    return [sorted(p) for p in parts]


def batch_costs(scenes: Sequence[Scene], opts_list: Sequence[Options]) -> List[float]:
    """Cost estimate of each render: samples x log2(primitives + 2)."""
    out = []
    for sc, o in zip(scenes, opts_list):
        n = sc.counts()["bounded"] + sc.counts()["planes"]
        out.append(float(o.width * o.height * o.spp) * float(np.log2(n + 2)))
    return out


def render_batch_sharded(scenes: Sequence[Scene], opts_list: Sequence[Options], group=None,
                         costs: Optional[Sequence[float]] = None,
                         render_item: Optional[Callable] = None, gpu=None, as_numpy: bool = True):
    """Renders a batch across the ranks of `group` (LPT by cost) and returns
    every image (height*width x 3), in input order, on every rank.

    Each rank renders its renders as one persistent batched launch into one
    flat device buffer (its images back to back, in index order); the
    buffers, padded to the largest, are gathered with one tensor all-gather,
    and every rank cuts the images out of the result (all ranks know the
    assignment and the sizes).  `render_item` substitutes another renderer
    returning host arrays (the CPU tests)."""
    import torch
    import torch.distributed as dist

    from .api import Batch

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    costs = batch_costs(scenes, opts_list) if costs is None else costs
    parts = assign_batch(costs, world)
    sizes = [int(o.width) * int(o.height) * 3 if not isinstance(o, tuple) else int(o[0]) * int(o[1]) * 3
             for o in opts_list]
    totals = [sum(sizes[i] for i in p) for p in parts]
    device = _device(group)
    buf = torch.zeros(max(max(totals), 1), dtype=torch.float64, device=device)
    mine = parts[rank]
    offs, cur = {}, 0
    for i in mine:
        offs[i] = cur
        cur += sizes[i]
    if mine:
        if render_item is not None:
            for i in mine:
                img = np.ascontiguousarray(render_item(scenes[i], opts_list[i]), np.float64).reshape(-1)
                buf[offs[i]:offs[i] + sizes[i]] = torch.from_numpy(img).to(device)
        else:
            for i in mine:
                scenes[i].upload()
            batch = Batch([scenes[i] for i in mine], [opts_list[i] for i in mine],
                          [buf.data_ptr() + 8 * offs[i] for i in mine], gpu)
            batch.launch(torch.cuda.current_stream().cuda_stream)
            batch.close()
    gathered = _gather_padded(buf, world, group)
    stride = buf.numel()
    images: list = [None] * len(scenes)
    for r, p in enumerate(parts):
        cur = r * stride
        for i in p:
            img = gathered[cur:cur + sizes[i]].view(-1, 3)
            images[i] = img.cpu().numpy() if as_numpy else img
            cur += sizes[i]
    return images
