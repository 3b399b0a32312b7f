"""Autotuner for the device execution choices.

For a render it times the megakernel at block sizes 64/128/256, the
megakernel with path regeneration at 128/256, the wavefront form at three
queue capacities (paths in flight: the default of one slot per pixel up to
4M, 1M and 256K) and the sorted wavefront form at two.  For a batch it times the batched persistent launch
at block sizes 64/128/256 with the renders in the given order or largest
first, its path-regeneration form at block sizes 128/256, and the same
renders as plain per-render launches (each with its own default choice) as
one more candidate.  Every candidate renders identical
pixels at the caller's precision (the choice only changes scheduling), so
the fastest one is kept; the precision itself is the caller's choice and is
part of the cache key, since the exact and fast builds differ in their best
configuration.  Results are cached per (GPU, scene class) in a JSON file, by
default ``~/.cache/zigtrace_b200/autotune.json`` (override with
ZT_AUTOTUNE_CACHE).
"""
from __future__ import annotations

import json
import math
import os
import statistics
from pathlib import Path
from typing import Callable, Dict, List, Optional, Sequence, Tuple

from .api import MODE_MEGAKERNEL, MODE_MEGAKERNEL_REGEN, MODE_WAVEFRONT, MODE_WAVEFRONT_SORTED, Batch, GpuConfig, Options, Scene, render_device

SINGLE_CANDIDATES: List[Tuple[int, int, int]] = [  # (mode, block_size, queue_capacity)
    (MODE_MEGAKERNEL, 64, 0), (MODE_MEGAKERNEL, 128, 0), (MODE_MEGAKERNEL, 256, 0),
    (MODE_MEGAKERNEL_REGEN, 128, 0), (MODE_MEGAKERNEL_REGEN, 256, 0),
    (MODE_WAVEFRONT, 128, 0), (MODE_WAVEFRONT, 128, 1 << 20), (MODE_WAVEFRONT, 128, 1 << 18),
    (MODE_WAVEFRONT_SORTED, 128, 0), (MODE_WAVEFRONT_SORTED, 128, 1 << 20)]
PLAIN = -1  # batch candidate: plain per-render launches instead of the batched launch
BATCH_CANDIDATES: List[Tuple[int, int, int]] = (  # (block_size, order, mode)
    [(bs, order, MODE_MEGAKERNEL) for bs in (64, 128, 256) for order in (0, 1)] +
    [(128, 1, MODE_MEGAKERNEL_REGEN), (256, 1, MODE_MEGAKERNEL_REGEN)] + [(PLAIN, 0, MODE_MEGAKERNEL)])


def cache_path() -> Path:
    return Path(os.environ.get("ZT_AUTOTUNE_CACHE", str(Path.home() / ".cache" / "zigtrace_b200" / "autotune.json")))


def _load() -> Dict:
    try:
        return json.loads(cache_path().read_text())
    except (OSError, ValueError):
        return {}


def _store(key: str, entry: Dict) -> None:
    data = _load()
    data[key] = entry
    p = cache_path()
    p.parent.mkdir(parents=True, exist_ok=True)
    tmp = p.with_suffix(".tmp")
    tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
    tmp.replace(p)


def gpu_key() -> str:
    import torch
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return f"{p.name}|sm{p.major}{p.minor}|{p.multi_processor_count}SM"


def _mag(x: float) -> int:
    return int(round(math.log10(max(x, 1.0))))


def scene_class(scene: Scene, opts: Options, precision: int = 0) -> str:
    """Coarse class of a render: orders of magnitude of primitives and
    pixels, whether it has lights and planes, spp, depth, light sampling and
    precision.  The Cornell box (1e1 primitives, lights, 256x256x64), the
    random spheres (1e2, a plane, no lights, depth 50) and the 1M-triangle
    terrain (1e6, lights) fall in different classes."""
    c = scene.counts()
    return (f"prims1e{_mag(c['bounded'] + c['planes'])}|planes{int(c['planes'] > 0)}|lights{int(c['lights'] > 0)}"
            f"|px1e{_mag(opts.width * opts.height)}|spp{opts.spp}|depth{opts.max_depth}"
            f"|nee{int(opts.light_sampling)}|prec{precision}")


def batch_class(scenes: Sequence[Scene], opts: Sequence[Options], precision: int = 0) -> str:
    px = sum(o.width * o.height for o in opts)
    prims = sum(s.counts()["bounded"] for s in scenes) / len(scenes)
    return (f"batch|n{len(scenes)}|px1e{_mag(px)}|meanprims1e{_mag(prims)}|spp{opts[0].spp}"
            f"|depth{opts[0].max_depth}|prec{precision}")


def _event_timer(fn: Callable[[], None], reps: int) -> float:
    """Median device milliseconds of fn() on the current stream."""
    import torch
    stream = torch.cuda.current_stream()
    fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    return statistics.median(times)


def choose(key: str, candidates: Sequence, run: Callable, reps: int = 2, use_cache: bool = True,
           timer: Callable[[Callable[[], None], int], float] = _event_timer):
    """Returns the fastest candidate for `key`, timing each with run(c) once
    per rep unless the cache already holds a choice."""
    if use_cache:
        hit = _load().get(key)
        if hit is not None and hit.get("best") is not None:
            return tuple(hit["best"]), hit["ms"], True
    ms = {}
    for c in candidates:
        ms[json.dumps(list(c))] = timer(lambda: run(c), reps)
    best = min(ms, key=ms.get)
    _store(key, {"best": json.loads(best), "ms": ms})
    return tuple(json.loads(best)), ms, False


def tune_render(scene: Scene, opts: Options, reps: int = 2, use_cache: bool = True, precision: int = 0,
                candidates: Optional[Sequence[Tuple[int, int, int]]] = None) -> Tuple[GpuConfig, Dict, bool]:
    """Fastest device configuration for rendering `scene` with `opts` at
    `precision`; returns (config, timings in ms per candidate, whether the
    choice came from the cache)."""
    import torch
    scene.upload()
    out = torch.empty(opts.width * opts.height * 3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def run(c):
        render_device(scene, opts, out.data_ptr(), stream,
                      GpuConfig(mode=c[0], block_size=c[1], queue_capacity=c[2], precision=precision))

    best, ms, cached = choose(f"{gpu_key()}|render|{scene_class(scene, opts, precision)}",
                              candidates or SINGLE_CANDIDATES, run, reps, use_cache)
    del out
    return GpuConfig(mode=best[0], block_size=best[1], queue_capacity=best[2], precision=precision), ms, cached


def tune_batch(scenes: Sequence[Scene], opts: Sequence[Options], reps: int = 2,
               use_cache: bool = True, precision: int = 0) -> Tuple[GpuConfig, int, Dict, bool]:
    """Fastest (block size, order) for a batch at `precision`; order is PLAIN
    when per-render launches beat every batched launch.  Returns (config,
    order, timings in ms, whether it came from the cache)."""
    import torch
    outs = [torch.empty(o.width * o.height * 3, dtype=torch.float64, device="cuda") for o in opts]
    stream = torch.cuda.current_stream().cuda_stream
    batches = {}

    def run(c):
        if c[0] == PLAIN:
            for s, o, t in zip(scenes, opts, outs):
                render_device(s, o, t.data_ptr(), stream, GpuConfig(precision=precision))
            return
        if c not in batches:
            batches[c] = Batch(scenes, opts, [t.data_ptr() for t in outs],
                               GpuConfig(mode=c[2], block_size=c[0], precision=precision), order=c[1])
        batches[c].launch(stream)

    best, ms, cached = choose(f"{gpu_key()}|{batch_class(scenes, opts, precision)}", BATCH_CANDIDATES, run, reps,
                              use_cache)
    torch.cuda.synchronize()
    for b in batches.values():
        b.close()
    if best[0] == PLAIN:
        return GpuConfig(precision=precision), PLAIN, ms, cached
    return GpuConfig(mode=best[2], block_size=best[0], precision=precision), best[1], ms, cached
