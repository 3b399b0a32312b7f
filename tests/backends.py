"""Two implementations of the reference's render API for shared tests:
the CPU oracle and the GPU path.  The reference's render-level tests are
written once against this interface and run on both."""
from __future__ import annotations

import numpy as np

import oracle as O
import zigtrace_b200 as zt


class OracleBackend:
    name = "oracle"

    def render(self, scene: zt.Scene, width, height, spp, max_depth, threads=1, seed=0, tile_size=16,
               light_sampling=True) -> np.ndarray:
        return O.OracleScene.from_scene(scene).render(width, height, spp, max_depth, threads=threads, seed=seed,
                                                      tile_size=tile_size, light_sampling=light_sampling)

    def mean_radiance(self, scene: zt.Scene, origin, direction, seed, n, max_depth, nee) -> np.ndarray:
        """Per-path radiance of meanRadiance (render.zig:290-302)."""
        os_ = O.OracleScene.from_scene(scene)
        rng = O.Rng.init(seed)
        return np.array([os_.trace_with(origin, direction, rng, max_depth, nee) for _ in range(n)])

    def trace_with(self, scene, origin, direction, rng_state, max_depth, nee):
        os_ = O.OracleScene.from_scene(scene)
        rng = O.Rng(rng_state)
        out = os_.trace_with(origin, direction, rng, max_depth, nee)
        rng_state[:] = rng.s
        return out


class GpuBackend:
    name = "gpu"

    def __init__(self, mode: int = zt.MODE_MEGAKERNEL):
        self.mode = mode

    def render(self, scene: zt.Scene, width, height, spp, max_depth, threads=1, seed=0, tile_size=16,
               light_sampling=True) -> np.ndarray:
        scene.build()
        opts = zt.Options(width=width, height=height, spp=spp, max_depth=max_depth, threads=threads, seed=seed,
                          tile_size=tile_size, light_sampling=light_sampling)
        return zt.render(scene, opts, zt.GpuConfig(mode=self.mode)).pixels

    def mean_radiance(self, scene: zt.Scene, origin, direction, seed, n, max_depth, nee) -> np.ndarray:
        scene.build()
        state = O.Rng.init(seed).s.copy()
        return zt.api.trace_paths(scene, origin, direction, state, n, max_depth, nee)

    def trace_with(self, scene, origin, direction, rng_state, max_depth, nee):
        scene.build()
        return zt.api.trace_paths(scene, origin, direction, rng_state, 1, max_depth, nee)[0]
