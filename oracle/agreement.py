"""Statistical agreement of two renders of the same scene, options and seed
(test infrastructure; only tests and the benchmark's CPU legs use it).

The bar is the one set for renders that are not bit-identical to the
reference algorithm (the fast traversal): per-channel relative RMSE
sqrt(mean((g - c)^2)) / mean(c) below 1e-3, and the mean luminance
(0.2126 r + 0.7152 g + 0.0722 b, the weights of src/light.zig:38-40) within
3 Monte Carlo standard errors of the oracle's, the standard error coming
from the oracle's per-pixel second moment of sample luminance.
"""
from __future__ import annotations

import numpy as np

LUMINANCE = np.array([0.2126, 0.7152, 0.0722])
RMSE_BAR = 1e-3
SE_BAR = 3.0


def image_agreement(gpu: np.ndarray, cpu: np.ndarray, m2: np.ndarray, spp: int) -> dict:
    """gpu, cpu: (n_pixels, 3) images; m2: per-pixel mean squared sample
    luminance of the cpu render (oracle render_moments / render_pixels_moments)."""
    g = np.asarray(gpu, np.float64).reshape(-1, 3)
    c = np.asarray(cpu, np.float64).reshape(-1, 3)
    n = len(c)
    rmse = np.sqrt(((g - c) ** 2).mean(axis=0)) / np.maximum(np.abs(c.mean(axis=0)), 1e-300)
    lum_g, lum_c = g @ LUMINANCE, c @ LUMINANCE
    var = np.maximum(m2 - lum_c ** 2, 0.0) * (spp / max(spp - 1, 1))  # per-pixel sample variance
    se = float(np.sqrt((var / spp).sum()) / n)
    dl = float(abs(lum_g.mean() - lum_c.mean()))
    ident = float((g == c).all(axis=1).mean())
    return {"rel_rmse": [float(x) for x in rmse], "max_rel_rmse": float(rmse.max()),
            "mean_luminance_gpu": float(lum_g.mean()), "mean_luminance_cpu": float(lum_c.mean()),
            "luminance_se": se, "luminance_diff_in_se": dl / se if se > 0 else (0.0 if dl == 0 else float("inf")),
            "identical_pixels": ident,
            "ok": bool(rmse.max() < RMSE_BAR and (dl <= SE_BAR * se))}
