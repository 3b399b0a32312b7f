"""The statistical bar for renders that are not bit-identical to the
reference algorithm (oracle/agreement.py), on the CPU: identical renders
pass, a render at another seed or with a planted 1% bias in the oracle's
image fails, and the second-moment buffer is consistent with the image."""
import numpy as np

import oracle as O
from oracle.agreement import image_agreement
from zigtrace_b200 import scenes


def _cornell(spp=8, seed=0):
    os_ = O.OracleScene.from_scene(scenes.cornell())
    return os_, os_.render_moments(48, 48, spp, 16, seed=seed)


def test_identical_renders_agree():
    _, (img, m2) = _cornell()
    a = image_agreement(img, img, m2, 8)
    assert a["ok"] and a["max_rel_rmse"] == 0 and a["identical_pixels"] == 1.0


def test_other_seed_fails_the_rmse_bar():
    os_, (img, m2) = _cornell()
    other = os_.render(48, 48, 8, 16, seed=1)
    a = image_agreement(other, img, m2, 8)
    assert not a["ok"] and a["max_rel_rmse"] > 0.1


def test_planted_bias_fails():
    _, (img, m2) = _cornell(spp=64)
    biased = img * 1.01  # a 1% error planted in a copy of the oracle's image
    a = image_agreement(biased, img, m2, 64)
    assert not a["ok"] and a["max_rel_rmse"] > 5e-3


def test_second_moment_bounds_the_pixel_luminance():
    _, (img, m2) = _cornell()
    lum = img @ np.array([0.2126, 0.7152, 0.0722])
    assert (m2 >= lum ** 2 * (1 - 1e-12)).all()  # E[l^2] >= E[l]^2 pixel by pixel
    assert m2.mean() > 0
