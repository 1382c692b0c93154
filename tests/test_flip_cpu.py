"""The LDR-FLIP restatement used to grade rendered frames (tests/flip.py)."""
import numpy as np

import flip


def test_identical_images_score_zero():
    img = np.random.default_rng(1).uniform(0, 1, (24, 32, 3))
    assert flip.mean_flip(img, img) == 0.0


def test_scores_grow_with_the_difference_and_stay_in_unit_range():
    rng = np.random.default_rng(2)
    img = rng.uniform(0.2, 0.8, (32, 32, 3))
    small = flip.mean_flip(img, np.clip(img + rng.normal(0, 0.01, img.shape), 0, 1))
    large = flip.mean_flip(img, np.clip(img + rng.normal(0, 0.1, img.shape), 0, 1))
    black_white = flip.flip_map(np.zeros((16, 16, 3)), np.ones((16, 16, 3)))
    assert 0.0 < small < large < 1.0
    assert black_white.min() > 0.5 and black_white.max() <= 1.0


def test_colour_error_maximum_is_green_against_blue():
    g = np.zeros((16, 16, 3)); g[..., 1] = 1.0
    b = np.zeros((16, 16, 3)); b[..., 2] = 1.0
    assert abs(flip.mean_flip(g, b) - 1.0) < 1e-6
