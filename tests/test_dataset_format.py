"""Sampling formulas of the audio-dataset generator (the reference's
experiments/neuPAT_audio/generate.py:85-99), on CPU."""
import math

import numpy as np
import pytest

from neuralat_b200.bem import dataset as D


def test_shell_points_follow_the_reference_mapping():
    rng = np.random.default_rng(3)
    base = rng.random((50, 3))
    center, r, rmax = (0.1, -0.2, 0.3), 0.25, 3.0
    pts = D.shell_points(base, center, r, rmax)
    rs = (base[:, 0] * (rmax - 1) + 1) * r
    theta = base[:, 1] * 2 * math.pi - math.pi
    phi = base[:, 2] * math.pi
    ref = np.stack([rs * np.sin(phi) * np.cos(theta), rs * np.sin(phi) * np.sin(theta), rs * np.cos(phi)], -1)
    np.testing.assert_allclose(pts - np.asarray(center), ref, rtol=0, atol=1e-12)
    dist = np.linalg.norm(pts - np.asarray(center), axis=1)
    assert np.all(dist >= r - 1e-12) and np.all(dist <= rmax * r + 1e-12)


@pytest.mark.parametrize("fraction,expected", [(0.0, 100.0), (0.5, 1000.0), (1.0, 10000.0)])
def test_log_frequency(fraction, expected):
    assert D.log_frequency(fraction, 100.0, 10000.0) == pytest.approx(expected)
