"""Seeded synthetic particle sets of the benchmark configurations.

The distributions of the field-solver benchmarks (there is no public dataset):
positions are drawn with ``numpy.random.default_rng(seed)`` and points outside the
root cell [-1, 1]^2 are drawn again (rejection, not clipping, which would pile points
onto the corners as coincident charges).

* ``uniform(n)``: uniform in [-1, 1]^2, charges +1/-1 equiprobable (config 1);
* ``gaussian(n, sigma)``: a 2D Gaussian, charges +1/-1 (config 2);
* ``mixture8(n)``: 8 Gaussians, centres uniform in [-0.8, 0.8]^2, sigma linspace(0.02,
  0.2, 8), uniform labels; charges +1/-1 with exactly n/2 of each (config 3);
* ``protons(n)``: positions N(0, 0.1^2), charges 1 (config 5).
"""

from __future__ import annotations

import numpy as np


def _redraw(rng, draw, n: int) -> np.ndarray:
    out = np.empty((2, 0))
    while out.shape[1] < n:
        pts = draw(n - out.shape[1] + 1024)
        keep = np.all(np.abs(pts) < 1.0, axis=0)
        out = np.concatenate((out, pts[:, keep]), axis=1)
    return np.ascontiguousarray(out[:, :n])


def _signs(rng, n: int) -> np.ndarray:
    return rng.choice([-1.0, 1.0], n)


def uniform(n: int, seed: int = 0):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1, 1, (2, n)), _signs(rng, n)


def gaussian(n: int, sigma: float = 0.3, seed: int = 0):
    rng = np.random.default_rng(seed)
    pos = _redraw(rng, lambda k: rng.normal(0, sigma, (2, k)), n)
    return pos, _signs(rng, n)


def mixture8(n: int, seed: int = 0):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-0.8, 0.8, (8, 2))
    sigmas = np.linspace(0.02, 0.2, 8)

    def draw(k):
        label = rng.integers(0, 8, k)
        return (centres[label] + sigmas[label, None] * rng.normal(size=(k, 2))).T

    pos = _redraw(rng, draw, n)
    charge = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    return pos, charge[rng.permutation(n)]


def protons(n: int, seed: int = 0):
    rng = np.random.default_rng(seed)
    pos = _redraw(rng, lambda k: rng.normal(0, 0.1, (2, k)), n)
    return pos, np.ones(n)
