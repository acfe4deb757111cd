"""CPU checks of small oracle pieces."""
from __future__ import annotations

from fractions import Fraction

import numpy as np

import oracle


def test_resolve_layers_is_the_rounded_exact_mean():
    """renderer/triangle.frag:14-23: mean of the layers' rgb, alpha 1; the
    oracle rounds the exact mean to nearest, ties up."""
    rng = np.random.default_rng(0)
    for n in (1, 2, 3, 8):
        layers = rng.integers(0, 256, (n, 3, 5, 4), dtype=np.uint8)
        got = oracle.resolve_layers(layers)
        assert (got[..., 3] == 255).all()
        for y in range(3):
            for x in range(5):
                for c in range(3):
                    mean = Fraction(int(layers[:, y, x, c].astype(int).sum()), n)
                    want = int(mean + Fraction(1, 2))  # floor(mean + 1/2): ties up
                    assert got[y, x, c] == want
