"""Pins the oracle's smoothgradient (Gaussian smoothing of the summed gradient when
ExtraParams.smoothgradkern > 0; src/EikSolv/utils.jl:22-96) to an independent statement
of the same operator: the reference pads the gradient with zeros, correlates it with the
normalised l^d kernel exp(-r^2/(2s)), s = l/2 - sqrt(l/2), and crops, which is scipy's
zero-padded correlation. The two sum in different orders, so they agree to rounding."""
import numpy as np
import pytest
from scipy import ndimage

import eikoracle as O
from eikonalsolvers import Grid2DCart, Grid3DCart


def _kernel(l, dim):
    pos = np.arange(l) - l // 2
    grids = np.meshgrid(*([pos] * dim), indexing="ij")
    r = np.sqrt(sum(g.astype(np.float64) ** 2 for g in grids))
    s = l / 2 - np.sqrt(l / 2)
    k = np.exp(-r ** 2 / (2.0 * s))
    return k / k.sum()


@pytest.mark.parametrize("l", [1, 3, 5, 9])
@pytest.mark.parametrize("shape", [(23, 17), (11, 9, 13)])
def test_oracle_smoothgradient_is_the_zero_padded_gaussian_correlation(l, shape):
    grd = Grid2DCart(hgrid=0.5, cooinit=(0.0, 0.0), grsize=shape) if len(shape) == 2 else \
        Grid3DCart(hgrid=0.5, cooinit=(0.0, 0.0, 0.0), grsize=shape)
    g = np.random.default_rng(l + len(shape)).normal(size=shape)
    got = O.smoothgradient(l, grd, g)
    want = ndimage.correlate(g, _kernel(l, len(shape)), mode="constant", cval=0.0)
    assert np.allclose(got, want, rtol=1e-13, atol=1e-14 * np.abs(g).max())
    if l == 1:
        assert np.array_equal(got, g)
