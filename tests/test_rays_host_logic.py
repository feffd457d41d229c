"""Host logic of the ray-tracing bindings (eikonalsolvers.api): the first size guess, the
retry with the exact size when the library reports the buffer too small
(EIK_ERR_OUT_OF_BUDGET), and the split of the concatenated points into rays."""
import numpy as np

from eikonalsolvers import Grid2DCart
from eikonalsolvers.api import _ray_capacity, _ray_inputs, _split_rays, _traced


def test_split_rays_in_receiver_order():
    recoff = np.array([0, 2, 3])
    npts = np.array([2, 3, 1])
    pts = np.arange(12, dtype=float)
    rays = _split_rays(npts, pts, recoff, 2)
    assert [len(r) for r in rays] == [2, 1]
    assert np.array_equal(rays[0][0], [[0, 1], [2, 3]])
    assert np.array_equal(rays[0][1], [[4, 5], [6, 7], [8, 9]])
    assert np.array_equal(rays[1][0], [[10, 11]])


def test_traced_retries_with_the_exact_size():
    g = Grid2DCart(hgrid=1.0, cooinit=(0.0, 0.0), grsize=(10, 10))
    cs, recoff, rec = _ray_inputs(g, np.array([[1.0, 1.0]]), [np.array([[2.0, 1.0], [1.0, 2.0]])])
    guess = _ray_capacity(g, cs, recoff, rec, 0.5)
    assert guess == 2 * (int(3.0 * 1.0 / 0.5) + 16)
    need = [guess, 5]  # the first ray is longer than its guess: the total does not fit
    calls = []

    def call(npts, pts, cap):
        calls.append(cap)
        npts[:2] = need
        if cap < sum(need):
            return -5
        pts[:sum(need) * 2] = np.arange(sum(need) * 2)
        return 0
    rc, rays = _traced(call, g, cs, recoff, rec, 0.5)
    assert rc == 0 and calls == [guess, sum(need)]
    assert rays[0][0].shape == (guess, 2) and rays[0][1].shape == (5, 2)
    assert rays[0][1][0, 0] == 2 * guess
