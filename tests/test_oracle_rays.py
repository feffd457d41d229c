"""Pins the ray-tracing oracle (tracerays, src/EikSolv/eikutils.jl:201-328, with the cubic
B-spline of Interpolations.jl restated in oracle/rays.cpp) on fields whose rays are known:
a linear traveltime field (the cubic B-spline with Line boundaries reproduces it, so every
step is exactly steplen*h against its gradient), a point-source field (rays are straight
lines into the source), and the reference's own rules (last point = source, a receiver
within h*sqrt(2) of the source gives a one-point ray, Grid3DSphere errors)."""
import numpy as np
import pytest

import eikoracle as O
from eikonalsolvers import Grid2DCart, Grid2DSphere, Grid3DCart, Grid3DSphere


def _xy(g):
    return np.array(g.x)[:, None], np.array(g.y)[None, :]


def test_linear_field_steps_are_exact():
    g = Grid2DCart(hgrid=0.5, cooinit=(0.0, 0.0), grsize=(60, 40))
    x, y = _xy(g)
    rays = O.tracerays(g, [0.3 * x + 0.4 * y], np.array([[0.2, 0.1]]), [np.array([[25.0, 15.0]])], steplen=0.01)
    r = rays[0][0]
    k = np.arange(1, 200)[:, None]
    assert np.abs(r[1:200] - (r[0] - 0.005 * k * np.array([0.6, 0.8]))).max() < 1e-12
    assert np.array_equal(r[-1], [0.2, 0.1]) and np.array_equal(r[0], [25.0, 15.0])
    # clamped onto the grid's border, then along it
    assert r[:, 1].min() == 0.0


@pytest.mark.parametrize("dim", [2, 3])
def test_point_source_rays_are_straight(dim):
    if dim == 2:
        g = Grid2DCart(hgrid=0.5, cooinit=(0.0, 0.0), grsize=(60, 40))
        x, y = _xy(g)
        src = np.array([12.3, 7.7])
        tt = np.sqrt((x - src[0]) ** 2 + (y - src[1]) ** 2) / 3.0
        rec = np.array([[25.0, 15.0], [1.0, 18.0], [12.5, 7.9]])
    else:
        g = Grid3DCart(hgrid=0.5, cooinit=(0.0, 0.0, 0.0), grsize=(30, 25, 20))
        x = np.array(g.x)[:, None, None]
        y = np.array(g.y)[None, :, None]
        z = np.array(g.z)[None, None, :]
        src = np.array([5.3, 6.1, 4.2])
        tt = np.sqrt((x - src[0]) ** 2 + (y - src[1]) ** 2 + (z - src[2]) ** 2) / 2.0
        rec = np.array([[12.0, 10.0, 0.0], [0.5, 0.5, 9.0], [5.4, 6.0, 4.3]])
    rays = O.tracerays(g, [tt], src[None, :], [rec], steplen=0.01)[0]
    for r, p in zip(rays[:2], rec[:2]):
        u = (p - src) / np.linalg.norm(p - src)
        v = r[:-1] - src
        perp = np.linalg.norm(v - np.outer(v @ u, u), axis=1)
        assert perp.max() < 0.02 * 0.5  # within 2 % of a cell of the straight line
        # the point before the source is the last one still h*sqrt(2) away (the next step,
        # replaced by the source, was within)
        d2 = np.linalg.norm(r[-2] - src)
        assert 0.5 * np.sqrt(2) <= d2 < 0.5 * np.sqrt(2) + 0.0051 and np.array_equal(r[-1], src)
        # steps of steplen*h
        assert np.allclose(np.linalg.norm(np.diff(r[:-1], axis=0), axis=1), 0.005, rtol=1e-9)
    # a receiver within h*sqrt(2) of the source: one point, the source
    assert rays[2].shape == (1, dim) and np.array_equal(rays[2][0], src)


def test_polar_rays_reach_the_source_and_3d_sphere_errors():
    g = Grid2DSphere(Δr=2.0, Δθ=0.25, cooinit=(5800.0, 10.0), grsize=(40, 50))
    r, th = np.array(g.r)[:, None], np.array(g.θ)[None, :]
    s = np.array([5840.0, 15.3])
    X, Y = r * np.cos(np.deg2rad(th)), r * np.sin(np.deg2rad(th))
    SX, SY = s[0] * np.cos(np.deg2rad(s[1])), s[0] * np.sin(np.deg2rad(s[1]))
    tt = np.sqrt((X - SX) ** 2 + (Y - SY) ** 2) / 5.0
    rays = O.tracerays(g, [tt], s[None, :], [np.array([[5878.0, 20.0], [5878.0, 11.0]])], steplen=0.5)[0]
    for ray in rays:
        P = np.c_[ray[:, 0] * np.cos(np.deg2rad(ray[:, 1])), ray[:, 0] * np.sin(np.deg2rad(ray[:, 1]))]
        steps = np.linalg.norm(np.diff(P[:-1], axis=0), axis=1)
        assert np.allclose(steps, 0.5, rtol=1e-9)  # steplen in km on a Grid2DSphere
        u = (P[0] - [SX, SY]) / np.linalg.norm(P[0] - [SX, SY])
        v = P[:-1] - [SX, SY]
        assert np.abs(v[:, 0] * u[1] - v[:, 1] * u[0]).max() < 0.5
        assert np.array_equal(ray[-1], s)
    g3 = Grid3DSphere(Δr=2.0, Δθ=0.25, Δφ=0.3, cooinit=(5800.0, 40.0, 10.0), grsize=(8, 8, 8))
    with pytest.raises(O.OracleError, match="not yet implemented"):
        O.tracerays(g3, [np.ones(g3.grsize)], np.array([[5806.0, 41.0, 11.0]]), [np.array([[5810.0, 41.5, 11.5]])])
