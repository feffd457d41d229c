"""VTK export (savemodelvtk, ext/SaveGrid2VTKExt.jl:17-415): the files written read back to
the grids' coordinates (node coordinates, or cell vertices half a spacing around them), the
spherical grids' points with the reference's mapping, and the arrays (extra trailing
dimension split into "key  #i"), in x-fastest order."""
import os

import numpy as np
import pytest

from eikonalsolvers import Grid2DCart, Grid2DSphere, Grid3DCart, Grid3DSphere
from eikonalsolvers.vtk import cosd, read_vtk, savemodelvtk, sind


def test_cartesian_2d_points_and_split_arrays(tmp_path):
    g = Grid2DCart(hgrid=0.5, cooinit=(1.0, 2.0), grsize=(7, 5))
    rng = np.random.default_rng(0)
    vel, grad = rng.random(g.grsize), rng.random(g.grsize + (2,))
    files = savemodelvtk(str(tmp_path / "m"), g, {"vel": vel, "grad": grad})
    assert files == [str(tmp_path / "m.vtr")] and os.path.exists(files[0])
    d = read_vtk(files[0])
    assert d["type"] == "RectilinearGrid" and d["extent"] == "0 6 0 4 0 0" and d["section"] == "PointData"
    assert np.array_equal(d["coords"][0], np.array(g.x)) and np.array_equal(d["coords"][1], np.array(g.y))
    assert np.array_equal(d["coords"][2], [0.0])
    assert np.array_equal(d["data"]["vel"], vel.ravel(order="F"))
    for i in range(2):
        assert np.array_equal(d["data"][f"grad  #{i + 1}"], grad[:, :, i].ravel(order="F"))


def test_cartesian_3d_cells(tmp_path):
    g = Grid3DCart(hgrid=0.25, cooinit=(0.0, 0.0, 0.0), grsize=(4, 3, 5))
    vel = np.arange(60, dtype=float).reshape(g.grsize)
    d = read_vtk(savemodelvtk(str(tmp_path / "c"), g, {"v": vel}, kind="cells")[0])
    assert d["extent"] == "0 4 0 3 0 5" and d["section"] == "CellData"
    for a, ax in zip(d["coords"], (g.x, g.y, g.z)):
        ax = np.array(ax)
        assert np.array_equal(a, np.concatenate([ax - 0.125, [ax[-1] + 0.125]]))
    assert np.array_equal(d["data"]["v"], vel.ravel(order="F"))
    with pytest.raises(RuntimeError, match="Wrong argument 'kind'"):
        savemodelvtk(str(tmp_path / "x"), g, {"v": vel}, kind="edges")


def test_sphere_2d(tmp_path):
    g = Grid2DSphere(Δr=2.0, Δθ=0.5, cooinit=(5800.0, 10.0), grsize=(4, 6))
    r, th = np.array(g.r), np.array(g.θ)
    v = np.ones(g.grsize)
    d = read_vtk(savemodelvtk(str(tmp_path / "s"), g, {"v": v})[0])
    assert d["type"] == "StructuredGrid" and d["extent"] == "0 3 0 5 0 0"
    P = d["points"].reshape(6, 4, 3)  # [θ, r, xyz]: r fastest
    for i in range(4):
        for j in range(6):
            assert np.array_equal(P[j, i], [r[i] * sind(th[j]), r[i] * cosd(th[j]), 0.0])
    d = read_vtk(savemodelvtk(str(tmp_path / "sc"), g, {"v": v}, kind="cells")[0])
    assert d["extent"] == "0 4 0 6 0 0" and d["section"] == "CellData"
    P = d["points"].reshape(7, 5, 3)
    assert np.array_equal(P[0, 0, :2], [(r[0] - 1.0) * sind(th[0] - 0.25), (r[0] - 1.0) * cosd(th[0] - 0.25)])
    assert np.array_equal(P[3, 2, :2], [(r[1] + 1.0) * sind(th[2] + 0.25), (r[1] + 1.0) * cosd(th[2] + 0.25)])
    assert np.array_equal(P[6, 0, :2], [(r[0] - 1.0) * sind(th[5] + 0.25), (r[0] - 1.0) * cosd(th[5] + 0.25)])
    assert savemodelvtk(str(tmp_path / "none"), g, {"v": v}, kind="edges") == []


def test_sphere_3d(tmp_path):
    g = Grid3DSphere(Δr=2.0, Δθ=0.5, Δφ=0.4, cooinit=(5800.0, 40.0, 10.0), grsize=(3, 4, 2))
    r, th, ph = np.array(g.r), np.array(g.θ), np.array(g.φ)
    v = np.arange(24, dtype=float).reshape(g.grsize)
    xyz = lambda a, b, c: [a * sind(b) * cosd(c), a * sind(b) * sind(c), a * cosd(b)]  # noqa: E731
    d = read_vtk(savemodelvtk(str(tmp_path / "p"), g, {"v": v})[0])
    P = d["points"].reshape(2, 4, 3, 3)
    assert np.array_equal(P[1, 2, 0], xyz(r[0], th[2], ph[1]))
    assert np.array_equal(d["data"]["v"], v.ravel(order="F"))
    d = read_vtk(savemodelvtk(str(tmp_path / "c"), g, {"v": v}, kind="cells")[0])
    assert d["extent"] == "0 3 0 4 0 2"
    P = d["points"].reshape(3, 5, 4, 3)  # [φ, θ, r]
    assert np.array_equal(P[2, 4, 3], xyz(r[2] + 1.0, th[3] + 0.25, ph[1] + 0.2))
    assert np.array_equal(P[0, 0, 0], xyz(r[0] - 1.0, th[0] - 0.25, ph[0] - 0.2))
    assert np.array_equal(P[0, 4, 0], xyz(r[0] - 1.0, th[3] + 0.25, ph[0] - 0.2))
    assert np.all(np.isfinite(P)) and not np.any(np.all(P == 0.0, axis=-1))  # every vertex assigned
