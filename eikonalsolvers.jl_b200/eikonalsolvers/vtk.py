"""VTK export of models and traveltime / gradient grids: ``savemodelvtk`` of the reference's
WriteVTK extension (ext/SaveGrid2VTKExt.jl:17-415), written without WriteVTK.

``savemodelvtk(flname, grd, datadict, kind="points")`` writes one VTK XML file:

* Cartesian grids: a RectilinearGrid (``flname.vtr``) whose coordinates are the grid's node
  coordinates (``kind="points"``: the arrays are point data) or the cell vertices half a
  spacing around them (``kind="cells"``: the arrays are cell data), as the reference does
  (SaveGrid2VTKExt.jl:17-140);
* spherical grids: a StructuredGrid (``flname.vts``) whose points are the nodes (or the cell
  vertices) mapped to Cartesian coordinates with the reference's formulas, x = r·sind(θ),
  y = r·cosd(θ) in 2D and x = r·sind(θ)·cosd(φ), y = r·sind(θ)·sind(φ), z = r·cosd(θ) in 3D,
  the cell vertices assigned edge by edge in the reference's order
  (SaveGrid2VTKExt.jl:147-412).

Every entry of ``datadict`` is an array shaped like the grid (index ``[i, j(, k)]``); an array
with one more dimension is written as one array per trailing index, named ``"key  #i"``
(1-based), as the reference does. The data are Float64, x fastest (the grids' own
column-major order), stored in raw appended form (UInt64 byte counts, little endian) that
ParaView and VTK read. A wrong ``kind`` on a Cartesian grid raises the reference's error; on a
spherical grid the reference writes nothing and so does this function. Returns the list of
files written.
"""
from __future__ import annotations

import math
import struct
from typing import Dict, List

import numpy as np

_DEG2RAD = math.pi / 180.0


def _sincosd(x: float):
    """sind/cosd with exact reduction by quarter turns (as Julia's sind/cosd)."""
    r = math.fmod(x, 360.0)
    if r < 0:
        r += 360.0
    q = int(math.floor((r + 45.0) / 90.0))
    y = (r - 90.0 * q) * _DEG2RAD
    sy, cy = math.sin(y), math.cos(y)
    q &= 3
    if q == 0:
        return sy, cy
    if q == 1:
        return cy, -sy
    if q == 2:
        return -sy, -cy
    return -cy, sy


def sind(x: float) -> float:
    return _sincosd(x)[0]


def cosd(x: float) -> float:
    return _sincosd(x)[1]


class _Appended:
    def __init__(self):
        self.blocks: List[bytes] = []
        self.offset = 0

    def add(self, arr: np.ndarray) -> int:
        data = np.ascontiguousarray(arr, dtype="<f8").tobytes()
        off = self.offset
        self.blocks.append(struct.pack("<Q", len(data)) + data)
        self.offset += 8 + len(data)
        return off


def _data_arrays(datadict: Dict, nd: int):
    """(name, column-major values) of every array, trailing extra dimension split."""
    out = []
    for key, arr in datadict.items():
        a = np.asarray(arr, dtype=np.float64)
        if a.ndim > nd:
            for i in range(a.shape[nd]):
                out.append((f"{key}  #{i + 1}", a[(Ellipsis, i)].ravel(order="F")))
        else:
            out.append((str(key), a.ravel(order="F")))
    return out


def _write(path: str, gtype: str, extent: str, arrays, section: str, geometry) -> str:
    app = _Appended()
    lines = ['<?xml version="1.0"?>',
             f'<VTKFile type="{gtype}" version="1.0" byte_order="LittleEndian" header_type="UInt64">',
             f'  <{gtype} WholeExtent="{extent}">', f'    <Piece Extent="{extent}">']
    lines.append(f"      <{section}>")
    for name, vals in arrays:
        off = app.add(vals)
        lines.append(f'        <DataArray type="Float64" Name="{name}" format="appended" offset="{off}"/>')
    lines.append(f"      </{section}>")
    if gtype == "RectilinearGrid":
        lines.append("      <Coordinates>")
        for name, c in zip(("x", "y", "z"), geometry):
            off = app.add(np.asarray(c, dtype=np.float64))
            lines.append(f'        <DataArray type="Float64" Name="{name}" format="appended" offset="{off}"/>')
        lines.append("      </Coordinates>")
    else:
        off = app.add(geometry)
        lines.append("      <Points>")
        lines.append(f'        <DataArray type="Float64" Name="Points" NumberOfComponents="3" format="appended" '
                     f'offset="{off}"/>')
        lines.append("      </Points>")
    lines += ["    </Piece>", f"  </{gtype}>", '  <AppendedData encoding="raw">']
    with open(path, "wb") as f:
        f.write(("\n".join(lines) + "\n   _").encode())
        for b in app.blocks:
            f.write(b)
        f.write(b"\n  </AppendedData>\n</VTKFile>\n")
    return path


def _extent(counts) -> str:
    c = list(counts) + [1] * (3 - len(counts))
    return " ".join(f"0 {n - 1}" for n in c)


def _fname(flname: str, ext: str) -> str:
    return flname if flname.endswith(ext) else flname + ext


def _cart(flname, grd, datadict, kind):
    axes = [np.asarray(a, dtype=np.float64) for a in ((grd.x, grd.y) if grd.ndim == 2 else (grd.x, grd.y, grd.z))]
    if kind == "cells":
        h2 = grd.hgrid / 2.0
        axes = [np.concatenate([a - h2, [a[-1] + h2]]) for a in axes]
        section = "CellData"
    elif kind == "points":
        section = "PointData"
    else:
        raise RuntimeError("savevtk(): Wrong argument 'kind'.")
    counts = [len(a) for a in axes]
    geom = axes + ([np.zeros(1)] if grd.ndim == 2 else [])
    return [_write(_fname(flname, ".vtr"), "RectilinearGrid", _extent(counts), _data_arrays(datadict, grd.ndim),
                   section, geom)]


def _sphere2d_points(grd, kind):
    r, th = list(grd.r), list(grd.θ)
    nr, nt = len(r), len(th)
    dr, dt = grd.Δr, grd.Δθ
    if kind == "points":
        xy = np.zeros((2, nr, nt))
        for it in range(nt):
            for ir in range(nr):
                xy[:, ir, it] = (r[ir] * sind(th[it]), r[ir] * cosd(th[it]))
        return xy, (nr, nt)
    xy = np.zeros((2, nr + 1, nt + 1))
    it = 0
    for ir in range(nr):  # lower θ edge
        xy[:, ir, it] = ((r[ir] - dr / 2) * sind(th[it] - dt / 2), (r[ir] - dr / 2) * cosd(th[it] - dt / 2))
        if ir == nr - 1:
            xy[:, ir + 1, it] = ((r[ir] + dr / 2) * sind(th[it] - dt / 2), (r[ir] + dr / 2) * cosd(th[it] - dt / 2))
    for it in range(nt):  # lower r edge
        ir = 0
        xy[:, ir, it] = ((r[ir] - dr / 2) * sind(th[it] - dt / 2), (r[ir] - dr / 2) * cosd(th[it] - dt / 2))
        if it == nt - 1:
            xy[:, ir, it + 1] = ((r[ir] - dr / 2) * sind(th[it] + dt / 2), (r[ir] - dr / 2) * cosd(th[it] + dt / 2))
    for it in range(nt):
        for ir in range(nr):
            xy[:, ir + 1, it + 1] = ((r[ir] + dr / 2) * sind(th[it] + dt / 2), (r[ir] + dr / 2) * cosd(th[it] + dt / 2))
    return xy, (nr + 1, nt + 1)


def _xyz(rr, tt, pp):
    return (rr * sind(tt) * cosd(pp), rr * sind(tt) * sind(pp), rr * cosd(tt))


def _sphere3d_points(grd, kind):
    r, th, ph = list(grd.r), list(grd.θ), list(grd.φ)
    nr, nt, nph = len(r), len(th), len(ph)
    dr, dt, dp = grd.Δr, grd.Δθ, grd.Δφ
    if kind == "points":
        xyz = np.zeros((3, nr, nt, nph))
        for ip in range(nph):
            for it in range(nt):
                for ir in range(nr):
                    xyz[:, ir, it, ip] = _xyz(r[ir], th[it], ph[ip])
        return xyz, (nr, nt, nph)
    xyz = np.zeros((3, nr + 1, nt + 1, nph + 1))
    ir = 0  # lower r boundary
    for ip in range(nph):
        for it in range(nt):
            xyz[:, ir, it, ip] = _xyz(r[ir] - dr / 2, th[it] - dt / 2, ph[ip] - dp / 2)
            if it == nt - 1:
                xyz[:, ir, it + 1, ip] = _xyz(r[ir] - dr / 2, th[it] + dt / 2, ph[ip] - dp / 2)
            if ip == nph - 1:
                xyz[:, ir, it, ip + 1] = _xyz(r[ir] - dr / 2, th[it] - dt / 2, ph[ip] + dp / 2)
            if ip == nph - 1 and it == nt - 1:
                xyz[:, ir, it + 1, ip + 1] = _xyz(r[ir] - dr / 2, th[it] + dt / 2, ph[ip] + dp / 2)
    it = 0  # lower θ boundary
    for ip in range(nph):
        for ir in range(nr):
            xyz[:, ir, it, ip] = _xyz(r[ir] - dr / 2, th[it] - dt / 2, ph[ip] - dp / 2)
            if ir == nr - 1:
                xyz[:, ir + 1, it, ip] = _xyz(r[ir] + dr / 2, th[it] - dt / 2, ph[ip] - dp / 2)
            if ip == nph - 1:
                xyz[:, ir, it, ip + 1] = _xyz(r[ir] - dr / 2, th[it] - dt / 2, ph[ip] + dp / 2)
            if ip == nph - 1 and ir == nr - 1:
                xyz[:, ir + 1, it, ip + 1] = _xyz(r[ir] + dr / 2, th[it] - dt / 2, ph[ip] + dp / 2)
    ip = 0  # lower φ boundary
    for ir in range(nr):
        for it in range(nt):
            xyz[:, ir, it, ip] = _xyz(r[ir] - dr / 2, th[it] - dt / 2, ph[ip] - dp / 2)
            if ir == nr - 1:
                xyz[:, ir + 1, it, ip] = _xyz(r[ir] + dr / 2, th[it] - dt / 2, ph[ip] - dp / 2)
            if it == nt - 1:
                xyz[:, ir, it + 1, ip] = _xyz(r[ir] - dr / 2, th[it] + dt / 2, ph[ip] - dp / 2)
            if ir == nr - 1:  # the reference's corner test reads `ir==nr && ir==nr`
                xyz[:, ir + 1, it + 1, ip] = _xyz(r[ir] + dr / 2, th[it] + dt / 2, ph[ip] - dp / 2)
    for ip in range(nph):
        for it in range(nt):
            for ir in range(nr):
                xyz[:, ir + 1, it + 1, ip + 1] = _xyz(r[ir] + dr / 2, th[it] + dt / 2, ph[ip] + dp / 2)
    return xyz, (nr + 1, nt + 1, nph + 1)


def _sphere(flname, grd, datadict, kind):
    if kind not in ("cells", "points"):
        return []  # the reference's spherical branches have no else: nothing is written
    pts, counts = (_sphere2d_points if grd.ndim == 2 else _sphere3d_points)(grd, kind)
    # points as (x, y, z) triples with the first grid index fastest; 2D grids lie in z = 0
    comp = pts.reshape(pts.shape[0], -1, order="F")
    if comp.shape[0] == 2:
        comp = np.vstack([comp, np.zeros((1, comp.shape[1]))])
    geom = np.ascontiguousarray(comp.T).ravel()
    section = "CellData" if kind == "cells" else "PointData"
    return [_write(_fname(flname, ".vts"), "StructuredGrid", _extent(counts), _data_arrays(datadict, grd.ndim),
                   section, geom)]


def savemodelvtk(flname: str, grd, datadict: Dict, kind: str = "points") -> List[str]:
    """Writes the arrays of ``datadict`` on ``grd`` to a VTK XML file (see the module doc)."""
    name = type(grd).__name__
    if name in ("Grid2DCart", "Grid3DCart"):
        return _cart(flname, grd, datadict, kind)
    if name in ("Grid2DSphere", "Grid3DSphere"):
        return _sphere(flname, grd, datadict, kind)
    raise TypeError(f"savemodelvtk: no method for {name}")


def read_vtk(path: str) -> dict:
    """Reads back a file written by ``savemodelvtk``: {"type", "extent", "coords" or "points",
    "data": {name: values}} (test helper and a minimal reader for the raw appended form)."""
    import xml.etree.ElementTree as ET
    raw = open(path, "rb").read()
    head, _, tail = raw.partition(b'<AppendedData encoding="raw">')
    start = tail.index(b"_") + 1
    blob = tail[start:]
    xml = head.decode() + '<AppendedData encoding="raw"/></VTKFile>'
    root = ET.fromstring(xml)

    def block(off):
        n = struct.unpack_from("<Q", blob, off)[0]
        return np.frombuffer(blob, dtype="<f8", count=n // 8, offset=off + 8).copy()
    gtype = root.attrib["type"]
    grid = root.find(gtype)
    piece = grid.find("Piece")
    out = {"type": gtype, "extent": grid.attrib["WholeExtent"], "data": {}}
    for sec in ("PointData", "CellData"):
        node = piece.find(sec)
        if node is not None:
            for da in node.findall("DataArray"):
                out["data"][da.attrib["Name"]] = block(int(da.attrib["offset"]))
            if len(node):
                out["section"] = sec
    if gtype == "RectilinearGrid":
        out["coords"] = [block(int(da.attrib["offset"])) for da in piece.find("Coordinates").findall("DataArray")]
    else:
        out["points"] = block(int(piece.find("Points").find("DataArray").attrib["offset"])).reshape(-1, 3)
    return out
