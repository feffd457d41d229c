"""The ray-tracing kernels' per-line and per-ray code (csrc/rays.cuh, shared by the CUDA
kernels and the host) run on the CPU under AddressSanitizer and UndefinedBehaviorSanitizer
(out-of-bounds and misaligned accesses abort the run), on the oracle's traveltime grids:
no sanitizer report, no address-check flag, and rays bit-identical to the oracle's."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import eikoracle as O
import refcases as RC
from eikonalsolvers import ExtraParams
from eikonalsolvers import configs as CF

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "eikonalsolvers.jl_b200", "csrc")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("rayhost")
    exe = str(d / "harness")
    cmd = ["g++", "-O1", "-g", "-std=c++17", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
           "-ffp-contract=off", "-include", "cstring", "-I", CSRC, os.path.join(HERE, "rays_host_harness.cpp"),
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip("sanitizer build unavailable: " + r.stderr[-300:])
    return exe, d


def _cases():
    c2 = [c for c in RC.all_forward_cases() if c["name"] == "2Dlingrad0"][0]
    w3 = CF.cfg3(scale=0.125, nsrc=2, nrec_side=3)
    return [("2Dlingrad0", c2["vel"], c2["grd"], c2["coordsrc"], c2["coordrec"]),
            ("3D-layered", w3.vel, w3.grd, w3.coordsrc, w3.coordrec)]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_ray_code_is_clean_under_sanitizers_and_matches_the_oracle(harness, case):
    exe, d = harness
    _, vel, grd, cs, rec = case
    cs = np.atleast_2d(np.asarray(cs, dtype=np.float64))
    if isinstance(rec, np.ndarray) and rec.dtype != object:
        rec = [rec]
    recs = [np.atleast_2d(np.asarray(r, dtype=np.float64)) for r in rec]
    _, tt = O.eiktraveltime(vel, grd, cs, recs, returntt=True, extraparams=ExtraParams())
    pad = lambda v, f: list(v) + [f] * (3 - len(v))  # noqa: E731
    meta = np.array([grd.kind, grd.ndim] + pad(grd.grsize, 1) + pad(grd.spacing, 0.0) + pad(grd.cooinit, 0.0) +
                    [0.01], dtype=np.float64)
    off = np.zeros(len(recs) + 1, dtype=np.int64)
    for i, r in enumerate(recs):
        off[i + 1] = off[i] + r.shape[0]
    files = {k: str(d / f"{k}.bin") for k in ("meta", "tt", "cs", "off", "rec", "out")}
    meta.tofile(files["meta"])
    np.concatenate([t.ravel(order="F") for t in tt]).tofile(files["tt"])
    cs.tofile(files["cs"])
    off.tofile(files["off"])
    np.concatenate(recs).tofile(files["rec"])
    r = subprocess.run([exe] + [files[k] for k in ("meta", "tt", "cs", "off", "rec", "out")], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "err 0 spline_err 0" in r.stdout
    raw = np.fromfile(files["out"])
    nray = int(off[-1])
    npts = raw[:nray].view(np.int64)
    pts = raw[nray:]
    want = O.tracerays(grd, tt, cs, recs, steplen=0.01)
    flat = [w for s in want for w in s]
    assert np.array_equal(npts, [w.shape[0] for w in flat])
    assert np.array_equal(pts, np.concatenate([w.ravel() for w in flat]))
