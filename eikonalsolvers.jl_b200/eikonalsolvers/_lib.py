"""ctypes binding of libeikcuda.so (include/eikcuda.h).

The library is built in-tree (``eikonalsolvers.jl_b200/build.py``) and loaded from
``eikonalsolvers.jl_b200/lib``. There is no CPU path: loading fails loudly when the
library is missing, and the first call fails when no CUDA device is present.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# EIKCUDA_LIB points at another build of the library (for example a tuning variant)
LIBPATH = os.environ.get("EIKCUDA_LIB") or os.path.join(os.path.dirname(_HERE), "lib", "libeikcuda.so")

EIK_OK = 0
ERRORS = {-1: "EIK_ERR_ASSERT", -2: "EIK_ERR_ERROR", -3: "EIK_ERR_CUDA", -4: "EIK_ERR_NOT_CONVERGED",
          -5: "EIK_ERR_OUT_OF_BUDGET", -6: "EIK_ERR_TIMEOUT", -7: "EIK_ERR_UNSUPPORTED"}

EXPORTED = ["eik_extra_defaults", "eik_ctx_create", "eik_ctx_destroy", "eik_last_error",
            "eik_model_upload", "eik_model_upload_device", "eik_model_release", "eik_traveltime",
            "eik_gradient", "eik_gradient_device", "eik_ctx_stream", "eik_ttimemisfit_noalloc",
            "eik_ctx_set_param", "eik_plan_gradient", "eik_plan_run", "eik_plan_destroy", "eik_tracerays",
            "eik_traveltime_rays", "eik_selftest_wait", "eik_gradient_bytes", "eik_traveltime_multi",
            "eik_gradient_groups"]

# eik_stats.warn_mask bits and the reference's @warn messages they stand for
WARNINGS = {
    0x1: "negative discriminant in the local traveltime update: one-dimensional update used "
         "(eikforward2D.jl:342, eikforward3D.jl:429)",
    0x2: "a source lies exactly halfway between grid nodes on an axis: it was shifted by 1e-4 of the "
         "spacing (eikmainfwd.jl:1298)",
    0x4: "the refined grid reached a border before the coarse grid took over (eikmainfwd.jl:731)",
    0x8: "a source coordinate is aligned with the grid: it was shifted by 1e-6 of the spacing for its "
         "derivative (eikmaingrad.jl:1250)",
    0x10: "a source lies on a node: the derivative of the traveltime there is set to zero "
          "(eikmaingrad.jl:1260)",
    0x20: "the refined grid covered the whole model: no edge stop",
}


def warn_mask_messages(mask: int):
    """Messages of the reference's @warn sites whose bits are set in an eik_stats.warn_mask."""
    return [msg for bit, msg in WARNINGS.items() if mask & bit]


class EikError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class EikAssertionError(EikError, AssertionError):
    pass


class eik_grid(C.Structure):
    _fields_ = [("kind", C.c_int32), ("ndim", C.c_int32), ("grsize", C.c_int64 * 3),
                ("spacing", C.c_double * 3), ("cooinit", C.c_double * 3)]


class eik_extra(C.Structure):
    _fields_ = [("refinearoundsrc", C.c_int32), ("downscalefactor", C.c_int32),
                ("noderadius", C.c_int32), ("radiussmoothgradsrc", C.c_int32),
                ("smoothgradkern", C.c_int32), ("parallelkind", C.c_int32),
                ("nthreads", C.c_int32), ("reserved", C.c_int32)]


class eik_stats(C.Structure):
    _fields_ = [("warn_mask", C.c_uint32), ("err_mask", C.c_uint32), ("tile_activations", C.c_uint64),
                ("node_evals", C.c_uint64), ("device_ms", C.c_double), ("fine_ms", C.c_double),
                ("solve_ms", C.c_double), ("adj_ms", C.c_double), ("adj_rounds", C.c_uint64),
                ("launches", C.c_uint64), ("fwd_rounds", C.c_uint64),
                ("fine_replays", C.c_uint64), ("fwd_visits", C.c_uint64 * 7), ("chunks", C.c_uint64), ("retries", C.c_uint64)]


_lib = None
_lock = threading.Lock()


def load():
    """Load libeikcuda.so (building it first when the sources are newer)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIBPATH):
            raise ImportError(f"libeikcuda.so not found at {LIBPATH}; run eikonalsolvers.jl_b200/build.py")
        L = C.CDLL(LIBPATH)
        P = C.c_void_p
        L.eik_extra_defaults.argtypes = [C.POINTER(eik_extra)]
        L.eik_extra_defaults.restype = None
        L.eik_ctx_create.argtypes = [C.c_int, C.c_size_t, C.POINTER(P)]
        L.eik_ctx_destroy.argtypes = [P]
        L.eik_last_error.argtypes = [P]
        L.eik_last_error.restype = C.c_char_p
        L.eik_model_upload.argtypes = [P, C.POINTER(eik_grid), P, C.POINTER(C.c_int64)]
        L.eik_model_upload_device.argtypes = [P, C.POINTER(eik_grid), P, C.POINTER(C.c_int64)]
        L.eik_model_release.argtypes = [P, C.c_int64]
        L.eik_traveltime.argtypes = [P, C.c_int64, C.c_int64, P, P, P, C.POINTER(eik_extra), P, P,
                                     C.POINTER(eik_stats)]
        L.eik_traveltime_multi.argtypes = [P, C.c_int64, P, P, P, P, P, C.POINTER(eik_extra), P, P,
                                           C.POINTER(eik_stats)]
        L.eik_traveltime_multi.restype = C.c_int
        L.eik_gradient_groups.argtypes = [P, C.c_int64, C.c_int64, P, P, P, P, P, P, C.c_int32,
                                          C.POINTER(eik_extra), P, P, P, C.POINTER(eik_stats)]
        L.eik_gradient_groups.restype = C.c_int
        L.eik_gradient.argtypes = [P, C.c_int64, C.c_int64, P, P, P, P, P, C.c_int32,
                                   C.POINTER(eik_extra), P, P, P, C.POINTER(eik_stats)]
        L.eik_gradient_device.argtypes = [P, C.c_int64, C.c_int64, P, P, P, P, P, C.c_int32,
                                          C.POINTER(eik_extra), P, P, P, C.POINTER(eik_stats)]
        L.eik_ttimemisfit_noalloc.argtypes = [C.POINTER(eik_grid), C.c_int64, P, P, P, P, P, P, P]
        L.eik_ttimemisfit_noalloc.restype = C.c_int
        L.eik_gradient_bytes.argtypes = [P, C.c_int64, C.c_int64, C.c_int64, C.POINTER(eik_extra), C.c_int32,
                                         C.POINTER(C.c_uint64)]
        L.eik_gradient_bytes.restype = C.c_int
        L.eik_selftest_wait.argtypes = [P, C.c_double]
        L.eik_selftest_wait.restype = C.c_int
        L.eik_ctx_set_param.argtypes = [P, C.c_char_p, C.c_double]
        L.eik_ctx_set_param.restype = C.c_int
        L.eik_ctx_stream.argtypes = [P]
        L.eik_ctx_stream.restype = C.c_void_p
        L.eik_plan_gradient.argtypes = [P, C.c_int64, C.c_int64, P, P, P, C.c_int32, C.POINTER(eik_extra),
                                        C.POINTER(P)]
        L.eik_plan_run.argtypes = [P, P, P, P, P, P, P, C.POINTER(eik_stats)]
        L.eik_plan_destroy.argtypes = [P]
        L.eik_tracerays.argtypes = [P, C.POINTER(eik_grid), C.c_int64, P, P, P, P, C.c_double, P, P, C.c_int64,
                                    C.POINTER(eik_stats)]
        L.eik_traveltime_rays.argtypes = [P, C.c_int64, C.c_int64, P, P, P, C.POINTER(eik_extra), C.c_double, P,
                                          P, P, C.c_int64, C.POINTER(eik_stats)]
        for f in ("eik_plan_gradient", "eik_plan_run", "eik_plan_destroy", "eik_tracerays", "eik_traveltime_rays"):
            getattr(L, f).restype = C.c_int
        for f in ("eik_ctx_create", "eik_ctx_destroy", "eik_model_upload", "eik_model_upload_device",
                  "eik_model_release", "eik_traveltime", "eik_gradient", "eik_gradient_device"):
            getattr(L, f).restype = C.c_int
        _lib = L
        return L


def check(rc: int, ctx=None):
    if rc == EIK_OK:
        return
    msg = load().eik_last_error(ctx).decode(errors="replace")
    if rc == -1:
        raise EikAssertionError(rc, msg)
    raise EikError(rc, msg)


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def grid_struct(grd) -> eik_grid:
    g = eik_grid()
    g.kind = grd.kind
    g.ndim = grd.ndim
    sp = list(grd.spacing) + [0.0] * (3 - grd.ndim)
    for a in range(3):
        g.grsize[a] = grd.grsize[a] if a < grd.ndim else 1
        g.cooinit[a] = grd.cooinit[a] if a < grd.ndim else 0.0
        g.spacing[a] = sp[a]
    return g


def extra_struct(extraparams, nthreads: int = 1) -> eik_extra:
    e = eik_extra()
    load().eik_extra_defaults(C.byref(e))
    e.nthreads = int(nthreads)
    if extraparams is not None:
        e.refinearoundsrc = int(extraparams.refinearoundsrc)
        e.downscalefactor = int(extraparams.grdrefpars.downscalefactor)
        e.noderadius = int(extraparams.grdrefpars.noderadius)
        e.radiussmoothgradsrc = int(extraparams.radiussmoothgradsrc)
        e.smoothgradkern = int(extraparams.smoothgradkern)
        e.parallelkind = {"serial": 0, "sharedmem": 1, "distribmem": 2}[extraparams.parallelkind]
    return e
