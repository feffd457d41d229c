"""EikonalSolvers.jl's forward (2nd-order FMM) and discrete-adjoint hot path on B200.

Python mirror of the reference's public API over the C-ABI library libeikcuda.so.
"""
from .structs import (ExtraParams, Grid2DCart, Grid2DSphere, Grid3DCart, Grid3DSphere,
                      GridRefinementPars, JuliaRange)
from .api import Context, EikonalWarning, GradientPlan, default_context, eikgradient, eiktraveltime, eikttimemisfit, tracerays
from .vtk import savemodelvtk

__all__ = ["Grid2DCart", "Grid3DCart", "Grid2DSphere", "Grid3DSphere", "ExtraParams",
           "GridRefinementPars", "JuliaRange", "Context", "EikonalWarning", "GradientPlan", "default_context", "eiktraveltime",
           "eikgradient", "eikttimemisfit", "tracerays", "savemodelvtk"]
