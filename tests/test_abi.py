"""CPU checks of the drop-in boundary: libeikcuda.so loads and exports every entry point
declared in include/eikcuda.h (no compute call: there may be no GPU here)."""
import ctypes as C
import os
import re

import pytest

from eikonalsolvers import _lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(REPO, "include", "eikcuda.h")).read()
    return sorted(set(re.findall(r"\b(eik_[a-z_]+)\s*\(", src)))


def test_header_declares_abi():
    syms = declared_symbols()
    assert set(_lib.EXPORTED) <= set(syms), set(_lib.EXPORTED) - set(syms)


def test_library_exports_every_declared_symbol():
    L = C.CDLL(_lib.LIBPATH)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_struct_sizes_match_header():
    assert C.sizeof(_lib.eik_grid) == 4 + 4 + 3 * 8 + 3 * 8 + 3 * 8
    assert C.sizeof(_lib.eik_extra) == 8 * 4
    assert C.sizeof(_lib.eik_stats) == 4 + 4 + 8 + 8 + 8


def test_extra_defaults_match_reference():
    # ExtraParams() defaults, src/EikSolv/eikstructs.jl:260-265
    e = _lib.extra_struct(None)
    assert (e.refinearoundsrc, e.downscalefactor, e.noderadius, e.radiussmoothgradsrc,
            e.smoothgradkern, e.parallelkind) == (1, 5, 3, 3, 0, 0)
