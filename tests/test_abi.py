"""CPU checks of the drop-in boundary: libeikcuda.so loads and exports every entry point
declared in include/eikcuda.h (no compute call: there may be no GPU here)."""
import ctypes as C
import os
import re
import shutil
import subprocess

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


def _c_layout(tmp_path, struct, fields):
    """sizeof and offsetof of a header struct, from a C compiler."""
    prog = tmp_path / "layout.c"
    lines = [f'printf("%zu\\n", sizeof({struct}));']
    lines += [f'printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    prog.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "eikcuda.h"\n'
                    "int main(void) {" + "".join(lines) + " return 0; }\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(REPO, "include"), str(prog), "-o", str(exe)],
                   check=True)
    out = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    return out[0], out[1:]


@pytest.mark.parametrize("name", ["eik_grid", "eik_extra", "eik_stats"])
def test_struct_layouts_match_header(tmp_path, name):
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    cls = getattr(_lib, name)
    fields = [f[0] for f in cls._fields_]
    size, offs = _c_layout(tmp_path, name, fields)
    assert C.sizeof(cls) == size
    assert [getattr(cls, f).offset for f in fields] == offs


def test_extra_defaults_match_reference():
    # ExtraParams() defaults, src/EikSolv/eikstructs.jl:260-265
    e = _lib.extra_struct(None)
    assert (e.refinearoundsrc, e.downscalefactor, e.noderadius, e.radiussmoothgradsrc,
            e.smoothgradkern, e.parallelkind) == (1, 5, 3, 3, 0, 0)


def test_warn_mask_messages_follow_the_reference_warn_sites():
    import warnings
    from eikonalsolvers import EikonalWarning, _lib
    from eikonalsolvers.api import _warn
    assert _lib.warn_mask_messages(0) == []
    msgs = _lib.warn_mask_messages(0x2 | 0x10)
    assert len(msgs) == 2 and "halfway" in msgs[0] and "node" in msgs[1]
    st = _lib.eik_stats()
    st.warn_mask = 0x1
    with warnings.catch_warnings(record=True) as rec:
        warnings.simplefilter("always")
        _warn(st)
    assert len(rec) == 1 and issubclass(rec[0].category, EikonalWarning)
    assert "discriminant" in str(rec[0].message)
