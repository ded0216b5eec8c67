"""The C-ABI library loads without a GPU and exports every symbol the header declares."""
import re
from pathlib import Path

from pyib_b200 import _lib, build

HEADER = Path(__file__).resolve().parents[1] / "include" / "pyib_b200.h"


def declared():
    txt = HEADER.read_text()
    return sorted(set(re.findall(r"^int (pyib_\w+)\(", txt, flags=re.M)))


def test_library_exports_header_symbols():
    build.build_library()
    syms = set(_lib.exported_symbols())
    assert set(declared()) <= set(_lib.EXPORTS)
    assert set(declared()) <= syms


def test_ctypes_structs_match_header_sizes():
    import ctypes as C
    # pyib_layout: 4 + 3*3*8*4 + 8*8 + 24*8 + 3*8 + 2*4, padded to 8
    assert C.sizeof(_lib.Layout) == 4 + 3 * 96 + 64 + 192 + 4 + 24 + 8
    assert C.sizeof(_lib.Params) == 6 * 8 + 6 * 4 + 3 * 8 + 2 * 4 + 8
    assert C.sizeof(_lib.SolveStats) == 8 + 4 * 8 + 8
    assert C.sizeof(_lib.StepStats) == 16 + 16


def test_create_rejects_bad_layout_without_gpu():
    import ctypes as C
    lib = _lib.load()
    L = _lib.Layout()
    L.nlevels = 0
    ptr = C.c_void_p()
    assert lib.pyib_create(C.byref(L), C.byref(ptr)) == _lib.E_ARG
