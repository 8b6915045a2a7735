"""The C ABI boundary without a GPU: the library is built for sm_100a, loads,
exports every entry point include/cenote_c.h declares, and fails loudly (an
error status, never a CPU fallback) when no capable GPU is present."""
import ctypes as C
import re
import subprocess

import pytest

import cenote_b200
from cenote_b200 import CenoteError, EXPORTED_SYMBOLS, LIB_PATH, library

HEADER = cenote_b200.LIB_PATH.parent.parent / "include" / "cenote_c.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(cenote_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_list_agree():
    assert declared_symbols() == sorted(EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol():
    lib = library()
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_library_carries_sm100a_code():
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB_PATH)], capture_output=True, text=True).stdout
    for name in declared_symbols():
        assert re.search(rf"\bT {name}$", out, re.M), name


def test_struct_layouts_match_the_header():
    assert C.sizeof(cenote_b200.Material) == 144
    assert C.sizeof(cenote_b200.Object) == 8 * 4 + 8 + 48 + 144 + 8
    assert cenote_b200.LIGHT_RECORD_DTYPE.itemsize == 80


def test_context_without_a_gpu_is_an_error_not_a_fallback():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(CenoteError) as e:
        cenote_b200.Context(0)
    assert e.value.code == -3
