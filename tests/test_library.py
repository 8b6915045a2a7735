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


STRUCT_MIRRORS = {  # C type in include/cenote_c.h -> its ctypes mirror in cenote_b200
    "cenote_material": "Material", "cenote_object": "Object", "cenote_camera": "CameraC",
    "cenote_texture": "TextureC", "cenote_environment": "EnvironmentC", "cenote_delta_light": "DeltaLightC",
    "cenote_options": "Options", "cenote_stats": "Stats", "cenote_tuning": "TuningC",
    "cenote_server_options": "ServerOptions", "cenote_job_status": "JobStatus",
    "cenote_server_counters": "ServerCounters",
}


def test_header_compiles_as_c_and_links(tmp_path):
    """The header as a C caller (a Rust bindgen crate, cgo) sees it: plain
    C99 with -pedantic -Werror, every declared entry point taken by address
    and resolved by the linker against the built library, and every struct
    the same size as the Python binding's mirror. The program runs without a
    GPU: it only reads cenote_last_error()."""
    syms = declared_symbols()
    src = ['#include "cenote_c.h"', "#include <stdio.h>", "#include <stddef.h>",
           "typedef void (*any_fn)(void);", "int main(void) {", "    const any_fn table[] = {"]
    src += [f"        (any_fn){s}," for s in syms]
    src += ["    };", '    printf("entries %u\\n", (unsigned)(sizeof table / sizeof table[0]));',
            '    printf("last_error [%s]\\n", cenote_last_error());']
    src += [f'    printf("sizeof {c} %u\\n", (unsigned)sizeof({c}));' for c in STRUCT_MIRRORS]
    src += ["    return 0;", "}"]
    c_file = tmp_path / "abi.c"
    c_file.write_text("\n".join(src) + "\n")
    exe = tmp_path / "abi"
    subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror",
                    "-Wno-cast-function-type", f"-I{HEADER.parent}", str(c_file), "-o", str(exe),
                    str(LIB_PATH), f"-Wl,-rpath,{LIB_PATH.parent}"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    assert f"entries {len(syms)}" in out
    sizes = dict(re.findall(r"sizeof (\w+) (\d+)", out))
    for c_name, py_name in STRUCT_MIRRORS.items():
        assert int(sizes[c_name]) == C.sizeof(getattr(cenote_b200, py_name)), c_name
