"""Build libcenote_b200.so in-tree: CUDA kernels for sm_100a plus the C++ host
library, linked against the static CUDA runtime.

    python -m cenote_b200.build          # or cenote_b200.build.build()

The BSDF lookup tables (cenote_b200/data/*.bin) are embedded into the library
as a generated include, so the .so is self-contained.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "_build"
LIB = PKG / "libcenote_b200.so"

CU_SOURCES = ["wavefront.cu", "probes.cu", "env_build.cu", "guide.cu", "bvh_gpu.cu"]
CPP_SOURCES = ["capi.cpp", "runtime.cpp", "server.cpp", "guide_api.cpp", "bvh_build.cpp", "texture_prep.cpp",
               "bc7_encode.cpp", "bc6h_encode.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _cuda_include(nvcc: str) -> Path:
    return Path(nvcc).resolve().parent.parent / "include"


def _tables_blob() -> Path:
    """ggx_energy.bin ++ ltc_sheen.bin as 32-bit words for capi.cpp."""
    data = (PKG / "data" / "ggx_energy.bin").read_bytes() + (PKG / "data" / "ltc_sheen.bin").read_bytes()
    assert len(data) == 16928 * 4, len(data)
    words = [int.from_bytes(data[i:i + 4], "little") for i in range(0, len(data), 4)]
    lines = []
    for i in range(0, len(words), 8):
        lines.append(", ".join(f"0x{w:08x}u" for w in words[i:i + 8]) + ",")
    path = OUT / "tables_blob.inc"
    text = "\n".join(lines) + "\n"
    if not path.exists() or path.read_text() != text:
        path.write_text(text)
    return path


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(map(str, cmd)) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")
    return r


def build(verbose: bool = False, ptxas_info: bool = False, defines=(), out_dir: Path | None = None,
          lib: Path | None = None) -> Path:
    """Compile and link. `defines`, `out_dir` and `lib` build tuning variants
    of the library side by side (objects and .so elsewhere than the default)."""
    out = Path(out_dir) if out_dir else OUT
    lib = Path(lib) if lib else LIB
    out.mkdir(parents=True, exist_ok=True)
    nvcc = _nvcc()
    inc = _tables_blob().parent
    dflags = [f"-D{d}" for d in defines]
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "cenote_c.h"]
    newest_header = max(p.stat().st_mtime for p in headers)
    objs = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = out / (src + ".o")
        objs.append(o)
        if o.exists() and o.stat().st_mtime > max(s.stat().st_mtime, newest_header) and not ptxas_info:
            continue
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
               *dflags, "-c", str(s), "-o", str(o)]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        r = _run(cmd)
        if verbose or ptxas_info:
            sys.stderr.write(r.stderr)
    for src in CPP_SOURCES:
        s = CSRC / src
        o = out / (src + ".o")
        objs.append(o)
        if o.exists() and o.stat().st_mtime > max(s.stat().st_mtime, newest_header,
                                                  (inc / "tables_blob.inc").stat().st_mtime):
            continue
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra", "-Wno-unused-parameter",
              *dflags, f"-I{_cuda_include(nvcc)}", f"-I{inc}", "-c", str(s), "-o", str(o)])
    if not lib.exists() or lib.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        _run([nvcc, *ARCH, "-shared", "-o", str(lib), *map(str, objs), "-lpthread"])
    return lib


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
