"""The tiled camera-path order (wave_pixel in cenote_b200/csrc/wavefront.h)
visits every pixel of the image exactly once, and 32 consecutive paths land
in one 8 x 4 block. Compiled here as host code with g++; no GPU."""
import pathlib
import shutil
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]

PROGRAM = r"""
#include <cstdio>
#include <cstdint>
#include <vector>
#define __host__
#define __device__
#include "wave_pixel_only.h"
int main() {
    const uint32_t sizes[][2] = {{8, 4}, {16, 8}, {1920, 1080}, {1280, 720}, {640, 360}, {256, 256}};
    for (auto& wh : sizes) {
        const uint32_t w = wh[0], h = wh[1];
        std::vector<uint8_t> seen(size_t(w) * h, 0);
        for (uint32_t j = 0; j < w * h; ++j) {
            const uint32_t p = wave_pixel(j, w);
            if (p >= w * h || seen[p]++) { std::printf("bad %u %u %u\n", w, h, j); return 1; }
            const uint32_t q = wave_pixel(j & ~31u, w);
            if (p / w / 4 != q / w / 4 || p % w / 8 != q % w / 8) { std::printf("tile %u %u %u\n", w, h, j); return 1; }
        }
        if (wave_pixel(77, 0) != 77) return 1;
    }
    std::puts("ok");
    return 0;
}
"""


def test_wave_pixel_is_a_tiled_bijection(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    src = (ROOT / "cenote_b200" / "csrc" / "wavefront.h").read_text()
    start = src.index("__host__ __device__ inline uint32_t wave_pixel")
    end = src.index("\n}\n", start) + 3
    (tmp_path / "wave_pixel_only.h").write_text("#include <cstdint>\n" + src[start:end])
    (tmp_path / "t.cpp").write_text(PROGRAM)
    subprocess.run(["g++", "-O1", "-I", str(tmp_path), "-o", str(tmp_path / "t"), str(tmp_path / "t.cpp")], check=True)
    out = subprocess.run([str(tmp_path / "t")], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout
