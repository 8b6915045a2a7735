"""Writes cenote_b200/csrc/bc7_tables.h: the partition and anchor tables of
the BC7 block format (2- and 3-subset partitions of a 4x4 block, 64 each, and
the texel whose index drops its top bit in each subset).

The tables are part of the published format (Khronos Data Format
Specification, section "BC7"; Direct3D 11 "BC7 format"). They are recovered
here by decoding crafted blocks with an independent BC7 decoder (Pillow's
BCn decoder, which ships in this environment), so no table is typed by hand:

  * partitions: mode 1 (two subsets) and mode 2 (three subsets) blocks whose
    subsets have distinct constant colours and all indices zero; each
    texel's decoded colour names its subset;
  * anchors: the same partitions with every index bit set; an anchor texel
    has one index bit fewer, so it decodes to a lower palette entry.

The texture prep encoder and the oracle's decoder both read the header; the
device never needs it (the texture unit decodes BC7 itself), and the GPU
tests hold the unit and the oracle's decoder bit-equal on random blocks of
every mode.

    python -m cenote_b200.bc7_tables      # rewrites the header
"""
import pathlib

import numpy as np

HEADER = pathlib.Path(__file__).resolve().parent / "csrc" / "bc7_tables.h"


class Bits:
    def __init__(self):
        self.v, self.n = 0, 0

    def put(self, value, count):
        self.v |= (value & ((1 << count) - 1)) << self.n
        self.n += count

    def block(self):
        assert self.n <= 128
        return self.v.to_bytes(16, "little")


def _decode(blocks):
    from PIL import Image

    n = len(blocks)
    img = Image.frombytes("RGBA", (4 * n, 4), b"".join(blocks), "bcn", 7)
    a = np.asarray(img).reshape(4, n, 4, 4).transpose(1, 0, 2, 3)  # block, row, column, channel
    return a.reshape(n, 16, 4)


def _mode1(partition, red, index_ones):
    b = Bits()
    b.put(0b10, 2)  # mode 1: one zero bit, then a one
    b.put(partition, 6)
    for c in range(3):
        for v in (red if c == 0 else (0, 0, 0, 0)):
            b.put(v, 6)
    b.put(0, 2)  # shared p-bits
    b.put((1 << 46) - 1 if index_ones else 0, 46)
    return b.block()


def _mode2(partition, red, index_ones):
    b = Bits()
    b.put(0b100, 3)  # mode 2
    b.put(partition, 6)
    for c in range(3):
        for v in (red if c == 0 else (0,) * 6):
            b.put(v, 5)
    b.put((1 << 29) - 1 if index_ones else 0, 29)
    return b.block()


def tables():
    p2 = _decode([_mode1(p, (0, 0, 63, 63), False) for p in range(64)])[:, :, 0]
    p3 = _decode([_mode2(p, (0, 0, 15, 15, 31, 31), False) for p in range(64)])[:, :, 0]
    part2 = np.searchsorted(np.unique(p2), p2)
    part3 = np.searchsorted(np.unique(p3), p3)
    assert part2.max() == 1 and part3.max() == 2
    a2 = _decode([_mode1(p, (0, 63, 0, 63), True) for p in range(64)])[:, :, 0]
    a3 = _decode([_mode2(p, (0, 31, 0, 31, 0, 31), True) for p in range(64)])[:, :, 0]
    anchor2 = np.zeros(64, np.int64)
    anchor3 = np.zeros((64, 2), np.int64)
    for p in range(64):
        low = np.nonzero(a2[p] != a2[p].max())[0]
        assert low[0] == 0 and len(low) == 2 and part2[p, low[1]] == 1
        anchor2[p] = low[1]
        low = np.nonzero(a3[p] != a3[p].max())[0]
        assert low[0] == 0 and len(low) == 3
        for t in low[1:]:
            anchor3[p, part3[p, t] - 1] = t
        assert part3[p, anchor3[p, 0]] == 1 and part3[p, anchor3[p, 1]] == 2
    return part2, part3, anchor2, anchor3


def main():
    part2, part3, anchor2, anchor3 = tables()

    def rows(a):
        return ",\n".join("    {" + ", ".join(map(str, r)) + "}" for r in a)

    text = f"""// Generated by cenote_b200/bc7_tables.py: the BC7 format's partition and
// anchor tables (Khronos Data Format Specification, "BC7"), recovered by
// decoding crafted blocks. Do not edit by hand.
#pragma once
#include <cstdint>

namespace bc7 {{

// Subset of each texel (row-major in the 4x4 block) for the 64 two-subset
// and the 64 three-subset partitions.
constexpr uint8_t PARTITION2[64][16] = {{
{rows(part2)}}};
constexpr uint8_t PARTITION3[64][16] = {{
{rows(part3)}}};
// The anchor texel of subset 1 (two subsets), and of subsets 1 and 2 (three
// subsets); texel 0 anchors subset 0. An anchor's index omits its top bit.
constexpr uint8_t ANCHOR2[64] = {{{", ".join(map(str, anchor2))}}};
constexpr uint8_t ANCHOR3[64][2] = {{
{rows(anchor3)}}};

}}  // namespace bc7
"""
    HEADER.write_text(text)
    print(HEADER)


if __name__ == "__main__":
    main()
