"""Generate the committed golden vectors under tests/golden/.

    python tests/golden/make_golden.py

sampler.npz: the first 256 (sample_2d, sample_1d) draws of nine (pixel,
dimension) keys from the CPU oracle's restatement of
crates/cenote/shaders/rng.slang. The reference ships no sampler vectors (its
test checks stratification only), so these pin the restatement against drift;
the GPU test checks the kernels against the oracle and against this file.
"""
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402

KEYS = [(0, 0), (7, 0), (123456, 3), (1, 1), (65535, 8), (921599, 9), (2**31 + 5, 12), (42, 103), (5, 2)]


def main():
    pts, vals = [], []
    for pixel, dim in KEYS:
        p, v = oracle.sampler(pixel, dim, 256)
        pts.append(p)
        vals.append(v)
    out = pathlib.Path(__file__).parent / "sampler.npz"
    np.savez_compressed(out, keys=np.array(KEYS, np.uint32), points=np.stack(pts), values=np.stack(vals))
    print(out)


if __name__ == "__main__":
    main()
