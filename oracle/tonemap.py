"""CPU oracle of the display transform — test infrastructure only.

A float32 numpy restatement of crates/cenote/shaders/tonemap.slang:16-99 (the
reference's own CPU mirror is crates/cenote/src/render/tonemap.rs:209-247):
exposure by 2^stops, ACEScg -> linear Rec.709 (SRGB_FROM_ACESCG), Stephen
Hill's analytic RRT+ODT fit (BakingLab; sRGB -> AP1 with the RRT saturation,
the rational curve, back to linear Rec.709), saturate, the sRGB transfer
(IEC 61966-2-1), round(saturate(c) * 255) and the RGBA8 pack with R in the low
byte and opaque alpha. Pinned to the reference's known-answer test
(tonemap.rs:171-207): six pixels at exposure 0.5, +-1 quantisation step.
"""
from __future__ import annotations

import numpy as np

F = np.float32
SRGB_FROM_ACESCG = np.array([[1.705050993, -0.621792121, -0.083258872],
                             [-0.130256418, 1.140804737, -0.010548319],
                             [-0.024003357, -0.128968976, 1.152972333]], F)
ACES_INPUT = np.array([[0.59719, 0.35458, 0.04823], [0.07600, 0.90834, 0.01566], [0.02840, 0.13383, 0.83777]], F)
ACES_OUTPUT = np.array([[1.60475, -0.53108, -0.07367], [-0.10208, 1.10813, -0.00605],
                        [-0.00327, -0.07276, 1.07602]], F)


def _mul(m: np.ndarray, v: np.ndarray) -> np.ndarray:
    """Each row summed left to right in float32, as the kernel does."""
    return np.stack([(m[r, 0] * v[..., 0] + m[r, 1] * v[..., 1]) + m[r, 2] * v[..., 2] for r in range(3)], -1)


def aces_display(acescg: np.ndarray) -> np.ndarray:
    """Display-linear Rec.709 in [0, 1] from linear ACEScg (tonemap.slang:51-62)."""
    v = _mul(ACES_INPUT, _mul(SRGB_FROM_ACESCG, acescg.astype(F)))
    a = v * (v + F(0.0245786)) - F(0.000090537)
    b = v * (F(0.983729) * v + F(0.4329510)) + F(0.238081)
    return np.clip(_mul(ACES_OUTPUT, a / b), F(0), F(1))


def srgb_encode(c: np.ndarray) -> np.ndarray:
    c = c.astype(F)
    with np.errstate(invalid="ignore"):
        hi = F(1.055) * np.power(np.maximum(c, F(0)), F(1.0 / 2.4)) - F(0.055)
    return np.where(c <= F(0.0031308), F(12.92) * c, hi).astype(F)


def tonemap(average: np.ndarray, exposure_stops: float) -> np.ndarray:
    """uint8 (..., 4) display texels from float (..., >=3) linear ACEScg averages."""
    rgb = average[..., :3].astype(F) * F(np.exp2(F(exposure_stops)))
    q = np.floor(np.clip(srgb_encode(aces_display(rgb)), 0, 1) * F(255) + F(0.5)).astype(np.uint8)
    return np.concatenate([q, np.full(q.shape[:-1] + (1,), 255, np.uint8)], -1)
