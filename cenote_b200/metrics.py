"""Image metrics: relMSE and LDR-FLIP.

LDR-FLIP follows Andersson et al., "FLIP: A Difference Evaluator for
Alternating Images" (HPG 2020): a colour pipeline (sRGB → YCxCz, contrast-
sensitivity filtering, Hunt-adjusted L*a*b*, HyAB distance compressed with
q_c = 0.7, p_c = 0.4, p_t = 0.95) and a feature pipeline (edge and point
detectors on normalised luminance, q_f = 0.5), combined per pixel as
ΔE_c^(1 − ΔE_f). The reference compares renders with the `nv-flip` crate
(0.1.2); this is written from the paper, so agreement with that crate's values
is not pinned bit for bit (identical images score exactly 0 either way).
`flip_ldr_linear` applies the reference's own preprocessing: clamp linear
values to [0, 1], quantise to 8 bits, and hand the bytes to FLIP as sRGB
(crates/cenote/tests/golden.rs:144-157).
"""
from __future__ import annotations

import numpy as np
from scipy import ndimage

PPD = 67.0206  # 0.7 m viewing distance, 0.7 m-wide 3840-pixel display

_RGB2XYZ = np.array([[10135552 / 24577794, 8788810 / 24577794, 4435075 / 24577794],
                     [2613072 / 12288897, 8788810 / 12288897, 887015 / 12288897],
                     [1425312 / 73733382, 8788810 / 73733382, 70074185 / 73733382]])
_XYZ2RGB = np.linalg.inv(_RGB2XYZ)
_WHITE = _RGB2XYZ @ np.ones(3)


def rel_mse(test: np.ndarray, ref: np.ndarray, eps: float = 1e-2) -> float:
    t, r = np.asarray(test, np.float64), np.asarray(ref, np.float64)
    return float(np.mean((t - r) ** 2 / (r ** 2 + eps)))


def _srgb_to_linear(c):
    return np.where(c <= 0.04045, c / 12.92, ((c + 0.055) / 1.055) ** 2.4)


def _xyz_to_ycxcz(xyz):
    x, y, z = (xyz[..., k] / _WHITE[k] for k in range(3))
    return np.stack([116.0 * y - 16.0, 500.0 * (x - y), 200.0 * (y - z)], -1)


def _ycxcz_to_xyz(v):
    y = (v[..., 0] + 16.0) / 116.0
    x = v[..., 1] / 500.0 + y
    z = y - v[..., 2] / 200.0
    return np.stack([x * _WHITE[0], y * _WHITE[1], z * _WHITE[2]], -1)


def _lab_hunt(lin):
    xyz = lin @ _RGB2XYZ.T / _WHITE
    d = 6.0 / 29.0
    f = np.where(xyz > d ** 3, np.cbrt(xyz), xyz / (3 * d * d) + 4.0 / 29.0)
    L = 116.0 * f[..., 1] - 16.0
    a = 500.0 * (f[..., 0] - f[..., 1])
    b = 200.0 * (f[..., 1] - f[..., 2])
    return np.stack([L, 0.01 * L * a, 0.01 * L * b], -1)


def _hyab(p, q):
    d = p - q
    return np.abs(d[..., 0]) + np.sqrt(d[..., 1] ** 2 + d[..., 2] ** 2)


def _csf_kernels(ppd):
    params = [(1.0, 0.0047, 0.0, 1e-5), (1.0, 0.0053, 0.0, 1e-5), (34.1, 0.04, 13.5, 0.025)]
    bmax = max(max(b1, b2) for _, b1, _, b2 in params)
    r = int(np.ceil(3.0 * np.sqrt(bmax / (2.0 * np.pi ** 2)) * ppd))
    x, y = np.meshgrid(np.arange(-r, r + 1), np.arange(-r, r + 1))
    z = (x / ppd) ** 2 + (y / ppd) ** 2
    out = []
    for a1, b1, a2, b2 in params:
        g = a1 * np.sqrt(np.pi / b1) * np.exp(-np.pi ** 2 * z / b1) + a2 * np.sqrt(np.pi / b2) * np.exp(-np.pi ** 2 * z / b2)
        out.append(g / g.sum())
    return out


def _feature_kernels(ppd):
    sd = 0.5 * 0.082 * ppd
    r = int(np.ceil(3 * sd))
    x, y = np.meshgrid(np.arange(-r, r + 1), np.arange(-r, r + 1))
    g = np.exp(-(x ** 2 + y ** 2) / (2 * sd * sd))
    out = []
    for gx in (-x * g, (x ** 2 / (sd * sd) - 1) * g):
        gx = np.where(gx < 0, gx / -gx[gx < 0].sum(), gx / gx[gx > 0].sum())
        out.append((gx, gx.T))
    return out


def _conv(img, k):
    return ndimage.convolve(img, k, mode="reflect")


def flip_map(ref_srgb: np.ndarray, test_srgb: np.ndarray, ppd: float = PPD) -> np.ndarray:
    """Per-pixel LDR-FLIP error for sRGB-encoded images in [0, 1], (H, W, 3)."""
    qc, qf, pc, pt = 0.7, 0.5, 0.4, 0.95
    ref_lin = _srgb_to_linear(np.asarray(ref_srgb, np.float64))
    test_lin = _srgb_to_linear(np.asarray(test_srgb, np.float64))
    ks = _csf_kernels(ppd)

    def filtered(lin):
        ycc = _xyz_to_ycxcz(lin @ _RGB2XYZ.T)
        f = np.stack([_conv(ycc[..., c], ks[c]) for c in range(3)], -1)
        return np.clip(_ycxcz_to_xyz(f) @ _XYZ2RGB.T, 0.0, 1.0)

    de = _hyab(_lab_hunt(filtered(ref_lin)), _lab_hunt(filtered(test_lin))) ** qc
    cmax = _hyab(_lab_hunt(np.array([0.0, 1.0, 0.0])), _lab_hunt(np.array([0.0, 0.0, 1.0]))) ** qc
    pccmax = pc * cmax
    dec = np.where(de < pccmax, (pt / pccmax) * de, pt + (de - pccmax) / (cmax - pccmax) * (1.0 - pt))

    (ex, ey), (px, py) = _feature_kernels(ppd)

    def features(lin):
        yn = (_xyz_to_ycxcz(lin @ _RGB2XYZ.T)[..., 0] + 16.0) / 116.0
        e = np.hypot(_conv(yn, ex), _conv(yn, ey))
        p = np.hypot(_conv(yn, px), _conv(yn, py))
        return e, p

    er, pr = features(ref_lin)
    et, ptt = features(test_lin)
    def_ = (np.maximum(np.abs(er - et), np.abs(pr - ptt)) / np.sqrt(2.0)) ** qf
    return dec ** (1.0 - def_)


def to_ldr8(linear_rgb: np.ndarray) -> np.ndarray:
    """The reference's FLIP input: clamp to [0, 1], scale by 255 in f32 and
    round halves away from zero (Rust's f32::round), as 8-bit levels / 255."""
    x = np.clip(np.asarray(linear_rgb, np.float32), np.float32(0), np.float32(1)) * np.float32(255)
    fl = np.floor(x)
    return np.where(x - fl >= np.float32(0.5), fl + 1, fl).astype(np.float64) / 255.0


def flip_ldr_linear(ref_linear: np.ndarray, test_linear: np.ndarray) -> float:
    """Mean LDR-FLIP between two linear renders, preprocessed like the reference's golden tests."""
    return float(flip_map(to_ldr8(ref_linear[..., :3]), to_ldr8(test_linear[..., :3])).mean())
