"""Measures the B200 texture unit's filtering (test infrastructure, run on a GPU).

The oracle's texture model (oracle/textures.h) restates what the unit returns:
the coordinate and weight quantisation, 16-bit levels for linear channels, and
for sRGB channels a decode to an 8-bit mantissa with an exponent fixed per
range of values. This script measures those facts through the library's
texel probe (cenote_probe_texture) and writes

  * tests/golden/texture_unit_taps.npz: per format a random 32x32 texture,
    taps at texel centres, on texel-centre rows (one axis filtered) and at
    random coordinates, and what the unit returned; tests/test_textures.py
    checks the oracle against these taps on the CPU;
  * on stdout, the sRGB decode table as the oracle declares it (SRGB_M,
    SRGB_E), and whether the oracle's model reproduces every tap.

    python oracle/measure_texture_unit.py [output.npz]
"""
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from cenote_b200 import Context, Scene, scenes as T  # noqa: E402

FORMATS = {
    "rgba8_srgb": (T.TEX_RGBA8_SRGB, 0),
    "rgba8_unorm": (T.TEX_RGBA8_UNORM, 0),
    "rgba32f": (T.TEX_RGBA32F, -1),
    "bc1_srgb": (T.TEX_BC1_SRGB, 8),
    "bc1_unorm": (T.TEX_BC1_UNORM, 8),
    "bc4": (T.TEX_BC4_UNORM, 8),
    "bc5": (T.TEX_BC5_UNORM, 16),
    "bc7_srgb": (T.TEX_BC7_SRGB, 16),
    "bc7_unorm": (T.TEX_BC7_UNORM, 16),
    "bc6h_uf16": (T.TEX_BC6H_UF16, 16),
    "bc6h_sf16": (T.TEX_BC6H_SF16, 16),
}

# BC6H mode bits (two for modes 1-2, five for the rest) and one reserved value.
BC6H_MODE_BITS = [0, 1, 2, 6, 10, 14, 18, 22, 26, 30, 3, 7, 11, 15, 19]


def bc6h_blocks(n, rng):
    """n random BC6H blocks cycling through the fourteen modes and a reserved one."""
    b = rng.integers(0, 256, (n, 16), dtype=np.uint8)
    for k in range(n):
        mv = BC6H_MODE_BITS[k % len(BC6H_MODE_BITS)]
        mask = 3 if mv < 2 else 31
        b[k, 0] = (int(b[k, 0]) & ~mask & 255) | mv
    return b.reshape(-1)


def bc7_blocks(n, rng):
    """n random BC7 blocks cycling through the eight modes and the invalid
    ninth (no mode bit in the first byte)."""
    b = rng.integers(0, 256, (n, 16), dtype=np.uint8)
    for k in range(n):
        mode = k % 9
        b[k, 0] = 0 if mode == 8 else (int(b[k, 0]) & ~((1 << (mode + 1)) - 1) & 255) | (1 << mode)
    return b.reshape(-1)


def random_texture(fmt, bpb, size, rng):
    if bpb == 0:
        data = rng.integers(0, 256, size * size * 4, dtype=np.uint8)
    elif bpb < 0:
        data = (rng.random((size, size, 4)) * 4.0).astype(np.float32)
    elif fmt in (T.TEX_BC7_SRGB, T.TEX_BC7_UNORM):
        data = bc7_blocks((size // 4) * (size // 4), rng)
    elif fmt in (T.TEX_BC6H_UF16, T.TEX_BC6H_SF16):
        data = bc6h_blocks((size // 4) * (size // 4), rng)
    else:
        data = rng.integers(0, 256, (size // 4) * (size // 4) * bpb, dtype=np.uint8)
    return T.Texture(fmt, size, size, data)


def probe(ctx, tex, uv):
    spec = T.cornell(8, 8, 1, 2)
    spec.textures = [tex]
    return Scene(ctx, spec).probe_texture(0, np.ascontiguousarray(uv, np.float32), 0)


def golden_taps(ctx, rng, size=32, taps=1000):
    out = {}
    centres = (np.stack(np.meshgrid(np.arange(size), np.arange(size)), -1).reshape(-1, 2) + 0.5) / size
    rows = (rng.integers(0, size, taps) + 0.5) / size
    for name, (fmt, bpb) in FORMATS.items():
        tex = random_texture(fmt, bpb, size, rng)
        uv = np.concatenate([centres, np.stack([rng.random(taps), rows], -1), rng.random((taps, 2))])
        uv = uv.astype(np.float32)
        out[f"{name}_data"] = np.asarray(tex.data).reshape(-1).view(np.uint8)
        out[f"{name}_uv"] = uv
        out[f"{name}_taps"] = probe(ctx, tex, uv)
    return out


def fp16_half_up(s, e):
    """s · 2^(e - 16) for an integer s >= 0, rounded to FP16, ties away from zero."""
    if s == 0:
        return 0.0
    lead = s.bit_length() - 1 + e - 16
    drop = (max(lead, -14) - 10) - (e - 16)
    if drop > 0:
        s = ((s + (1 << (drop - 1))) >> drop) << drop
    return float(np.ldexp(float(s), e - 16))


def srgb_table(ctx):
    """Mantissa and exponent of the unit's decode of each sRGB value: the
    value at a texel centre, then the exponent (the value's binade or one
    above) that explains half-way taps between it and 48 darker values."""
    w, h = 512, 16
    px = np.zeros((h, w, 4), np.uint8)
    px[..., 3] = 255
    for k in range(256):
        px[:, 2 * k, :3] = k
        px[:, 2 * k + 1, :3] = np.linspace(0, max(k - 1, 0), 48).astype(np.uint8).reshape(h, 3)
    tex = T.Texture(T.TEX_RGBA8_SRGB, w, h, px.reshape(-1).copy())
    ys = (np.arange(h) + 0.5) / h
    centre = probe(ctx, tex, np.stack([(2 * np.arange(256) + 0.5) / w, np.full(256, ys[0])], -1))[:, 0]
    uv = np.stack(np.meshgrid((2 * np.arange(256) + 1.0) / w, ys), -1).reshape(-1, 2)  # weights 128 / 128
    half = probe(ctx, tex, uv).reshape(h, 256, 4)[..., :3]
    m_out, e_out = np.zeros(256, np.int64), np.full(256, -126, np.int64)
    for k in range(1, 256):
        e0 = int(np.frexp(np.float64(centre[k]))[1])
        for e in (e0, e0 + 1):
            m = float(centre[k]) * 2.0 ** (8 - e)
            if m != np.floor(m) or m > 255:
                continue
            ok = True
            for r in range(h):
                for c in range(3):
                    p = int(px[r, 2 * k + 1, c])
                    ep = int(e_out[p]) if p else e
                    eb = max(e, ep)  # the pair shares the larger exponent
                    q = int(m_out[p]) >> (eb - ep) if eb - ep < 8 else 0
                    s = 128 * (int(m) >> (eb - e)) + 128 * q
                    ok &= np.float32(fp16_half_up(s, eb)) == half[r, k, c]
            if ok:
                m_out[k], e_out[k] = int(m), e
                break
        else:
            raise RuntimeError(f"no exponent explains sRGB value {k}")
    return m_out, e_out


def main():
    ctx = Context(0)
    rng = np.random.default_rng(20261203)
    taps = golden_taps(ctx, rng)
    out = pathlib.Path(sys.argv[1]) if len(sys.argv) > 1 else ROOT / "tests" / "golden" / "texture_unit_taps.npz"
    np.savez_compressed(out, **taps)
    ok = True
    for name, (fmt, _) in FORMATS.items():
        data = taps[f"{name}_data"]
        if fmt == T.TEX_RGBA32F:
            data = data.view(np.float32).reshape(32, 32, 4)
        tex = T.Texture(fmt, 32, 32, data)
        ref = oracle.texture_sample(tex, taps[f"{name}_uv"], 0)
        same = np.array_equal(ref, taps[f"{name}_taps"])
        ok &= same
        print(f"{name}: oracle {'bit-equal' if same else 'DIFFERS'}, max {np.abs(ref - taps[name + '_taps']).max():.3g}")
    m, e = srgb_table(ctx)
    print("SRGB_M =", ", ".join(map(str, m)))
    print("SRGB_E =", ", ".join(map(str, e)))
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
