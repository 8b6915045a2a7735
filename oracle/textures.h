// Test infrastructure (CPU oracle): material textures, restated.
//
// What the reference's bindless table does per tap (shaders/textures.slang:
// 24-82, samplers of crates/cenote/src/gpu/image.rs:117-141): one level,
// bilinear filtering, repeat addressing on both axes, sRGB-stored colour
// decoded per texel before filtering, then Rec.709 -> ACEScg for colour slots,
// the red channel for scalars, and x/y -> unit z for tangent-space normals.
//
// The formats are the ones the CUDA path accepts (cenote_c.h): RGBA8 (sRGB or
// linear), RGBA32F, and block-compressed BC1 (sRGB or linear), BC4 and BC5.
// Block layouts follow the published BCn formats (Microsoft's "Texture Block
// Compression in Direct3D 11" / the Khronos Data Format Specification, "S3TC"
// and "RGTC" sections): BC1 = two RGB565 endpoints and 2-bit indices,
// four-colour mode when c0 > c1, else three colours and transparent black; BC4
// = two 8-bit endpoints and 3-bit indices, eight-value mode when r0 > r1, else
// six values plus 0 and 1; BC5 = two BC4 blocks (red, then green).
//
// Those formats leave the interpolated palette entries' precision to the
// decoder; the reference decodes with its GPU's texture unit, as the CUDA
// path does. The palettes here are the B200 texture unit's, measured through
// cenote_probe_texture on random blocks at texel centres (every one of 65,536
// texels per format reproduced exactly; tests/test_textures.py keeps the
// device and this decoder bit-equal):
//  * BC1 returns 8-bit levels. Endpoints expand by bit replication. The
//    5-bit channels interpolate from the raw 5-bit values, as
//    floor(11 (2 a + b) / 4) for the one-third entries and
//    floor(33 (a + b) / 8) for the three-colour midpoint; the 6-bit channel
//    interpolates from the expanded 8-bit values E0, E1 with d = E1 - E0 as
//    floor((256 E0 + n d + floor(d / 4) + 128) / 256), n = 80 for a
//    one-third entry and 128 for the midpoint.
//  * BC4 and BC5 return 16-bit levels: entry = (a r0 + b r1) / 65535 with
//    integer weights a + b = 257 (endpoints r·257), in eight-value mode
//    (221, 36), (185, 72), (144, 113) and their mirrors, in six-value mode
//    (209, 48), (161, 96) and their mirrors.
//
// The bilinear weights are quantised to 1/256, the 8-bit fraction CUDA's
// texture unit documents for linear filtering: the unit scales the
// coordinate by the texture's size in FP32, rounds it to 1/256 of a texel
// (halves up) and wraps it after (as measured on random coordinates: every
// tap of 64- and 1024-texel axes reproduced). sRGB texels decode exactly here; the unit's own decode and its
// filtering of sRGB texels keep a lower precision (within 0.4 % of a texel's
// value), which the parity tests bound.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace oracle {

enum TexFormat : uint32_t {
    TEX_RGBA8_SRGB = 1,
    TEX_RGBA8_UNORM = 2,
    TEX_RGBA32F = 3,
    TEX_BC1_SRGB = 4,
    TEX_BC1_UNORM = 5,
    TEX_BC4_UNORM = 6,
    TEX_BC5_UNORM = 7,
};

inline float srgb_decode(float v) {
    return v <= 0.04045f ? v / 12.92f : std::pow((v + 0.055f) / 1.055f, 2.4f);
}

inline void bc1_palette(const uint8_t* b, float pal[4][4]) {
    uint16_t c[2];
    std::memcpy(c, b, 4);
    const bool four = c[0] > c[1];
    auto floor_div = [](int32_t x, int32_t d) { return x >= 0 ? x / d : -((-x + d - 1) / d); };
    for (int ch = 0; ch < 3; ++ch) {
        const int shift = ch == 0 ? 11 : (ch == 1 ? 5 : 0);
        const int bits = ch == 1 ? 6 : 5;
        const int32_t mask = (1 << bits) - 1;
        const int32_t a = (c[0] >> shift) & mask, bb = (c[1] >> shift) & mask;
        const int32_t e0 = bits == 6 ? (a << 2) | (a >> 4) : (a << 3) | (a >> 2);
        const int32_t e1 = bits == 6 ? (bb << 2) | (bb >> 4) : (bb << 3) | (bb >> 2);
        int32_t p2, p3 = 0;
        if (bits == 6) {
            auto interp = [&](int32_t ea, int32_t eb, int32_t n) {
                const int32_t d = eb - ea;
                return floor_div(256 * ea + n * d + floor_div(d, 4) + 128, 256);
            };
            p2 = four ? interp(e0, e1, 80) : interp(e0, e1, 128);
            if (four) p3 = interp(e1, e0, 80);
        } else {
            p2 = four ? (11 * (2 * a + bb)) / 4 : (33 * (a + bb)) / 8;
            if (four) p3 = (11 * (a + 2 * bb)) / 4;
        }
        pal[0][ch] = float(e0);
        pal[1][ch] = float(e1);
        pal[2][ch] = float(p2);
        pal[3][ch] = float(p3);
    }
    pal[0][3] = pal[1][3] = pal[2][3] = 255.0f;
    pal[3][3] = four ? 255.0f : 0.0f;
}

// BC4 palette in 16-bit levels (0..65535).
inline void bc4_palette(const uint8_t* b, float pal[8]) {
    static const int32_t w8[6][2] = {{221, 36}, {185, 72}, {144, 113}, {113, 144}, {72, 185}, {36, 221}};
    static const int32_t w6[4][2] = {{209, 48}, {161, 96}, {96, 161}, {48, 209}};
    const int32_t r0 = b[0], r1 = b[1];
    pal[0] = float(257 * r0);
    pal[1] = float(257 * r1);
    if (r0 > r1) {
        for (int k = 0; k < 6; ++k) pal[2 + k] = float(w8[k][0] * r0 + w8[k][1] * r1);
    } else {
        for (int k = 0; k < 4; ++k) pal[2 + k] = float(w6[k][0] * r0 + w6[k][1] * r1);
        pal[6] = 0.0f;
        pal[7] = 65535.0f;
    }
}

inline uint32_t bc4_index(const uint8_t* b, int texel) {
    uint64_t bits = 0;
    for (int k = 0; k < 6; ++k) bits |= uint64_t(b[2 + k]) << (8 * k);
    return uint32_t(bits >> (3 * texel)) & 7u;
}

// A decoded texture: linear RGBA float texels, row 0 first.
struct Texture {
    uint32_t width = 0, height = 0;
    std::vector<float> texels;

    const float* at(uint32_t x, uint32_t y) const { return &texels[4 * (size_t(y) * width + x)]; }

    // Decode `data` of the given format; false on an unknown format or BC
    // dimensions that are not multiples of 4.
    bool decode(uint32_t format, uint32_t w, uint32_t h, const void* data) {
        width = w;
        height = h;
        texels.assign(size_t(4) * w * h, 0.0f);
        const uint8_t* p = static_cast<const uint8_t*>(data);
        switch (format) {
        case TEX_RGBA8_SRGB:
        case TEX_RGBA8_UNORM:
            for (size_t i = 0; i < size_t(w) * h; ++i)
                for (int c = 0; c < 4; ++c) {
                    float v = float(p[4 * i + c]) / 255.0f;
                    texels[4 * i + c] = (format == TEX_RGBA8_SRGB && c < 3) ? srgb_decode(v) : v;
                }
            return true;
        case TEX_RGBA32F:
            std::memcpy(texels.data(), data, texels.size() * 4);
            return true;
        case TEX_BC1_SRGB:
        case TEX_BC1_UNORM:
        case TEX_BC4_UNORM:
        case TEX_BC5_UNORM: {
            if (w % 4 || h % 4) return false;
            const size_t block = (format == TEX_BC5_UNORM) ? 16 : 8;
            const uint32_t bw = w / 4, bh = h / 4;
            for (uint32_t by = 0; by < bh; ++by)
                for (uint32_t bx = 0; bx < bw; ++bx) {
                    const uint8_t* b = p + block * (size_t(by) * bw + bx);
                    for (int t = 0; t < 16; ++t) {
                        float* o = &texels[4 * ((size_t(by) * 4 + t / 4) * w + bx * 4 + t % 4)];
                        if (format == TEX_BC1_SRGB || format == TEX_BC1_UNORM) {
                            float pal[4][4];
                            bc1_palette(b, pal);
                            uint32_t idx;
                            std::memcpy(&idx, b + 4, 4);
                            const float* e = pal[(idx >> (2 * t)) & 3u];
                            for (int c = 0; c < 4; ++c) {
                                float v = e[c] / 255.0f;
                                o[c] = (format == TEX_BC1_SRGB && c < 3) ? srgb_decode(v) : v;
                            }
                        } else {
                            float pr[8];
                            bc4_palette(b, pr);
                            o[0] = float(double(pr[bc4_index(b, t)]) / 65535.0);
                            o[1] = 0.0f;
                            if (format == TEX_BC5_UNORM) {
                                float pg[8];
                                bc4_palette(b + 8, pg);
                                o[1] = float(double(pg[bc4_index(b + 8, t)]) / 65535.0);
                            }
                            o[2] = 0.0f;
                            o[3] = 1.0f;
                        }
                    }
                }
            return true;
        }
        default:
            return false;
        }
    }

    // One bilinear tap at normalised (u, v), repeat addressing.
    void sample(float u, float v, float out[4]) const {
        // The texel-space coordinate c·n in FP32, quantised to 1/256 of a
        // texel (halves up), less half a texel, then wrapped: its integer
        // part picks the texels, its fraction is the weight (the unit's
        // coordinate path as measured; exact for power-of-two sizes).
        auto axis = [](float c, uint32_t n, uint32_t* i0, uint32_t* i1, float* a) {
            const float xs = c * float(n);
            const int64_t q = int64_t(std::floor(double(xs) * 256.0 + 0.5)) - 128;
            const int64_t i = q >= 0 ? q / 256 : -((-q + 255) / 256);
            const int64_t m = int64_t(n);
            *i0 = uint32_t(((i % m) + m) % m);
            *i1 = uint32_t((((i + 1) % m) + m) % m);
            *a = float(q - i * 256) / 256.0f;
        };
        uint32_t x0, x1, y0, y1;
        float a, b;
        axis(u, width, &x0, &x1, &a);
        axis(v, height, &y0, &y1, &b);
        const float *t00 = at(x0, y0), *t10 = at(x1, y0), *t01 = at(x0, y1), *t11 = at(x1, y1);
        for (int c = 0; c < 4; ++c)
            out[c] = (1.0f - a) * (1.0f - b) * t00[c] + a * (1.0f - b) * t10[c] + (1.0f - a) * b * t01[c] +
                     a * b * t11[c];
    }
};

}  // namespace oracle
