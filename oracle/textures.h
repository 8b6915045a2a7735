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
// Block decoding follows the published BCn layouts (Microsoft's "Texture
// Block Compression in Direct3D 11" / the Khronos Data Format Specification,
// "S3TC" and "RGTC" sections): BC1 = two RGB565 endpoints and 2-bit indices,
// four-colour mode when c0 > c1, else three colours and transparent black; BC4
// = two 8-bit endpoints and 3-bit indices, eight-value mode when r0 > r1, else
// six values plus 0 and 1; BC5 = two BC4 blocks (red, then green). Palette
// entries are computed in float from the 8-bit-expanded endpoints.
//
// The bilinear weights are quantised to 1/256, the 8-bit fraction CUDA's
// texture unit documents for linear filtering; a hardware tap and this one
// may still differ by a rounding of that fraction and of the palette, which
// the parity tests bound.
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
    for (int k = 0; k < 2; ++k) {
        uint32_t r5 = (c[k] >> 11) & 31u, g6 = (c[k] >> 5) & 63u, b5 = c[k] & 31u;
        pal[k][0] = float((r5 << 3) | (r5 >> 2));
        pal[k][1] = float((g6 << 2) | (g6 >> 4));
        pal[k][2] = float((b5 << 3) | (b5 >> 2));
        pal[k][3] = 255.0f;
    }
    for (int i = 0; i < 3; ++i) {
        if (c[0] > c[1]) {
            pal[2][i] = (2.0f * pal[0][i] + pal[1][i]) / 3.0f;
            pal[3][i] = (pal[0][i] + 2.0f * pal[1][i]) / 3.0f;
        } else {
            pal[2][i] = (pal[0][i] + pal[1][i]) / 2.0f;
            pal[3][i] = 0.0f;
        }
    }
    pal[2][3] = 255.0f;
    pal[3][3] = c[0] > c[1] ? 255.0f : 0.0f;
}

inline void bc4_palette(const uint8_t* b, float pal[8]) {
    float r0 = b[0], r1 = b[1];
    pal[0] = r0;
    pal[1] = r1;
    if (b[0] > b[1]) {
        for (int k = 1; k <= 6; ++k) pal[1 + k] = (float(7 - k) * r0 + float(k) * r1) / 7.0f;
    } else {
        for (int k = 1; k <= 4; ++k) pal[1 + k] = (float(5 - k) * r0 + float(k) * r1) / 5.0f;
        pal[6] = 0.0f;
        pal[7] = 255.0f;
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
                            o[0] = pr[bc4_index(b, t)] / 255.0f;
                            o[1] = 0.0f;
                            if (format == TEX_BC5_UNORM) {
                                float pg[8];
                                bc4_palette(b + 8, pg);
                                o[1] = pg[bc4_index(b + 8, t)] / 255.0f;
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
        auto axis = [](float c, uint32_t n, uint32_t* i0, uint32_t* i1, float* a) {
            float x = (c - std::floor(c)) * float(n) - 0.5f;
            float f = std::floor(x);
            float frac = std::nearbyint((x - f) * 256.0f) / 256.0f;
            int64_t i = int64_t(f);
            if (frac >= 1.0f) {
                frac = 0.0f;
                i += 1;
            }
            int64_t m = int64_t(n);
            *i0 = uint32_t(((i % m) + m) % m);
            *i1 = uint32_t((((i + 1) % m) + m) % m);
            *a = frac;
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
