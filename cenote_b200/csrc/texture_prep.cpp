// Host texture prep: sizes and the BC block encoders, the step
// crates/cenote/src/texture.rs:221-405 runs before upload (there with an
// external BC7/BC6H/BC4/BC5 encoder; here BC7 as the reference's colour
// format, in bc7_encode.cpp, and BC1/BC4/BC5 below).
//
// Encoder, per 4x4 block (written for this library):
//  * BC1: endpoints from the block's principal colour axis (mean + power
//    iteration on the covariance), the two extreme projections quantised to
//    RGB565 and ordered c0 > c1 (four-colour mode); each texel takes the
//    nearest of the four palette colours; one least-squares refit of the
//    endpoints from those indices is kept when it lowers the block's error.
//    A block whose endpoints quantise equal uses index 0 throughout.
//  * BC4: endpoints = the block's max and min (eight-value mode when they
//    differ), nearest palette index per texel. BC5 = BC4 on red, then green.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/cenote_c.h"
#include "texture_prep.h"

namespace cn {

uint64_t texture_bytes(uint32_t format, uint32_t w, uint32_t h) {
    if (w == 0 || h == 0 || w > 32768 || h > 32768) return 0;
    const uint64_t px = uint64_t(w) * h;
    switch (format) {
    case CENOTE_TEXTURE_RGBA8_SRGB:
    case CENOTE_TEXTURE_RGBA8_UNORM:
        return px * 4;
    case CENOTE_TEXTURE_RGBA32F:
        return px * 16;
    case CENOTE_TEXTURE_BC1_SRGB:
    case CENOTE_TEXTURE_BC1_UNORM:
    case CENOTE_TEXTURE_BC4_UNORM:
        return (w % 4 || h % 4) ? 0 : (px / 16) * 8;
    case CENOTE_TEXTURE_BC5_UNORM:
    case CENOTE_TEXTURE_BC7_SRGB:
    case CENOTE_TEXTURE_BC7_UNORM:
    case CENOTE_TEXTURE_BC6H_UF16:
    case CENOTE_TEXTURE_BC6H_SF16:
        return (w % 4 || h % 4) ? 0 : (px / 16) * 16;
    default:
        return 0;
    }
}

namespace {

struct Rgb {
    float r, g, b;
};

uint16_t pack565(Rgb c) {
    auto q = [](float v, int bits) {
        int m = (1 << bits) - 1;
        int x = int(std::lround(std::clamp(v, 0.0f, 255.0f) * float(m) / 255.0f));
        return std::clamp(x, 0, m);
    };
    return uint16_t((q(c.r, 5) << 11) | (q(c.g, 6) << 5) | q(c.b, 5));
}

Rgb unpack565(uint16_t c) {
    uint32_t r5 = (c >> 11) & 31u, g6 = (c >> 5) & 63u, b5 = c & 31u;
    return {float((r5 << 3) | (r5 >> 2)), float((g6 << 2) | (g6 >> 4)), float((b5 << 3) | (b5 >> 2))};
}

float dist2(Rgb a, Rgb b) {
    float dr = a.r - b.r, dg = a.g - b.g, db = a.b - b.b;
    return dr * dr + dg * dg + db * db;
}

// Indices and squared error of a block against endpoints (c0 > c1 assumed).
float bc1_fit(const Rgb* px, uint16_t c0, uint16_t c1, uint32_t* indices) {
    Rgb e0 = unpack565(c0), e1 = unpack565(c1);
    Rgb pal[4] = {e0, e1,
                  {(2 * e0.r + e1.r) / 3, (2 * e0.g + e1.g) / 3, (2 * e0.b + e1.b) / 3},
                  {(e0.r + 2 * e1.r) / 3, (e0.g + 2 * e1.g) / 3, (e0.b + 2 * e1.b) / 3}};
    float err = 0.0f;
    uint32_t idx = 0;
    for (int t = 0; t < 16; ++t) {
        int best = 0;
        float bd = dist2(px[t], pal[0]);
        for (int k = 1; k < 4; ++k) {
            float d = dist2(px[t], pal[k]);
            if (d < bd) {
                bd = d;
                best = k;
            }
        }
        err += bd;
        idx |= uint32_t(best) << (2 * t);
    }
    *indices = idx;
    return err;
}

void write_bc1(uint8_t* out, uint16_t c0, uint16_t c1, uint32_t idx) {
    std::memcpy(out, &c0, 2);
    std::memcpy(out + 2, &c1, 2);
    std::memcpy(out + 4, &idx, 4);
}

void encode_bc1_block(const Rgb* px, uint8_t* out) {
    Rgb mean{0, 0, 0};
    for (int t = 0; t < 16; ++t) {
        mean.r += px[t].r / 16;
        mean.g += px[t].g / 16;
        mean.b += px[t].b / 16;
    }
    float cov[6] = {0, 0, 0, 0, 0, 0};
    for (int t = 0; t < 16; ++t) {
        float r = px[t].r - mean.r, g = px[t].g - mean.g, b = px[t].b - mean.b;
        cov[0] += r * r; cov[1] += r * g; cov[2] += r * b;
        cov[3] += g * g; cov[4] += g * b; cov[5] += b * b;
    }
    float ax[3] = {1.0f, 1.0f, 1.0f};
    for (int it = 0; it < 8; ++it) {
        float x = cov[0] * ax[0] + cov[1] * ax[1] + cov[2] * ax[2];
        float y = cov[1] * ax[0] + cov[3] * ax[1] + cov[4] * ax[2];
        float z = cov[2] * ax[0] + cov[4] * ax[1] + cov[5] * ax[2];
        float n = std::max({std::fabs(x), std::fabs(y), std::fabs(z)});
        if (n <= 0.0f) break;
        ax[0] = x / n;
        ax[1] = y / n;
        ax[2] = z / n;
    }
    float lo = 1e30f, hi = -1e30f;
    for (int t = 0; t < 16; ++t) {
        float p = (px[t].r - mean.r) * ax[0] + (px[t].g - mean.g) * ax[1] + (px[t].b - mean.b) * ax[2];
        lo = std::min(lo, p);
        hi = std::max(hi, p);
    }
    float n2 = ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2];
    if (n2 <= 0.0f) n2 = 1.0f;
    Rgb ea{mean.r + ax[0] * hi / n2, mean.g + ax[1] * hi / n2, mean.b + ax[2] * hi / n2};
    Rgb eb{mean.r + ax[0] * lo / n2, mean.g + ax[1] * lo / n2, mean.b + ax[2] * lo / n2};
    uint16_t c0 = pack565(ea), c1 = pack565(eb);
    if (c0 < c1) std::swap(c0, c1);
    if (c0 == c1) {
        write_bc1(out, c0, c1, 0u);
        return;
    }
    uint32_t idx;
    float err = bc1_fit(px, c0, c1, &idx);
    // Least-squares refit of both endpoints from the chosen indices.
    const float w0[4] = {1.0f, 0.0f, 2.0f / 3.0f, 1.0f / 3.0f};
    float aa = 0, ab = 0, bb = 0;
    Rgb xa{0, 0, 0}, xb{0, 0, 0};
    for (int t = 0; t < 16; ++t) {
        float a = w0[(idx >> (2 * t)) & 3u], b = 1.0f - a;
        aa += a * a; ab += a * b; bb += b * b;
        xa.r += a * px[t].r; xa.g += a * px[t].g; xa.b += a * px[t].b;
        xb.r += b * px[t].r; xb.g += b * px[t].g; xb.b += b * px[t].b;
    }
    float det = aa * bb - ab * ab;
    if (std::fabs(det) > 1e-6f) {
        Rgb na{(bb * xa.r - ab * xb.r) / det, (bb * xa.g - ab * xb.g) / det, (bb * xa.b - ab * xb.b) / det};
        Rgb nb{(aa * xb.r - ab * xa.r) / det, (aa * xb.g - ab * xa.g) / det, (aa * xb.b - ab * xa.b) / det};
        uint16_t d0 = pack565(na), d1 = pack565(nb);
        if (d0 < d1) std::swap(d0, d1);
        if (d0 != d1) {
            uint32_t idx2;
            float err2 = bc1_fit(px, d0, d1, &idx2);
            if (err2 < err) {
                c0 = d0;
                c1 = d1;
                idx = idx2;
            }
        }
    }
    write_bc1(out, c0, c1, idx);
}

void encode_bc4_block(const uint8_t* v, uint8_t* out) {
    uint8_t hi = *std::max_element(v, v + 16), lo = *std::min_element(v, v + 16);
    out[0] = hi;
    out[1] = lo;
    uint64_t bits = 0;
    if (hi != lo) {
        float pal[8];
        pal[0] = hi;
        pal[1] = lo;
        for (int k = 1; k <= 6; ++k) pal[1 + k] = (float(7 - k) * hi + float(k) * lo) / 7.0f;
        for (int t = 0; t < 16; ++t) {
            int best = 0;
            float bd = std::fabs(float(v[t]) - pal[0]);
            for (int k = 1; k < 8; ++k) {
                float d = std::fabs(float(v[t]) - pal[k]);
                if (d < bd) {
                    bd = d;
                    best = k;
                }
            }
            bits |= uint64_t(best) << (3 * t);
        }
    }
    for (int k = 0; k < 6; ++k) out[2 + k] = uint8_t(bits >> (8 * k));
}

}  // namespace

bool texture_encode(uint32_t format, const uint8_t* rgba, uint32_t w, uint32_t h, uint8_t* out) {
    if (texture_bytes(format, w, h) == 0) return false;
    const bool bc1 = format == CENOTE_TEXTURE_BC1_SRGB || format == CENOTE_TEXTURE_BC1_UNORM;
    const bool bc7 = format == CENOTE_TEXTURE_BC7_SRGB || format == CENOTE_TEXTURE_BC7_UNORM;
    if (!bc1 && !bc7 && format != CENOTE_TEXTURE_BC4_UNORM && format != CENOTE_TEXTURE_BC5_UNORM) return false;
    const uint32_t bw = w / 4, bh = h / 4;
    const size_t block = (format == CENOTE_TEXTURE_BC5_UNORM || bc7) ? 16 : 8;
    auto rows = [&](uint32_t by0, uint32_t by1) {
        for (uint32_t by = by0; by < by1; ++by)
            for (uint32_t bx = 0; bx < bw; ++bx) {
                uint8_t* dst = out + block * (size_t(by) * bw + bx);
                Rgb px[16];
                uint8_t ch[2][16], raw[16][4];
                for (int t = 0; t < 16; ++t) {
                    const uint8_t* p = rgba + 4 * ((size_t(by) * 4 + t / 4) * w + bx * 4 + t % 4);
                    px[t] = {float(p[0]), float(p[1]), float(p[2])};
                    ch[0][t] = p[0];
                    ch[1][t] = p[1];
                    std::memcpy(raw[t], p, 4);
                }
                if (bc7) {
                    encode_bc7_block(raw, dst);
                } else if (bc1) {
                    encode_bc1_block(px, dst);
                } else {
                    encode_bc4_block(ch[0], dst);
                    if (format == CENOTE_TEXTURE_BC5_UNORM) encode_bc4_block(ch[1], dst + 8);
                }
            }
    };
    // Blocks are independent: split the block rows over the host's threads.
    const uint32_t threads = std::max(1u, std::min(std::thread::hardware_concurrency(), std::max(1u, bh / 16)));
    std::vector<std::thread> pool;
    for (uint32_t k = 0; k < threads; ++k)
        pool.emplace_back(rows, bh * k / threads, bh * (k + 1) / threads);
    for (auto& t : pool) t.join();
    return true;
}

bool texture_encode_float(uint32_t format, const float* rgba, uint32_t w, uint32_t h, uint8_t* out) {
    if (format != CENOTE_TEXTURE_BC6H_UF16 || texture_bytes(format, w, h) == 0) return false;
    const uint32_t bw = w / 4, bh = h / 4;
    auto rows = [&](uint32_t by0, uint32_t by1) {
        for (uint32_t by = by0; by < by1; ++by)
            for (uint32_t bx = 0; bx < bw; ++bx) {
                float px[16][4];
                for (int t = 0; t < 16; ++t)
                    std::memcpy(px[t], rgba + 4 * ((size_t(by) * 4 + t / 4) * w + bx * 4 + t % 4), 16);
                encode_bc6h_block(px, out + 16 * (size_t(by) * bw + bx));
            }
    };
    const uint32_t threads = std::max(1u, std::min(std::thread::hardware_concurrency(), std::max(1u, bh / 16)));
    std::vector<std::thread> pool;
    for (uint32_t k = 0; k < threads; ++k)
        pool.emplace_back(rows, bh * k / threads, bh * (k + 1) / threads);
    for (auto& t : pool) t.join();
    return true;
}

}  // namespace cn
