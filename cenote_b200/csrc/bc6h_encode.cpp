// BC6H (unsigned) block encoder for texture prep: the reference encodes
// float colour textures as BC6H_UFLOAT (crates/cenote/src/texture.rs:283-306,
// through an external encoder; negative radiance clamps to zero); this one
// is written for this library.
//
// Per 4x4 block of RGB floats: each texel becomes its FP16 bit pattern
// (negatives and NaN to 0, above the FP16 range to the largest finite), and
// the block is fitted in that integer domain, where BC6H interpolates (a
// logarithmic scale in the value). The one-region modes are tried: 11
// (10-bit endpoints), 12, 13 and 14 (an 11-, 12- or 16-bit base endpoint and
// a 9-, 8- or 4-bit signed delta to the other); endpoints are the block's
// principal-axis extremes, each quantised to the code whose decoded FP16
// pattern lands nearest, indices the nearest of the 16 palette entries, then
// one least-squares refit; the mode with the lowest squared error (in FP16
// bit units) wins. Two-region modes are not used.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "texture_prep.h"

namespace cn {
namespace {

constexpr int W4[16] = {0, 4, 9, 13, 17, 21, 26, 30, 34, 38, 43, 47, 51, 55, 60, 64};

// FP16 bit pattern of a float, round to nearest even; the unsigned format's
// domain: negatives and NaN give 0, values past the largest finite FP16 give
// it (0x7BFF).
int half_bits(float v) {
    if (!(v > 0.0f)) return 0;
    if (v >= 65504.0f) return 0x7BFF;
    int e;
    const float m = std::frexp(v, &e);  // v = m 2^e, m in [0.5, 1)
    if (e < -13) {                      // subnormal FP16: units of 2^-24
        const float q = std::nearbyint(std::ldexp(v, 24));
        return int(q);
    }
    const float q = std::nearbyint(std::ldexp(m, 11));  // 11 significant bits
    int mant = int(q), exp = e - 1;
    if (mant == 2048) {
        mant = 1024;
        ++exp;
    }
    const int bits = ((exp + 15) << 10) | (mant - 1024);
    return std::min(bits, 0x7BFF);
}

// The FP16 pattern an unsigned endpoint code of `prec` bits decodes to when
// a texel takes it whole (unquantise, then the final 31/64 scale).
int decoded(int q, int prec) {
    int u;
    if (prec >= 15) u = q;
    else if (q == 0) u = 0;
    else if (q == (1 << prec) - 1) u = 0xFFFF;
    else u = ((q << 16) + 0x8000) >> prec;
    return (u * 31) >> 6;
}

int unquantised(int q, int prec) {
    if (prec >= 15) return q;
    if (q == 0) return 0;
    if (q == (1 << prec) - 1) return 0xFFFF;
    return ((q << 16) + 0x8000) >> prec;
}

int quantise(float target, int prec) {
    const int maxq = (1 << prec) - 1;
    const float t = std::clamp(target, 0.0f, float(0x7BFF));
    const int guess = int(std::lround(t * 64.0f / 31.0f / float(1 << (16 - std::min(prec, 16)))));
    int best = 0, bd = INT_MAX;
    for (int d = -2; d <= 2; ++d) {
        const int q = std::clamp(guess + d, 0, maxq);
        const int diff = decoded(q, prec) - int(std::lround(t));
        if (std::abs(diff) < bd) {
            bd = std::abs(diff);
            best = q;
        }
    }
    return best;
}

struct Mode {
    int value;  // five mode bits, LSB first in the stream
    int prec, delta;  // endpoint bits; delta bits (0: both endpoints stored whole)
};
constexpr Mode MODES[4] = {{3, 10, 0}, {7, 11, 9}, {11, 12, 8}, {15, 16, 4}};

struct Writer {
    uint8_t* out;
    int pos = 0;
    void put(uint32_t v, int n) {
        for (int i = 0; i < n; ++i, ++pos)
            if ((v >> i) & 1u) out[pos >> 3] = uint8_t(out[pos >> 3] | (1u << (pos & 7)));
    }
    // Bits lo..hi of v, high bit first (the stored order of the transformed
    // modes' top base-endpoint bits).
    void put_reversed(uint32_t v, int lo, int hi) {
        for (int b = hi; b >= lo; --b) put((v >> b) & 1u, 1);
    }
};

// Palette error of the block for endpoint codes q[2][3]; fills indices.
int64_t assign(const int h[16][3], const int q[2][3], int prec, uint8_t idx[16]) {
    int pal[16][3];
    for (int c = 0; c < 3; ++c) {
        const int a = unquantised(q[0][c], prec), b = unquantised(q[1][c], prec);
        for (int k = 0; k < 16; ++k) pal[k][c] = ((((64 - W4[k]) * a + W4[k] * b + 32) >> 6) * 31) >> 6;
    }
    int64_t err = 0;
    for (int t = 0; t < 16; ++t) {
        int64_t bd = INT64_MAX;
        int best = 0;
        for (int k = 0; k < 16; ++k) {
            int64_t d = 0;
            for (int c = 0; c < 3; ++c) {
                const int64_t x = pal[k][c] - h[t][c];
                d += x * x;
            }
            if (d < bd) {
                bd = d;
                best = k;
            }
        }
        idx[t] = uint8_t(best);
        err += bd;
    }
    return err;
}

void principal_ends(const int h[16][3], float f[2][3]) {
    float mean[3] = {0, 0, 0};
    for (int t = 0; t < 16; ++t)
        for (int c = 0; c < 3; ++c) mean[c] += float(h[t][c]) / 16.0f;
    float cov[3][3] = {};
    for (int t = 0; t < 16; ++t)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) cov[a][b] += (float(h[t][a]) - mean[a]) * (float(h[t][b]) - mean[b]);
    int top = 0;
    for (int c = 1; c < 3; ++c)
        if (cov[c][c] > cov[top][top]) top = c;
    float ax[3] = {cov[0][top], cov[1][top], cov[2][top]};
    for (int it = 0; it < 8; ++it) {
        float nx[3] = {0, 0, 0}, mx = 0.0f;
        for (int a = 0; a < 3; ++a) {
            for (int b = 0; b < 3; ++b) nx[a] += cov[a][b] * ax[b];
            mx = std::max(mx, std::fabs(nx[a]));
        }
        if (mx <= 0.0f) break;
        for (int c = 0; c < 3; ++c) ax[c] = nx[c] / mx;
    }
    const float n2 = ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2];
    float lo = 0.0f, hi = 0.0f;
    if (n2 > 0.0f) {
        lo = 1e30f;
        hi = -1e30f;
        for (int t = 0; t < 16; ++t) {
            float s = 0.0f;
            for (int c = 0; c < 3; ++c) s += (float(h[t][c]) - mean[c]) * ax[c];
            lo = std::min(lo, s);
            hi = std::max(hi, s);
        }
    }
    for (int c = 0; c < 3; ++c) {
        f[0][c] = mean[c] + (n2 > 0.0f ? ax[c] * lo / n2 : 0.0f);
        f[1][c] = mean[c] + (n2 > 0.0f ? ax[c] * hi / n2 : 0.0f);
    }
}

// Least-squares endpoints (FP16-pattern units) from the indices; false when
// every texel took the same weight.
bool refit(const int h[16][3], const uint8_t idx[16], float f[2][3]) {
    float aa = 0, ab = 0, bb = 0, xa[3] = {0, 0, 0}, xb[3] = {0, 0, 0};
    for (int t = 0; t < 16; ++t) {
        const float b = float(W4[idx[t]]) / 64.0f, a = 1.0f - b;
        aa += a * a;
        ab += a * b;
        bb += b * b;
        for (int c = 0; c < 3; ++c) {
            xa[c] += a * float(h[t][c]);
            xb[c] += b * float(h[t][c]);
        }
    }
    const float det = aa * bb - ab * ab;
    if (std::fabs(det) < 1e-6f) return false;
    for (int c = 0; c < 3; ++c) {
        f[0][c] = (bb * xa[c] - ab * xb[c]) / det;
        f[1][c] = (aa * xb[c] - ab * xa[c]) / det;
    }
    return true;
}

// Endpoint codes of `m` for float endpoints f; false when the second
// endpoint is out of the delta's reach.
bool codes(const float f[2][3], const Mode& m, int q[2][3]) {
    for (int c = 0; c < 3; ++c) {
        q[0][c] = quantise(f[0][c], m.prec);
        q[1][c] = quantise(f[1][c], m.prec);
        if (m.delta) {
            const int lim = 1 << (m.delta - 1);
            q[1][c] = std::clamp(q[1][c], std::max(0, q[0][c] - lim), std::min((1 << m.prec) - 1, q[0][c] + lim - 1));
        }
    }
    return true;
}

void write_block(const Mode& m, int q[2][3], uint8_t idx[16], uint8_t out[16]) {
    if (idx[0] >= 8) {  // texel 0 anchors with three index bits
        for (int c = 0; c < 3; ++c) std::swap(q[0][c], q[1][c]);
        for (int t = 0; t < 16; ++t) idx[t] = uint8_t(15 - idx[t]);
    }
    std::memset(out, 0, 16);
    Writer w{out};
    w.put(uint32_t(m.value), 5);
    for (int c = 0; c < 3; ++c) w.put(uint32_t(q[0][c]) & 1023u, 10);
    if (m.delta == 0) {
        for (int c = 0; c < 3; ++c) w.put(uint32_t(q[1][c]), 10);
    } else {
        for (int c = 0; c < 3; ++c) {
            const uint32_t d = uint32_t(q[1][c] - q[0][c]) & ((1u << m.delta) - 1u);
            w.put(d, m.delta);
            const uint32_t base = uint32_t(q[0][c]);
            if (m.prec == 11) w.put((base >> 10) & 1u, 1);
            else w.put_reversed(base, 10, m.prec - 1);
        }
    }
    for (int t = 0; t < 16; ++t) w.put(idx[t], t == 0 ? 3 : 4);
}

}  // namespace

void encode_bc6h_block(const float px[16][4], uint8_t out[16]) {
    int h[16][3];
    for (int t = 0; t < 16; ++t)
        for (int c = 0; c < 3; ++c) h[t][c] = half_bits(px[t][c]);
    int64_t best = INT64_MAX;
    for (const Mode& m : MODES) {
        float f[2][3];
        principal_ends(h, f);
        for (int pass = 0; pass < 2; ++pass) {
            int q[2][3];
            uint8_t idx[16];
            codes(f, m, q);
            const int64_t err = assign(h, q, m.prec, idx);
            if (err < best) {
                best = err;
                write_block(m, q, idx, out);
            }
            if (pass == 0 && !refit(h, idx, f)) break;
        }
    }
}

}  // namespace cn
