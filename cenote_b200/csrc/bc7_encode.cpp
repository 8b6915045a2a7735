// BC7 block encoder for texture prep: the reference compresses every 8-bit
// colour texture to BC7 before upload (crates/cenote/src/texture.rs:249-281,
// through an external encoder); this one is written for this library.
//
// Per 4x4 block of RGBA8 (bytes as stored, so an sRGB texture is encoded in
// its stored space, as the reference's encoder sees it):
//  * a block of one colour: mode 6 with the endpoint pair, p-bits and index
//    that reproduce the colour best, from a table of every value each
//    (p-bits, index) pair reaches (exact for most colours);
//  * otherwise mode 6 (one subset, RGBA with a p-bit per endpoint, 4-bit
//    indices) and, for opaque blocks, modes 1 (two subsets, 6-bit RGB and a
//    shared p-bit, 3-bit indices) and 3 (two subsets, 7-bit RGB and a p-bit
//    per endpoint, 2-bit indices) over the three two-subset partitions whose
//    subsets lie closest to a line in colour space; each subset's endpoints
//    are its principal-axis extremes, quantised under every p-bit choice,
//    then refitted twice by least squares from the chosen indices. The mode
//    with the lowest squared error wins.
// The block layout, weights and anchors are the format's (Khronos Data
// Format Specification, "BC7"; partitions and anchors in bc7_tables.h).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "bc7_tables.h"
#include "texture_prep.h"

namespace cn {
namespace {

constexpr int W2[4] = {0, 21, 43, 64};
constexpr int W3[8] = {0, 9, 18, 27, 37, 46, 55, 64};
constexpr int W4[16] = {0, 4, 9, 13, 17, 21, 26, 30, 34, 38, 43, 47, 51, 55, 60, 64};

const int* weights(int bits) { return bits == 2 ? W2 : (bits == 3 ? W3 : W4); }

inline int lerp8(int a, int b, int w) { return ((64 - w) * a + w * b + 32) >> 6; }

inline int expand(int v, int n) { return n >= 8 ? v : (v << (8 - n)) | (v >> (2 * n - 8)); }

struct Spec {
    int mode, ns, cb, ab;
    int pmode;  // 0: no p-bits, 1: one per endpoint, 2: one per subset
    int ib;
};
constexpr Spec MODE1{1, 2, 6, 0, 2, 3};
constexpr Spec MODE3{3, 2, 7, 0, 1, 2};
constexpr Spec MODE6{6, 1, 7, 7, 1, 4};
// Two-subset partitions encoded in full, best-ranked first (3, 6, 12 and all
// 64 give 46.90, 46.92, 46.93 and 46.94 dB on a 256x256 value-noise texture).
constexpr int TRY_PARTITIONS = 3;

// One subset's endpoints: stored codes, p-bits and the 8-bit values they
// expand to.
struct Ends {
    int code[2][4];
    int p[2];
    int q[2][4];
};

struct Subset {
    Ends e;
    float err;
};

void quantise(const float f[2][4], const Spec& m, int p0, int p1, Ends* out) {
    const int p[2] = {p0, p1};
    for (int k = 0; k < 2; ++k) {
        out->p[k] = p[k];
        for (int c = 0; c < 4; ++c) {
            const int bits = c < 3 ? m.cb : m.ab;
            if (bits == 0) {
                out->code[k][c] = 0;
                out->q[k][c] = 255;
                continue;
            }
            const bool hasp = m.pmode != 0;
            const int n = bits + (hasp ? 1 : 0), maxc = (1 << bits) - 1;
            const float target = std::clamp(f[k][c], 0.0f, 255.0f);
            const float scaled = target * float((1 << n) - 1) / 255.0f;
            const int guess = hasp ? int(std::lround((scaled - float(p[k])) * 0.5f)) : int(std::lround(scaled));
            int best = 0;
            float bd = 1e30f;
            for (int d = -1; d <= 1; ++d) {
                const int cc = std::clamp(guess + d, 0, maxc);
                const float diff = float(expand(hasp ? (cc << 1) | p[k] : cc, n)) - target;
                if (diff * diff < bd) {
                    bd = diff * diff;
                    best = cc;
                }
            }
            out->code[k][c] = best;
            out->q[k][c] = expand(hasp ? (best << 1) | p[k] : best, n);
        }
    }
}

// Nearest palette entry per texel of the subset; squared error over `nc`
// channels (3: alpha is 255 in the modes without it).
float assign(const uint8_t px[16][4], const int* ts, int n, const Ends& e, int ib, int nc, uint8_t* idx) {
    const int* w = weights(ib);
    const int np = 1 << ib;
    int pal[16][4];
    for (int k = 0; k < np; ++k)
        for (int c = 0; c < 4; ++c) pal[k][c] = lerp8(e.q[0][c], e.q[1][c], w[k]);
    float err = 0.0f;
    for (int j = 0; j < n; ++j) {
        const int t = ts[j];
        int best = 0, bd = INT_MAX;
        for (int k = 0; k < np; ++k) {
            int d = 0;
            for (int c = 0; c < nc; ++c) {
                const int x = pal[k][c] - px[t][c];
                d += x * x;
            }
            if (d < bd) {
                bd = d;
                best = k;
            }
        }
        idx[t] = uint8_t(best);
        err += float(bd);
    }
    return err;
}

// Extremes of the subset's texels along their principal axis.
void axis_ends(const uint8_t px[16][4], const int* ts, int n, int nc, float f[2][4]) {
    float mean[4] = {0, 0, 0, 0};
    for (int j = 0; j < n; ++j)
        for (int c = 0; c < nc; ++c) mean[c] += float(px[ts[j]][c]) / float(n);
    float cov[4][4] = {};
    for (int j = 0; j < n; ++j) {
        float d[4] = {0, 0, 0, 0};
        for (int c = 0; c < nc; ++c) d[c] = float(px[ts[j]][c]) - mean[c];
        for (int a = 0; a < nc; ++a)
            for (int b = 0; b < nc; ++b) cov[a][b] += d[a] * d[b];
    }
    // Power iteration from the column of the largest variance (a start that
    // cannot be orthogonal to the principal axis unless the block is flat).
    int top = 0;
    for (int c = 1; c < nc; ++c)
        if (cov[c][c] > cov[top][top]) top = c;
    float ax[4] = {0, 0, 0, 0};
    for (int c = 0; c < nc; ++c) ax[c] = cov[c][top];
    for (int it = 0; it < 8; ++it) {
        float nx[4] = {0, 0, 0, 0}, mx = 0.0f;
        for (int a = 0; a < nc; ++a) {
            for (int b = 0; b < nc; ++b) nx[a] += cov[a][b] * ax[b];
            mx = std::max(mx, std::fabs(nx[a]));
        }
        if (mx <= 0.0f) break;
        for (int c = 0; c < nc; ++c) ax[c] = nx[c] / mx;
    }
    float n2 = 0.0f;
    for (int c = 0; c < nc; ++c) n2 += ax[c] * ax[c];
    float lo = 0.0f, hi = 0.0f;
    if (n2 > 0.0f) {
        lo = 1e30f;
        hi = -1e30f;
        for (int j = 0; j < n; ++j) {
            float s = 0.0f;
            for (int c = 0; c < nc; ++c) s += (float(px[ts[j]][c]) - mean[c]) * ax[c];
            lo = std::min(lo, s);
            hi = std::max(hi, s);
        }
    } else {
        n2 = 1.0f;
    }
    for (int c = 0; c < 4; ++c) {
        f[0][c] = c < nc ? mean[c] + ax[c] * lo / n2 : 255.0f;
        f[1][c] = c < nc ? mean[c] + ax[c] * hi / n2 : 255.0f;
    }
}

// Least-squares endpoints for the subset given its indices; false when the
// indices do not determine them (all equal).
bool refit(const uint8_t px[16][4], const int* ts, int n, int nc, const uint8_t* idx, int ib, float f[2][4]) {
    const int* w = weights(ib);
    float aa = 0, ab = 0, bb = 0, xa[4] = {0, 0, 0, 0}, xb[4] = {0, 0, 0, 0};
    for (int j = 0; j < n; ++j) {
        const float b = float(w[idx[ts[j]]]) / 64.0f, a = 1.0f - b;
        aa += a * a;
        ab += a * b;
        bb += b * b;
        for (int c = 0; c < nc; ++c) {
            xa[c] += a * float(px[ts[j]][c]);
            xb[c] += b * float(px[ts[j]][c]);
        }
    }
    const float det = aa * bb - ab * ab;
    if (std::fabs(det) < 1e-6f) return false;
    for (int c = 0; c < 4; ++c) {
        f[0][c] = c < nc ? (bb * xa[c] - ab * xb[c]) / det : 255.0f;
        f[1][c] = c < nc ? (aa * xb[c] - ab * xa[c]) / det : 255.0f;
    }
    return true;
}

Subset fit_subset(const uint8_t px[16][4], const int* ts, int n, const Spec& m, int nc, uint8_t* idx) {
    int pb[4][2] = {{0, 0}, {1, 1}, {0, 1}, {1, 0}};
    const int choices = m.pmode == 0 ? 1 : (m.pmode == 2 ? 2 : 4);
    Subset best{};
    best.err = 1e30f;
    uint8_t tmp[16];
    float f[2][4];
    axis_ends(px, ts, n, nc, f);
    for (int pass = 0; pass < 3; ++pass) {
        for (int k = 0; k < choices; ++k) {
            Ends e;
            quantise(f, m, pb[k][0], pb[k][1], &e);
            const float err = assign(px, ts, n, e, m.ib, nc, tmp);
            if (err < best.err) {
                best.err = err;
                best.e = e;
                for (int j = 0; j < n; ++j) idx[ts[j]] = tmp[ts[j]];
            }
        }
        if (pass < 2 && !refit(px, ts, n, nc, idx, m.ib, f)) break;
    }
    return best;
}

struct Writer {
    uint8_t* out;
    int pos = 0;
    void put(uint32_t v, int n) {
        for (int i = 0; i < n; ++i, ++pos)
            if ((v >> i) & 1u) out[pos >> 3] = uint8_t(out[pos >> 3] | (1u << (pos & 7)));
    }
};

// Writes a one- or two-subset block of mode `m`; the anchors' indices are
// made to fit (top bit clear) by swapping that subset's endpoints.
void write_block(const Spec& m, int part, Ends* ends, uint8_t* idx, uint8_t* out) {
    const int np = 1 << m.ib;
    for (int s = 0; s < m.ns; ++s) {
        const int anchor = s == 0 ? 0 : bc7::ANCHOR2[part];
        if (idx[anchor] >= np / 2) {
            Ends& e = ends[s];
            for (int c = 0; c < 4; ++c) {
                std::swap(e.code[0][c], e.code[1][c]);
                std::swap(e.q[0][c], e.q[1][c]);
            }
            std::swap(e.p[0], e.p[1]);
            for (int t = 0; t < 16; ++t)
                if ((m.ns == 1 ? 0 : bc7::PARTITION2[part][t]) == s) idx[t] = uint8_t(np - 1 - idx[t]);
        }
    }
    std::memset(out, 0, 16);
    Writer w{out};
    w.put(1u << m.mode, m.mode + 1);
    if (m.ns == 2) w.put(uint32_t(part), 6);
    for (int c = 0; c < 3; ++c)
        for (int s = 0; s < m.ns; ++s)
            for (int k = 0; k < 2; ++k) w.put(uint32_t(ends[s].code[k][c]), m.cb);
    if (m.ab)
        for (int s = 0; s < m.ns; ++s)
            for (int k = 0; k < 2; ++k) w.put(uint32_t(ends[s].code[k][3]), m.ab);
    for (int s = 0; s < m.ns; ++s) {
        if (m.pmode == 1) {
            w.put(uint32_t(ends[s].p[0]), 1);
            w.put(uint32_t(ends[s].p[1]), 1);
        } else if (m.pmode == 2) {
            w.put(uint32_t(ends[s].p[0]), 1);
        }
    }
    for (int t = 0; t < 16; ++t) {
        const bool anchor = t == 0 || (m.ns == 2 && t == bc7::ANCHOR2[part]);
        w.put(idx[t], m.ib - (anchor ? 1 : 0));
    }
}

// Mode 6 single-colour table: for p-bits (p0, p1), index i and value v, the
// 7-bit codes (c0, c1) whose interpolation lands nearest v, and how far.
struct SolidEntry {
    uint8_t c0, c1, err;
};
SolidEntry g_solid[2][2][16][256];
std::once_flag g_solid_once;

void build_solid() {
    for (int p0 = 0; p0 < 2; ++p0)
        for (int p1 = 0; p1 < 2; ++p1)
            for (int i = 0; i < 16; ++i) {
                SolidEntry* row = g_solid[p0][p1][i];
                for (int v = 0; v < 256; ++v) row[v].err = 255;
                for (int c0 = 0; c0 < 128; ++c0)
                    for (int c1 = 0; c1 < 128; ++c1) {
                        const int v = lerp8((c0 << 1) | p0, (c1 << 1) | p1, W4[i]);
                        row[v] = {uint8_t(c0), uint8_t(c1), 0};
                    }
                // Values no pair reaches take the nearest reached one.
                for (int v = 0; v < 256; ++v) {
                    if (row[v].err == 0) continue;
                    for (int d = 1; d < 256; ++d) {
                        if (v - d >= 0 && g_solid[p0][p1][i][v - d].err == 0) {
                            row[v] = {row[v - d].c0, row[v - d].c1, uint8_t(d)};
                            break;
                        }
                        if (v + d < 256 && row[v + d].err == 0) {
                            row[v] = {row[v + d].c0, row[v + d].c1, uint8_t(d)};
                            break;
                        }
                    }
                }
            }
}

float encode_solid(const uint8_t* rgba, uint8_t* out) {
    std::call_once(g_solid_once, build_solid);
    int best = INT_MAX, bp0 = 0, bp1 = 0, bi = 0;
    for (int p0 = 0; p0 < 2; ++p0)
        for (int p1 = 0; p1 < 2; ++p1)
            for (int i = 0; i < 16; ++i) {
                int err = 0;
                for (int c = 0; c < 4; ++c) {
                    const int d = g_solid[p0][p1][i][rgba[c]].err;
                    err += d * d;
                }
                if (err < best) {
                    best = err;
                    bp0 = p0;
                    bp1 = p1;
                    bi = i;
                }
            }
    Ends e;
    e.p[0] = bp0;
    e.p[1] = bp1;
    for (int c = 0; c < 4; ++c) {
        const SolidEntry& s = g_solid[bp0][bp1][bi][rgba[c]];
        e.code[0][c] = s.c0;
        e.code[1][c] = s.c1;
        e.q[0][c] = (s.c0 << 1) | bp0;
        e.q[1][c] = (s.c1 << 1) | bp1;
    }
    uint8_t idx[16];
    std::memset(idx, bi, 16);
    write_block(MODE6, 0, &e, idx, out);
    return float(best) * 16.0f;
}

}  // namespace

void encode_bc7_block(const uint8_t px[16][4], uint8_t out[16]) {
    bool solid = true, opaque = true;
    for (int t = 0; t < 16; ++t) {
        solid = solid && std::memcmp(px[t], px[0], 4) == 0;
        opaque = opaque && px[t][3] == 255;
    }
    float best = 1e30f;
    if (solid) {
        best = encode_solid(px[0], out);
        if (best == 0.0f) return;
    }
    uint8_t cand[16], idx[16];
    int all[16];
    for (int t = 0; t < 16; ++t) all[t] = t;
    {
        Ends e[1];
        Subset s = fit_subset(px, all, 16, MODE6, 4, idx);
        e[0] = s.e;
        if (s.err < best) {
            best = s.err;
            write_block(MODE6, 0, e, idx, out);
        }
    }
    if (!opaque || best == 0.0f) return;
    // Two-subset partitions ranked by how far each subset's texels lie from
    // their principal axis (the error a line fit leaves, before quantisation).
    float score[64];
    for (int part = 0; part < 64; ++part) {
        score[part] = 0.0f;
        for (int s = 0; s < 2; ++s) {
            int ts[16], n = 0;
            for (int t = 0; t < 16; ++t)
                if (bc7::PARTITION2[part][t] == s) ts[n++] = t;
            float f[2][4];
            axis_ends(px, ts, n, 3, f);
            float dir[3], d2 = 0.0f;
            for (int c = 0; c < 3; ++c) {
                dir[c] = f[1][c] - f[0][c];
                d2 += dir[c] * dir[c];
            }
            for (int j = 0; j < n; ++j) {
                float v[3], along = 0.0f, len2 = 0.0f;
                for (int c = 0; c < 3; ++c) {
                    v[c] = float(px[ts[j]][c]) - f[0][c];
                    along += v[c] * dir[c];
                    len2 += v[c] * v[c];
                }
                score[part] += d2 > 0.0f ? len2 - along * along / d2 : len2;
            }
        }
    }
    int order[64];
    for (int k = 0; k < 64; ++k) order[k] = k;
    std::partial_sort(order, order + TRY_PARTITIONS, order + 64, [&](int a, int b) { return score[a] < score[b]; });
    for (int r = 0; r < TRY_PARTITIONS; ++r) {
        const int part = order[r];
        int ts[2][16], n[2] = {0, 0};
        for (int t = 0; t < 16; ++t) {
            const int s = bc7::PARTITION2[part][t];
            ts[s][n[s]++] = t;
        }
        for (const Spec* m : {&MODE1, &MODE3}) {
            Ends e[2];
            float err = 0.0f;
            for (int s = 0; s < 2; ++s) {
                Subset fit = fit_subset(px, ts[s], n[s], *m, 3, idx);
                e[s] = fit.e;
                err += fit.err;
            }
            if (err < best) {
                best = err;
                write_block(*m, part, e, idx, cand);
                std::memcpy(out, cand, 16);
            }
        }
    }
}

}  // namespace cn
