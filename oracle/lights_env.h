// Test infrastructure (CPU oracle): the light list's alias table, the
// environment's sampling tables and their GPU-side samplers, restated from
//   crates/cenote/src/lights.rs:123-275        (host alias build, f64 Vose)
//   crates/cenote/shaders/lights.slang:93-160  (sampleLights)
//   crates/cenote/src/environment.rs:130-218   (host CDF/pdf tables, f64)
//   crates/cenote/shaders/environment.slang    (sampleCdf, sample, pdf, radiance)
//   crates/cenote/src/scene/mod.rs:665-671     (select_probability)
//   crates/cenote/src/color.rs:13-31           (Rec.709 → ACEScg, AP1 luminance)
#pragma once
#include <cstdint>
#include <cstring>
#include <vector>
#include "textures.h"
#include "vec.h"

namespace oracle {

using V3f = V3<float>;
constexpr uint32_t LIGHT_NONE = 0xffffffffu;
constexpr uint32_t KIND_TRIANGLE = 0, KIND_DISTANT = 1, KIND_POINT = 2;
constexpr uint32_t LIGHT_SAMPLING_MIS = 0, LIGHT_SAMPLING_BSDF = 1, LIGHT_SAMPLING_NEE = 2;

// color.rs:367-369 — an f32 dot product, evaluated left to right.
inline float luminance(V3f c) { return c.x * 0.2722287f + c.y * 0.6740818f + c.z * 0.0536895f; }

// color.rs:351-361 — column-major Mat3 times a vector.
inline V3f acescg_from_rec709(V3f c) {
    return {0.6130974f * c.x + 0.33952314f * c.y + 0.04737945f * c.z,
            0.07019373f * c.x + 0.9163539f * c.y + 0.013452399f * c.z,
            0.020615594f * c.x + 0.10956978f * c.y + 0.86981466f * c.z};
}

// The 80-byte light record, lights.rs:79-115 / lights.slang:49-65.
struct LightRecord {
    float anchor[3];
    float pdf;
    float edge1[3];
    float alias_threshold;
    float edge2[3];
    uint32_t alias_index;
    float emission[3];
    uint32_t instance;
    uint32_t kind;
    uint32_t primitive;
    uint32_t pad0[2];
};
static_assert(sizeof(LightRecord) == 80, "light record is 80 bytes");

struct TriangleLight {
    V3f corners[3];
    V3f emission;
    uint32_t instance, primitive;
};
struct DeltaLight {
    uint32_t kind;  // KIND_DISTANT (anchor = travel direction) or KIND_POINT (anchor = position)
    V3f anchor;
    V3f emission;   // irradiance / intensity
};

inline V3f rd3(const float* f) { return {f[0], f[1], f[2]}; }
inline void wr3(float* f, V3f v) { f[0] = v.x; f[1] = v.y; f[2] = v.z; }

inline double triangle_area(const LightRecord& r) {  // lights.rs:135-137
    return double(length(cross(rd3(r.edge1), rd3(r.edge2)))) / 2.0;
}
inline double light_power(const LightRecord& r) {  // lights.rs:123-130
    double luma = double(luminance(rd3(r.emission)));
    if (r.kind == KIND_TRIANGLE) return 3.141592653589793 * luma * triangle_area(r);
    if (r.kind == KIND_DISTANT) return luma;
    return 4.0 * 3.141592653589793 * luma;
}

inline std::vector<LightRecord> raw_light_records(const std::vector<TriangleLight>& tris,
                                                  const std::vector<DeltaLight>& deltas) {  // lights.rs:236-275
    std::vector<LightRecord> out;
    auto rec = [](uint32_t kind, V3f anchor, V3f e1, V3f e2, V3f em, uint32_t inst, uint32_t prim) {
        LightRecord r;
        std::memset(&r, 0, sizeof r);
        wr3(r.anchor, anchor);
        r.pdf = 0.0f;
        wr3(r.edge1, e1);
        r.alias_threshold = 1.0f;
        wr3(r.edge2, e2);
        r.alias_index = 0;
        wr3(r.emission, em);
        r.instance = inst;
        r.kind = kind;
        r.primitive = prim;
        return r;
    };
    for (const auto& t : tris)
        out.push_back(rec(KIND_TRIANGLE, t.corners[0], t.corners[1] - t.corners[0],
                          t.corners[2] - t.corners[0], t.emission, t.instance, t.primitive));
    for (const auto& d : deltas)
        out.push_back(rec(d.kind, d.anchor, V3f(0.0f), V3f(0.0f), d.emission, LIGHT_NONE, 0));
    return out;
}

inline double total_light_power(const std::vector<TriangleLight>& tris, const std::vector<DeltaLight>& deltas) {
    double s = 0.0;  // lights.rs:229-231 — a sequential f64 sum
    for (const auto& r : raw_light_records(tris, deltas)) s += light_power(r);
    return s;
}

// lights.rs:175-224: power-proportional Walker/Vose alias table in f64 with
// the reference's stack discipline (stable partition, pop from the back).
inline std::vector<LightRecord> build_lights(const std::vector<TriangleLight>& tris,
                                             const std::vector<DeltaLight>& deltas) {
    std::vector<LightRecord> records = raw_light_records(tris, deltas);
    std::vector<double> powers;
    for (const auto& r : records) powers.push_back(light_power(r));
    double total = 0.0;
    for (double p : powers) total += p;
    if (total <= 0.0) return records;
    for (size_t i = 0; i < records.size(); ++i) {
        double selection = powers[i] / total;
        if (records[i].kind == KIND_TRIANGLE) {
            double area = triangle_area(records[i]);
            records[i].pdf = area > 0.0 ? float(selection / area) : 0.0f;
        } else {
            records[i].pdf = float(selection);
        }
    }
    double n = double(powers.size());
    std::vector<double> share;
    for (double p : powers) share.push_back(p * n / total);
    std::vector<size_t> small, large;
    for (size_t i = 0; i < share.size(); ++i) (share[i] < 1.0 ? small : large).push_back(i);
    while (!small.empty() && !large.empty()) {
        size_t poor = small.back();
        small.pop_back();
        size_t rich = large.back();
        large.pop_back();
        records[poor].alias_threshold = float(share[poor]);
        records[poor].alias_index = uint32_t(rich);
        share[rich] -= 1.0 - share[poor];
        (share[rich] < 1.0 ? small : large).push_back(rich);
    }
    return records;
}
// Note: Rust's `while let (Some(poor), Some(rich)) = (small.pop(), large.pop())`
// pops BOTH before testing, so when `large` runs dry first, one `small` entry
// is popped and dropped (it keeps threshold 1). The loop above pops only when
// both are non-empty, which leaves that entry untouched too: identical output.

inline float select_probability(double env_power, double light_power) {  // scene/mod.rs:665-671
    if (light_power == 0.0) return env_power > 0.0 ? 1.0f : 0.0f;
    return float(env_power / (env_power + light_power));
}

struct LightConnection {  // lights.slang:70-87
    V3f direction;
    float tmax;
    V3f radiance;
    float pdf;
    bool delta;
    uint32_t instance, primitive;
    float bary_x, bary_y;
};

inline LightConnection sample_lights(const LightRecord* lights, uint32_t count, float u, float upx,
                                     float upy, V3f from) {  // lights.slang:93-160
    float scaled = u * float(count);
    uint32_t slot = std::min(uint32_t(scaled), count - 1);
    const LightRecord* light = &lights[slot];
    if (scaled - float(slot) >= light->alias_threshold) light = &lights[light->alias_index];
    LightConnection c;
    c.pdf = 0.0f;
    c.direction = V3f(0.0f);
    c.tmax = 1e30f;
    c.radiance = rd3(light->emission);
    c.delta = light->kind != KIND_TRIANGLE;
    c.instance = light->instance;
    c.primitive = light->primitive;
    c.bary_x = c.bary_y = 0.0f;
    if (light->kind == KIND_TRIANGLE) {
        float su = std::sqrt(upx);
        c.bary_x = 1.0f - su;
        c.bary_y = upy * su;
        V3f position = rd3(light->anchor) + c.bary_x * rd3(light->edge1) + c.bary_y * rd3(light->edge2);
        V3f delta = position - from;
        float r2 = dot(delta, delta);
        V3f normal = normalize(cross(rd3(light->edge1), rd3(light->edge2)));
        V3f direction = delta * (1.0f / std::sqrt(r2));
        float cos_light = -dot(normal, direction);
        if (r2 > 0.0f && cos_light > 0.0f && light->pdf > 0.0f) {
            c.direction = direction;
            c.pdf = light->pdf * r2 / cos_light;
            c.tmax = std::sqrt(r2) * 1.001f;
        }
    } else if (light->kind == KIND_DISTANT) {
        c.direction = -rd3(light->anchor);
        c.pdf = light->pdf;
    } else {
        V3f delta = rd3(light->anchor) - from;
        float r2 = dot(delta, delta);
        if (r2 > 0.0f && light->pdf > 0.0f) {
            float r = std::sqrt(r2);
            c.direction = delta / r;
            c.radiance = rd3(light->emission) / r2;
            c.pdf = light->pdf;
            c.tmax = r;
        }
    }
    return c;
}

// ---- environment ----------------------------------------------------------

struct EnvTables {
    uint32_t width = 1, height = 1;
    std::vector<float> texels;       // RGBA, row-major, row 0 = +Y
    std::vector<float> marginal;     // height + 1
    std::vector<float> conditional;  // height × (width + 1)
    std::vector<float> pdfs;         // height × width
    double power = 0.0;
};

inline void build_env_tables(EnvTables& e) {  // environment.rs:130-218
    const size_t w = e.width, h = e.height;
    const double PI = 3.141592653589793;
    std::vector<double> lum(w * h);
    for (size_t i = 0; i < w * h; ++i)
        lum[i] = double(luminance(V3f(e.texels[4 * i], e.texels[4 * i + 1], e.texels[4 * i + 2])));
    std::vector<double> weight(w * h, 0.0);
    for (size_t row = 0; row < h; ++row) {
        double sin_theta = std::sin((double(row) + 0.5) / double(h) * PI);
        for (size_t col = 0; col < w; ++col) {
            double peak = 0.0;
            for (int dr = -1; dr <= 1; ++dr) {
                long rr = long(row) + dr;
                size_t r = rr < 0 ? 0 : std::min(size_t(rr), h - 1);
                for (int dc = -1; dc <= 1; ++dc) {
                    long cc = ((long(col) + dc) % long(w) + long(w)) % long(w);
                    peak = std::max(peak, lum[r * w + size_t(cc)]);
                }
            }
            weight[row * w + col] = peak * sin_theta;
        }
    }
    double total = 0.0;
    for (double v : weight) total += v;
    e.marginal.assign(h + 1, 0.0f);
    double running = 0.0;
    for (size_t row = 0; row < h; ++row) {
        double rs = 0.0;
        for (size_t col = 0; col < w; ++col) rs += weight[row * w + col];
        running += rs;
        e.marginal[row + 1] = total > 0.0 ? float(running / total) : 0.0f;
    }
    e.marginal[h] = 1.0f;
    e.conditional.assign(h * (w + 1), 0.0f);
    for (size_t row = 0; row < h; ++row) {
        double rs = 0.0;
        for (size_t col = 0; col < w; ++col) rs += weight[row * w + col];
        float* cdf = &e.conditional[row * (w + 1)];
        double run = 0.0;
        for (size_t col = 0; col < w; ++col) {
            run += weight[row * w + col];
            cdf[col + 1] = rs > 0.0 ? float(run / rs) : 0.0f;
        }
        cdf[w] = 1.0f;
    }
    double scale = total > 0.0 ? double(w * h) / total : 0.0;
    e.pdfs.resize(w * h);
    for (size_t i = 0; i < w * h; ++i) e.pdfs[i] = float(weight[i] * scale);
    double power = 0.0;
    for (size_t row = 0; row < h; ++row) {
        double theta0 = double(row) / double(h) * PI;
        double theta1 = double(row + 1) / double(h) * PI;
        double solid = 2.0 * PI / double(w) * (std::cos(theta0) - std::cos(theta1));
        double ls = 0.0;
        for (size_t col = 0; col < w; ++col) ls += lum[row * w + col];
        power += solid * ls;
    }
    e.power = power;
}

constexpr float PI_F = 3.14159265358979323846f;

struct CdfSlot {
    uint32_t index;
    float position;
};
inline CdfSlot sample_cdf(const float* cdf, uint32_t count, float u) {  // environment.slang:41-58
    uint32_t lo = 0, hi = count;
    while (lo + 1 < hi) {
        uint32_t mid = (lo + hi) / 2;
        if (cdf[mid] <= u) lo = mid;
        else hi = mid;
    }
    float width = cdf[lo + 1] - cdf[lo];
    float frac = width > 0.0f ? (u - cdf[lo]) / width : 0.0f;
    return {lo, (float(lo) + frac) / float(count)};
}

inline void uv_from_direction(V3f d, float* u, float* v) {  // environment.slang:74-78
    *u = 0.5f + std::atan2(d.x, -d.z) / (2.0f * PI_F);
    *v = std::acos(clampv(d.y, -1.0f, 1.0f)) / PI_F;
}
inline V3f direction_from_uv(float u, float v) {  // environment.slang:80-85
    float phi = 2.0f * PI_F * (u - 0.5f);
    float theta = PI_F * v;
    float st = std::sin(theta);
    return {st * std::sin(phi), std::cos(theta), -st * std::cos(phi)};
}

// Bilinear filtering with the sampler's address modes (wrap in u, clamp in
// v; environment.rs:16-17), texel centres at (i + 0.5) / n, as the texture
// unit the reference and the kernels sample through computes it (measured
// on a B200, see textures.h): the texel-space coordinate in FP32, rounded
// to 1/256 of a texel (halves up), less half a texel; its integer part picks
// the texels and its fraction the unit's integer weights, and the FP32
// texels filter as unit_filter_float does.
inline V3f env_bilinear(const EnvTables& e, float u, float v) {
    auto axis = [](float c, uint32_t n, long* i, int32_t* a) {
        const float xs = c * float(n);
        const long q = long(std::floor(double(xs) * 256.0 + 0.5)) - 128;
        *i = q >= 0 ? q / 256 : -((-q + 255) / 256);
        *a = int32_t(q - *i * 256);
    };
    long ix, iy;
    int32_t ax, ay;
    axis(u, e.width, &ix, &ax);
    axis(v, e.height, &iy, &ay);
    auto wrap = [&](long i) { long w = long(e.width); return size_t(((i % w) + w) % w); };
    auto clampi = [&](long j) { return size_t(std::min(std::max(j, 0L), long(e.height) - 1)); };
    const size_t xs[4] = {wrap(ix), wrap(ix + 1), wrap(ix), wrap(ix + 1)};
    const size_t ys[4] = {clampi(iy), clampi(iy), clampi(iy + 1), clampi(iy + 1)};
    int32_t w[4];
    unit_weights(ax, ay, w);
    float out[3];
    for (int c = 0; c < 3; ++c) {
        float t[4];
        for (int k = 0; k < 4; ++k) t[k] = e.texels[4 * (ys[k] * e.width + xs[k]) + c];
        out[c] = unit_filter_float(t, w);
    }
    return V3f(out[0], out[1], out[2]);
}

inline V3f env_radiance(const EnvTables& e, V3f d) {  // environment.slang:88-90
    float u, v;
    uv_from_direction(d, &u, &v);
    return env_bilinear(e, u, v);
}

struct EnvSample {
    V3f direction, radiance;
    float pdf;
    uint32_t row, col;
};
inline EnvSample env_sample(const EnvTables& e, float ux, float uy) {  // environment.slang:94-107
    CdfSlot row = sample_cdf(e.marginal.data(), e.height, ux);
    CdfSlot col = sample_cdf(e.conditional.data() + size_t(row.index) * (e.width + 1), e.width, uy);
    float u = col.position, v = row.position;
    float sin_theta = std::sin(PI_F * v);
    EnvSample s;
    s.direction = direction_from_uv(u, v);
    s.radiance = env_bilinear(e, u, v);
    s.pdf = sin_theta > 0.0f ? e.pdfs[size_t(row.index) * e.width + col.index] / (2.0f * PI_F * PI_F * sin_theta)
                             : 0.0f;
    s.row = row.index;
    s.col = col.index;
    return s;
}
inline float env_pdf(const EnvTables& e, V3f d) {  // environment.slang:111-120
    float sin_theta = std::sqrt(std::max(0.0f, 1.0f - d.y * d.y));
    if (sin_theta <= 0.0f) return 0.0f;
    float u, v;
    uv_from_direction(d, &u, &v);
    uint32_t col = std::min(uint32_t(u * float(e.width)), e.width - 1);
    uint32_t row = std::min(uint32_t(v * float(e.height)), e.height - 1);
    return e.pdfs[size_t(row) * e.width + col] / (2.0f * PI_F * PI_F * sin_theta);
}

}  // namespace oracle
