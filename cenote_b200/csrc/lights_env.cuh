// Next-event sampling on the device: the power-proportional alias walk over
// the light list (crates/cenote/shaders/lights.slang:93-160) and the
// environment's marginal/conditional CDF sampler, pdf and radiance lookup
// (crates/cenote/shaders/environment.slang:41-120). Radiance is read through
// a hardware-filtered texture (bilinear, wrap in u, clamp in v), the same
// sampler state the reference binds (crates/cenote/src/environment.rs:16-17).
#pragma once
#include "records.h"
#include "vecmath.cuh"

namespace cn {

constexpr float ENV_PI = 3.14159265358979323846f;

struct LightConn {
    float3 direction;
    float tmax;
    float3 radiance;
    float pdf;
    bool delta;
    uint32_t instance, primitive;
    uint32_t record;  // the light record drawn (slot or its alias)
    float b1, b2;     // triangle lights: the sampled point's barycentrics (lights.slang:76-87)
};

__device__ __forceinline__ LightConn sample_lights(const LightRecord* lights, uint32_t count, float u, float2 up,
                                                   float3 from) {
    float scaled = u * float(count);
    uint32_t slot = min(uint32_t(scaled), count - 1);
    uint32_t rec = slot;
    if (scaled - float(slot) >= __ldg(&lights[slot].alias_threshold)) rec = __ldg(&lights[slot].alias_index);
    const LightRecord* L = lights + rec;
    // The record in five 16-byte loads.
    const float4* q = reinterpret_cast<const float4*>(L);
    float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3), e = __ldg(q + 4);
    float3 anchor = xyz(a), edge1 = xyz(b), edge2 = xyz(c), emission = xyz(d);
    float lpdf = a.w;
    uint32_t kind = __float_as_uint(e.x);
    LightConn r;
    r.pdf = 0.0f;
    r.direction = f3(0.0f);
    r.tmax = 1e30f;
    r.radiance = emission;
    r.delta = kind != KIND_TRIANGLE;
    r.instance = __float_as_uint(d.w);
    r.primitive = __float_as_uint(e.y);
    r.record = rec;
    r.b1 = r.b2 = 0.0f;
    if (kind == KIND_TRIANGLE) {
        float su = sqrtf(up.x);
        float b1 = 1.0f - su, b2 = up.y * su;
        r.b1 = b1;
        r.b2 = b2;
        float3 pos = anchor + b1 * edge1 + b2 * edge2;
        float3 delta = pos - from;
        float r2 = dot(delta, delta);
        float3 n = normalize(cross(edge1, edge2));
        float3 dir = delta * rsqrtf(r2);
        float cl = -dot(n, dir);
        if (r2 > 0.0f && cl > 0.0f && lpdf > 0.0f) {
            r.direction = dir;
            r.pdf = lpdf * r2 / cl;
            r.tmax = sqrtf(r2) * 1.001f;
        }
    } else if (kind == KIND_DISTANT) {
        r.direction = -anchor;
        r.pdf = lpdf;
    } else {
        float3 delta = anchor - from;
        float r2 = dot(delta, delta);
        if (r2 > 0.0f && lpdf > 0.0f) {
            float rr = sqrtf(r2);
            r.direction = delta / rr;
            r.radiance = emission / r2;
            r.pdf = lpdf;
            r.tmax = rr;
        }
    }
    return r;
}

// The last index i < count with cdf[i] <= u, and the position inside it.
// The cutpoint table narrows the search first: with b = floor(u·ENV_CUTS),
// b / ENV_CUTS <= u < (b + 1) / ENV_CUTS, so the answer lies between the
// answers for those two values, cut[b] and cut[b + 1]; the search then runs
// the same comparison over that range and returns the same index as a search
// of the whole CDF, in one or two steps where the distribution is smooth.
__device__ __forceinline__ uint32_t sample_cdf(const float* cdf, const uint32_t* cut, uint32_t count, float u,
                                               float* position) {
    const uint32_t b = min(uint32_t(u * float(ENV_CUTS)), ENV_CUTS - 1u);
    uint32_t lo = __ldg(cut + b), hi = __ldg(cut + b + 1) + 1u;
    while (lo + 1 < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(cdf + mid) <= u) lo = mid;
        else hi = mid;
    }
    float c0 = __ldg(cdf + lo), c1 = __ldg(cdf + lo + 1);
    float w = c1 - c0;
    float frac = w > 0.0f ? (u - c0) / w : 0.0f;
    *position = (float(lo) + frac) / float(count);
    return lo;
}

__device__ __forceinline__ float2 env_uv(float3 d) {
    return make_float2(0.5f + atan2f(d.x, -d.z) / (2.0f * ENV_PI), acosf(clampf(d.y, -1.0f, 1.0f)) / ENV_PI);
}
__device__ __forceinline__ float3 env_dir(float u, float v) {
    float sp, cp, st, ct;
    sincosf(2.0f * ENV_PI * (u - 0.5f), &sp, &cp);
    sincosf(ENV_PI * v, &st, &ct);
    return f3(st * sp, ct, -st * cp);
}
__device__ __forceinline__ float3 env_lookup(const DeviceScene& s, float u, float v) {
    float4 t = tex2D<float4>(cudaTextureObject_t(s.env_tex), u, v);
    return xyz(t);
}
__device__ __forceinline__ float3 env_radiance(const DeviceScene& s, float3 d) {
    float2 uv = env_uv(d);
    return env_lookup(s, uv.x, uv.y);
}

struct EnvSample {
    float3 direction, radiance;
    float pdf;
    uint32_t row, col;
};
__device__ __forceinline__ EnvSample env_sample(const DeviceScene& s, float2 u) {
    float v, uu;
    uint32_t row = sample_cdf(s.env_marginal, s.env_cut, s.env_h, u.x, &v);
    uint32_t col = sample_cdf(s.env_conditional + size_t(row) * (s.env_w + 1), s.env_cut + size_t(row + 1) * (ENV_CUTS + 1),
                              s.env_w, u.y, &uu);
    float st = sinf(ENV_PI * v);
    EnvSample r;
    r.direction = env_dir(uu, v);
    r.radiance = env_lookup(s, uu, v);
    r.pdf = st > 0.0f ? __ldg(s.env_pdfs + size_t(row) * s.env_w + col) / (2.0f * ENV_PI * ENV_PI * st) : 0.0f;
    r.row = row;
    r.col = col;
    return r;
}
__device__ __forceinline__ float env_pdf(const DeviceScene& s, float3 d) {
    float st = sqrtf(fmaxf(0.0f, 1.0f - d.y * d.y));
    if (st <= 0.0f) return 0.0f;
    float2 uv = env_uv(d);
    uint32_t col = min(uint32_t(uv.x * float(s.env_w)), s.env_w - 1);
    uint32_t row = min(uint32_t(uv.y * float(s.env_h)), s.env_h - 1);
    return __ldg(s.env_pdfs + size_t(row) * s.env_w + col) / (2.0f * ENV_PI * ENV_PI * st);
}

}  // namespace cn
