// The OpenPBR closure on the device, FP32: EON diffuse, GGX (alpha = r²,
// separable Smith), spherical-caps VNDF sampling, exact dielectric and
// Schlick conductor Fresnel, Kulla-Conty compensation from the baked tables,
// coat, LTC fuzz, rough and thin-walled glass, one-sample-MIS lobe choice.
// Every formula follows crates/cenote/shaders/openpbr.slang (line numbers in
// the comments); the tables are read with the same clamped multilinear rule,
// as FP32 software lerps over point loads through the read-only cache.
#pragma once
#include "records.h"
#include "vecmath.cuh"

namespace cn {

constexpr float PBR_PI = 3.14159265358979f;  // openpbr.slang:40
constexpr float MIN_SPECULAR_ROUGHNESS = 0.035f;
constexpr uint32_t T_GGX_E = 0, T_GGX_E_AVG = 1024, T_GLASS_E = 1056, T_GLASS_E_AVG = 5152,
                   T_GLASS_INV_E = 5408, T_GLASS_INV_E_AVG = 9504, T_DIELECTRIC_E = 9760,
                   T_SHEEN_A = 13856, T_SHEEN_B = 14880, T_SHEEN_R = 15904, T_FLOATS = 16928;
constexpr uint32_t LOBE_DIFFUSE = 0, LOBE_SPECULAR = 1, LOBE_TRANSMISSION = 2, LOBE_COAT = 3, LOBE_FUZZ = 4;

// :97-121
__device__ __forceinline__ float tread1(const float* t, uint32_t off, uint32_t size, float x) {
    float fx = saturatef(x) * float(size - 1);
    uint32_t i = min(uint32_t(fx), size - 1);
    uint32_t j = min(i + 1, size - 1);
    return lerpf(__ldg(t + off + i), __ldg(t + off + j), fx - float(i));
}
__device__ __forceinline__ float tread2(const float* t, uint32_t off, uint32_t sx, uint32_t sy, float x, float y) {
    float fy = saturatef(y) * float(sy - 1);
    uint32_t i = min(uint32_t(fy), sy - 1);
    uint32_t j = min(i + 1, sy - 1);
    return lerpf(tread1(t, off + sx * i, sx, x), tread1(t, off + sx * j, sx, x), fy - float(i));
}
__device__ __forceinline__ float tread3(const float* t, uint32_t off, uint32_t s, float x, float y, float z) {
    float fz = saturatef(z) * float(s - 1);
    uint32_t i = min(uint32_t(fz), s - 1);
    uint32_t j = min(i + 1, s - 1);
    uint32_t plane = s * s;
    return lerpf(tread2(t, off + plane * i, s, s, x, y), tread2(t, off + plane * j, s, s, x, y), fz - float(i));
}
__device__ __forceinline__ float ior_remap(float eta) { return sqrtf(fabsf(eta - 1.0f) / (eta + 1.0f)); }

// EON diffuse, :134-166
constexpr float FON_A = 0.5f - 2.0f / (3.0f * PBR_PI);
constexpr float FON_B = 2.0f / 3.0f - 28.0f / (15.0f * PBR_PI);
__device__ __forceinline__ float fon_albedo(float mu, float r) {
    float g = 1.0f - mu;
    float gop = g * (0.0571085289f + g * (0.491881867f + g * (-0.332181442f + g * 0.0714429953f)));
    return (1.0f + r * gop) / (1.0f + FON_A * r);
}
__device__ __forceinline__ float3 eon_brdf(float3 rho, float r, float3 wi, float3 wo) {
    float s = dot(wi, wo) - wi.z * wo.z;
    float sot = s > 0.0f ? s / fmaxf(wi.z, wo.z) : s;
    float A = 1.0f / (1.0f + FON_A * r);
    float3 single = (rho / PBR_PI) * A * (1.0f + r * sot);
    float ai = fon_albedo(wi.z, r), ao = fon_albedo(wo.z, r);
    float aavg = A * (1.0f + FON_B * r);
    float3 rm = (rho * rho) * aavg / (f3(1.0f) - rho * (1.0f - aavg));
    const float eps = 1e-7f;
    float3 multi = (rm / PBR_PI) * fmaxf(eps, 1.0f - ao) * fmaxf(eps, 1.0f - ai) / fmaxf(eps, 1.0f - aavg);
    return single + multi;
}

// GGX, :179-216
// GGX D. For a unit half vector the reference's denominator hz²(α²−1)+1
// equals hx²+hy²+hz²α²; the latter has no cancellation as hz → 1, where the
// former loses up to ~1e-3 relative in FP32 at the 0.035 roughness floor.
__device__ __forceinline__ float ggx_d(float alpha, float3 h) {
    float a2 = alpha * alpha;
    float d = fmaf(h.z * h.z, a2, h.x * h.x + h.y * h.y);
    return h.z > 0.0f ? a2 / (PBR_PI * d * d) : 0.0f;
}
__device__ __forceinline__ float smith_g1(float alpha, float vz) {
    float a2 = alpha * alpha;
    return 2.0f * fabsf(vz) / (fabsf(vz) + sqrtf(vz * vz * (1.0f - a2) + a2));
}
__device__ __forceinline__ float3 sample_vndf(float3 wo, float alpha, float ux, float uy) {
    float3 ws = normalize(f3(wo.x * alpha, wo.y * alpha, wo.z));
    float phi = 2.0f * PBR_PI * ux;
    float z = fmaf(1.0f - uy, 1.0f + ws.z, -ws.z);
    float st = sqrtf(clampf(1.0f - z * z, 0.0f, 1.0f));
    float sp, cp;
    sincosf(phi, &sp, &cp);
    float3 h = f3(st * cp, st * sp, z) + ws;
    return normalize(f3(h.x * alpha, h.y * alpha, h.z));
}
__device__ __forceinline__ float vndf_reflect_pdf(float alpha, float3 wo, float3 h) {
    return smith_g1(alpha, wo.z) * ggx_d(alpha, h) / (4.0f * wo.z);
}

// Fresnel, :221-277
__device__ __forceinline__ float3 fresnel_schlick(float3 f0, float c) {
    float m = 1.0f - fabsf(c);
    float m2 = m * m;
    return f0 + (1.0f - f0) * m2 * m2 * m;
}
__device__ __forceinline__ float fresnel_dielectric(float eta, float cosine) {
    float mu = fabsf(cosine);
    float sin2 = 1.0f - mu * mu;
    float cos2t = 1.0f - sin2 / (eta * eta);
    if (cos2t < 0.0f) return 1.0f;
    float t0 = sqrtf(cos2t);
    float t1 = eta * t0, t2 = eta * mu;
    float rs = (mu - t1) / (mu + t1);
    float rp = (t0 - t2) / (t0 + t2);
    return (rs * rs + rp * rp) / 2.0f;
}
__device__ __forceinline__ float fresnel_dielectric_average(float eta) {
    if (eta < 1.0f) return 0.997118f + eta * (0.1014f - eta * (0.965241f + eta * 0.130607f));
    return (eta - 1.0f) / (4.08567f + 1.00071f * eta);
}
__device__ __forceinline__ float3 fresnel_ms(float3 fss, float eavg) {
    return fss * eavg / (f3(1.0f) - fss * (1.0f - eavg));
}

struct Closure {  // :295-340
    float3 base_color, fuzz_color, glass_tint, thin_r, thin_t, base_weight, conductor_scale, glass_scale, aov_albedo;
    float metalness, transmission_weight, coat_weight, coat_ior, fuzz_weight, base_roughness;
    float alpha, coat_alpha, eta;
    float fuzz_a, fuzz_b, fuzz_r, fuzz_atten, coat_e, coat_scale, spec_e, dielectric_scale;
    float thin_alpha, thin_scale_r, thin_scale_t, thin_t_share;
    float w_fuzz, w_coat, w_spec, w_diffuse, w_total;
    bool exiting, has_specular, thin_walled;
};

__device__ __forceinline__ float3 reflection_scale(const float* t, float rough, float mu, float3 fss) {
    float e = fmaxf(1e-4f, tread2(t, T_GGX_E, 32, 32, rough, mu));
    float eavg = tread1(t, T_GGX_E_AVG, 32, rough);
    return 1.0f + fresnel_ms(fss, eavg) * ((1.0f - e) / e);
}
__device__ __forceinline__ float reflection_scale1(const float* t, float rough, float mu, float fss) {
    float e = fmaxf(1e-4f, tread2(t, T_GGX_E, 32, 32, rough, mu));
    float eavg = tread1(t, T_GGX_E_AVG, 32, rough);
    return 1.0f + (fss * eavg / (1.0f - fss * (1.0f - eavg))) * ((1.0f - e) / e);
}
__device__ __forceinline__ float dielectric_albedo(const float* t, float rough, float mu, float eta) {
    if (eta < 1.0f) return fresnel_dielectric(eta, mu);
    return tread3(t, T_DIELECTRIC_E, 16, rough, mu, ior_remap(eta));
}

// :391-587
__device__ __forceinline__ Closure resolve_closure(const float* t, const Material& m, float3 wo, bool exiting) {
    Closure c;
    c.base_color = ld3(m.base_color);
    c.fuzz_color = ld3(m.fuzz_color);
    c.metalness = m.metalness;
    c.transmission_weight = m.transmission_weight;
    c.coat_weight = m.coat_weight;
    c.coat_ior = m.coat_ior;
    c.fuzz_weight = m.fuzz_weight;
    c.base_roughness = m.base_roughness;
    c.thin_walled = m.thin_walled != 0;
    c.exiting = exiting;
    c.has_specular = exiting || m.metalness > 0.0f || m.transmission_weight > 0.0f || m.specular_weight > 0.0f;
    const float mu = wo.z;
    const bool coat_on = m.coat_weight > 0.0f && !exiting;
    float rough = clampf(m.specular_roughness, MIN_SPECULAR_ROUGHNESS, 1.0f);
    float coat_rough = clampf(m.coat_roughness, MIN_SPECULAR_ROUGHNESS, 1.0f);
    if (coat_on) {
        float var = fminf(1.0f, rough * rough * rough * rough + 2.0f * coat_rough * coat_rough * coat_rough * coat_rough);
        rough = lerpf(rough, sqrtf(sqrtf(var)), m.coat_weight);
    }
    c.alpha = rough * rough;
    c.coat_alpha = coat_rough * coat_rough;

    float eta_s = fmaxf(m.specular_ior, 1e-4f);
    if (coat_on) {
        float eta_bc = m.coat_ior > eta_s ? m.coat_ior / eta_s : eta_s / m.coat_ior;
        eta_s = lerpf(eta_s, eta_bc, m.coat_weight);
    }
    float f0 = (eta_s - 1.0f) * (eta_s - 1.0f) / ((eta_s + 1.0f) * (eta_s + 1.0f));
    float weight = clampf(m.specular_weight, 0.0f, f0 > 1e-6f ? 1.0f / f0 : 0.0f);
    float epsilon = signf(eta_s - 1.0f) * sqrtf(weight * f0);
    float eta = (1.0f + epsilon) / fmaxf(1e-3f, 1.0f - epsilon);
    if (fabsf(eta - 1.0f) < 1e-3f) eta = eta < 1.0f ? 1.0f - 1e-3f : 1.0f + 1e-3f;
    c.eta = exiting ? 1.0f / eta : eta;

    c.fuzz_a = 0.0f;
    c.fuzz_b = 0.0f;
    c.fuzz_r = 0.0f;
    c.fuzz_atten = 1.0f;
    if (m.fuzz_weight > 0.0f && !exiting) {
        float fr = clampf(m.fuzz_roughness, 1e-3f, 1.0f);
        float a = tread2(t, T_SHEEN_A, 32, 32, mu, fr);
        float r = tread2(t, T_SHEEN_R, 32, 32, mu, fr);
        if (fabsf(a) >= 1e-5f && r >= 1e-5f) {
            c.fuzz_a = a;
            c.fuzz_b = tread2(t, T_SHEEN_B, 32, 32, mu, fr);
            c.fuzz_r = r;
            c.fuzz_atten = 1.0f - m.fuzz_weight * r;
        }
    }

    c.coat_e = 0.0f;
    c.coat_scale = 1.0f;
    float3 coat_atten = f3(1.0f);
    if (coat_on) {
        c.coat_e = dielectric_albedo(t, coat_rough, mu, m.coat_ior);
        float fss_coat = fresnel_dielectric_average(m.coat_ior);
        c.coat_scale = reflection_scale1(t, coat_rough, mu, fss_coat);
        // coatDarkening, :371-384
        float k_rough = 1.0f - (1.0f - fss_coat) / (m.coat_ior * m.coat_ior);
        float k_smooth = fresnel_dielectric(m.coat_ior, mu);
        float rough_diffuse = lerpf(1.0f, rough, saturatef(m.specular_weight * f0));
        float base_rough = lerpf(rough_diffuse, rough, m.metalness);
        float k = lerpf(k_smooth, k_rough, base_rough);
        float3 base_albedo = lerp3(c.base_color, f3(1.0f), (1.0f - m.metalness) * m.transmission_weight);
        float3 darkened = (1.0f - k) / fmax3(f3(1e-4f), 1.0f - base_albedo * k);
        float3 dark = lerp3(f3(1.0f), darkened, m.coat_weight * m.coat_darkening);
        coat_atten = lerp3(f3(1.0f), ld3(m.coat_color) * (1.0f - c.coat_e), m.coat_weight) * dark;
    }
    c.base_weight = c.fuzz_atten * coat_atten;

    c.spec_e = c.has_specular ? dielectric_albedo(t, rough, mu, c.eta) : 0.0f;
    c.conductor_scale = reflection_scale(t, rough, mu, lerp3(c.base_color, f3(1.0f), 1.0f / 21.0f));
    c.dielectric_scale = reflection_scale1(t, rough, mu, fresnel_dielectric_average(c.eta));

    float3 tcol = ld3(m.transmission_color);
    c.glass_tint = m.transmission_depth == 0.0f ? tcol : f3(1.0f);
    float geta = c.eta;
    uint32_t goff = T_GLASS_E, gavg = T_GLASS_E_AVG;
    if (geta < 1.0f) {
        geta = 1.0f / geta;
        goff = T_GLASS_INV_E;
        gavg = T_GLASS_INV_E_AVG;
    }
    float gz = ior_remap(geta);
    float ge = fmaxf(1e-4f, tread3(t, goff, 16, rough, mu, gz));
    float geavg = tread2(t, gavg, 16, 16, rough, gz);
    c.glass_scale = 1.0f + fresnel_ms(c.glass_tint, geavg) * ((1.0f - ge) / ge);

    c.thin_r = f3(0.0f);
    c.thin_t = f3(0.0f);
    c.thin_alpha = c.alpha;
    c.thin_scale_r = 1.0f;
    c.thin_scale_t = 1.0f;
    c.thin_t_share = 0.0f;
    const bool thin = c.thin_walled && m.transmission_weight > 0.0f;
    if (thin) {
        float teta = fmaxf(eta, 1.0f / eta);
        float r1 = fresnel_dielectric(teta, mu);
        float t1 = 1.0f - r1;
        float cos2t = fmaxf(0.0f, 1.0f - (1.0f - mu * mu) / (teta * teta));
        float3 absorb = cos2t > 0.0f ? pow3(clamp3(tcol, 1e-4f, 1.0f), f3(1.0f / sqrtf(cos2t))) : f3(0.0f);
        float3 denom = fmax3(f3(1e-4f), 1.0f - absorb * absorb * (r1 * r1));
        c.thin_t = absorb * (t1 * t1) / denom;
        c.thin_r = r1 + c.thin_t * (r1 * absorb);
        float thin_rough = clampf(rough * sqrtf(3.4f * (teta - 1.0f) * (teta - 0.5f) * (teta - 0.5f) / (teta * teta * teta)),
                                  MIN_SPECULAR_ROUGHNESS, 1.0f);
        c.thin_alpha = thin_rough * thin_rough;
        c.thin_scale_r = reflection_scale1(t, rough, mu, 1.0f);
        c.thin_scale_t = reflection_scale1(t, thin_rough, mu, 1.0f);
        float total = avg3(c.thin_r) + avg3(c.thin_t);
        c.thin_t_share = total > 0.0f ? avg3(c.thin_t) / total : 0.0f;
    }

    float schlick_s = saturatef((c.spec_e - f0) / fmaxf(1e-4f, 1.0f - f0));
    float3 metal_e = lerp3(c.base_color, f3(1.0f), schlick_s);
    float glass_total = thin ? avg3(c.thin_r + c.thin_t) : c.spec_e + (1.0f - c.spec_e) * avg3(c.glass_tint);
    float dielectric_e = lerpf(c.spec_e, glass_total, m.transmission_weight);
    float base_avg = avg3(c.base_weight);
    c.w_fuzz = exiting ? 0.0f : m.fuzz_weight * c.fuzz_r * avg3(c.fuzz_color);
    c.w_coat = exiting ? 0.0f : c.fuzz_atten * m.coat_weight * c.coat_e;
    c.w_spec = c.has_specular ? base_avg * lerpf(dielectric_e, avg3(metal_e), m.metalness) : 0.0f;
    c.w_diffuse = exiting ? 0.0f
                          : base_avg * (1.0f - m.metalness) * (1.0f - m.transmission_weight) * (1.0f - c.spec_e) *
                                avg3(c.base_color);
    if (exiting) c.w_spec = 1.0f;
    c.w_total = c.w_fuzz + c.w_coat + c.w_spec + c.w_diffuse;

    float3 glass_color = thin ? c.thin_r + c.thin_t : f3(c.spec_e) + (1.0f - c.spec_e) * c.glass_tint;
    if (exiting) {
        c.aov_albedo = glass_color;
    } else {
        float3 dcol = lerp3(f3(c.spec_e), glass_color, m.transmission_weight);
        float3 scol = c.has_specular ? lerp3(dcol, metal_e, m.metalness) : f3(0.0f);
        c.aov_albedo = m.fuzz_weight * c.fuzz_r * c.fuzz_color + f3(c.fuzz_atten * m.coat_weight * c.coat_e) +
                       c.base_weight *
                           (scol + (1.0f - m.metalness) * (1.0f - m.transmission_weight) * (1.0f - c.spec_e) * c.base_color);
    }
    return c;
}

__device__ __forceinline__ float aov_record_fraction(const Closure& c, uint32_t lobe) {  // :596-608
    float alpha;
    if (lobe == LOBE_COAT) alpha = c.coat_alpha;
    else if (lobe == LOBE_SPECULAR) alpha = c.alpha;
    else if (lobe == LOBE_TRANSMISSION) alpha = c.thin_walled ? c.thin_alpha : c.alpha;
    else return 1.0f;
    return saturatef(sqrtf(alpha) / 0.15f);
}
__device__ __forceinline__ float3 aov_pass_tint(const Closure& c, uint32_t lobe) {  // :614-622
    if (lobe == LOBE_TRANSMISSION) return c.glass_tint;
    if (lobe == LOBE_SPECULAR) return lerp3(f3(1.0f), c.base_color, c.metalness);
    return f3(1.0f);
}

__device__ __forceinline__ float sheen_density(const Closure& c, float3 w) {  // :629-636
    float a = c.fuzz_a, b = c.fuzz_b;
    float q = a * w.x + b * w.z;
    float ls = q * q + (a * w.y) * (a * w.y) + w.z * w.z;
    float ratio = a / ls;
    return fmaxf(w.z, 0.0f) * ratio * ratio / PBR_PI;
}
__device__ __forceinline__ float3 align_to_view(float3 v, float3 wo, bool inverse) {  // :639-647
    float len = sqrtf(wo.x * wo.x + wo.y * wo.y);
    if (len < 1e-6f) return v;
    float cp = wo.x / len;
    float sp = (inverse ? -wo.y : wo.y) / len;
    return f3(cp * v.x + sp * v.y, cp * v.y - sp * v.x, v.z);
}
__device__ __forceinline__ float reflection_core(float alpha, float3 wi, float3 wo, float3 h) {  // :650-653
    return ggx_d(alpha, h) * smith_g1(alpha, wo.z) * smith_g1(alpha, wi.z) / (4.0f * wo.z * wi.z);
}

// evalBsdf, :681-744
__device__ __forceinline__ float3 eval_bsdf(const Closure& c, float3 wi, float3 wo) {
    if (wo.z <= 0.0f || wi.z == 0.0f) return f3(0.0f);
    if (wi.z < 0.0f) {
        float gs = c.exiting ? 1.0f : (1.0f - c.metalness) * c.transmission_weight;
        if (gs <= 0.0f || (c.exiting && c.thin_walled)) return f3(0.0f);
        if (c.thin_walled) {
            float3 fl = f3(wi.x, wi.y, -wi.z);
            float3 h = normalize(fl + wo);
            float core = reflection_core(c.thin_alpha, fl, wo, h);
            return c.base_weight * gs * c.thin_t * c.thin_scale_t * core;
        }
        float3 hu = wo + c.eta * wi;
        float len2 = dot(hu, hu);
        if (len2 < 1e-9f) return f3(0.0f);
        float3 h = hu / sqrtf(len2);
        h = h.z >= 0.0f ? h : -h;
        float cvh = dot(h, wo), clh = dot(h, wi);
        if (cvh <= 0.0f || clh >= 0.0f) return f3(0.0f);
        float f = fresnel_dielectric(c.eta, cvh);
        float core = ggx_d(c.alpha, h) * smith_g1(c.alpha, wo.z) * smith_g1(c.alpha, wi.z) * cvh * (c.eta * c.eta) *
                     fabsf(clh) / (wo.z * fabsf(wi.z) * len2);
        return c.base_weight * gs * (1.0f - f) * c.glass_tint * c.glass_scale * core;
    }
    float3 result = f3(0.0f);
    if (c.fuzz_r > 0.0f) {
        float d = sheen_density(c, align_to_view(wi, wo, false));
        result = result + c.fuzz_weight * c.fuzz_color * c.fuzz_r * d / wi.z;
    }
    float3 h = normalize(wi + wo);
    if (c.coat_weight > 0.0f && !c.exiting) {
        float cf = fresnel_dielectric(c.coat_ior, dot(h, wo));
        result = result + f3(c.fuzz_atten * c.coat_weight * cf * c.coat_scale * reflection_core(c.coat_alpha, wi, wo, h));
    }
    float3 base = f3(0.0f);
    if (c.has_specular) {  // baseReflection, :660-677
        float core = reflection_core(c.alpha, wi, wo, h);
        float cvh = dot(h, wo);
        float fd = fresnel_dielectric(c.eta, cvh);
        if (c.exiting) {
            base = core * fd * c.glass_scale;
        } else {
            float3 conductor = fresnel_schlick(c.base_color, cvh) * c.conductor_scale;
            float3 diel = c.thin_walled ? lerp3(f3(fd * c.dielectric_scale), c.thin_r * c.thin_scale_r, c.transmission_weight)
                                        : lerp3(f3(fd * c.dielectric_scale), fd * c.glass_scale, c.transmission_weight);
            base = core * lerp3(diel, conductor, c.metalness);
        }
    }
    if (!c.exiting)
        base = base + (1.0f - c.metalness) * (1.0f - c.transmission_weight) * (1.0f - c.spec_e) *
                          eon_brdf(c.base_color, c.base_roughness, wi, wo);
    return result + c.base_weight * base;
}

__device__ __forceinline__ float reflect_probability(const Closure& c, float fresnel) {  // :748-752
    float gs = c.exiting ? 1.0f : (1.0f - c.metalness) * c.transmission_weight;
    float tr = c.thin_walled ? c.thin_t_share : 1.0f - fresnel;
    return 1.0f - gs * tr;
}

// bsdfPdf, :756-808
__device__ __forceinline__ float bsdf_pdf(const Closure& c, float3 wi, float3 wo) {
    if (wo.z <= 0.0f || wi.z == 0.0f || c.w_total <= 0.0f) return 0.0f;
    if (wi.z < 0.0f) {
        if (c.w_spec <= 0.0f) return 0.0f;
        float p;
        if (c.thin_walled) {
            float3 fl = f3(wi.x, wi.y, -wi.z);
            float3 h = normalize(fl + wo);
            p = vndf_reflect_pdf(c.thin_alpha, wo, h) * (1.0f - reflect_probability(c, 0.0f));
        } else {
            float3 hu = wo + c.eta * wi;
            float len2 = dot(hu, hu);
            if (len2 < 1e-9f) return 0.0f;
            float3 h = hu / sqrtf(len2);
            h = h.z >= 0.0f ? h : -h;
            float cvh = dot(h, wo), clh = dot(h, wi);
            if (cvh <= 0.0f || clh >= 0.0f) return 0.0f;
            float f = fresnel_dielectric(c.eta, cvh);
            float vndf = smith_g1(c.alpha, wo.z) * ggx_d(c.alpha, h) * cvh / wo.z;
            float jac = (c.eta * c.eta) * fabsf(clh) / len2;
            p = vndf * jac * (1.0f - reflect_probability(c, f));
        }
        return c.w_spec * p / c.w_total;
    }
    float3 h = normalize(wi + wo);
    float p = 0.0f;
    if (c.w_fuzz > 0.0f) p += c.w_fuzz * sheen_density(c, align_to_view(wi, wo, false));
    if (c.w_coat > 0.0f) p += c.w_coat * vndf_reflect_pdf(c.coat_alpha, wo, h);
    if (c.w_spec > 0.0f) {
        float f = fresnel_dielectric(c.eta, dot(h, wo));
        p += c.w_spec * vndf_reflect_pdf(c.alpha, wo, h) * reflect_probability(c, f);
    }
    if (c.w_diffuse > 0.0f) p += c.w_diffuse * wi.z / PBR_PI;
    return p / c.w_total;
}

struct BsdfSample {
    float3 wi;
    float pdf;
    uint32_t lobe;
};

// The closure's value and pdf for one direction: the shading kernel needs both
// for the next-event direction and for the scattered one, and evaluating
// them together shares the half vector, D and G1 terms. (Inline: out of line
// the closure moves to local memory, which costs more than the instruction
// cache it saves.)
struct EvalPdf {
    float3 f;
    float pdf;
};

__device__ __forceinline__ EvalPdf eval_pdf(const Closure& c, float3 wi, float3 wo) {
    EvalPdf r;
    r.f = eval_bsdf(c, wi, wo);
    r.pdf = bsdf_pdf(c, wi, wo);
    return r;
}

// sampleBsdf, :821-884, without its closing pdf evaluation: returns false
// (no direction, pdf 0) where the reference returns pdf 0 early.
__device__ __forceinline__ bool sample_bsdf_dir(const Closure& c, float3 wo, float u_lobe, float ux, float uy,
                                                BsdfSample& r);

__device__ __forceinline__ BsdfSample sample_bsdf(const Closure& c, float3 wo, float u_lobe, float ux, float uy) {
    BsdfSample r;
    if (sample_bsdf_dir(c, wo, u_lobe, ux, uy, r)) r.pdf = bsdf_pdf(c, r.wi, wo);
    return r;
}

__device__ __forceinline__ bool sample_bsdf_dir(const Closure& c, float3 wo, float u_lobe, float ux, float uy,
                                                BsdfSample& r) {
    r.wi = f3(0.0f, 0.0f, 1.0f);
    r.pdf = 0.0f;
    r.lobe = LOBE_DIFFUSE;
    if (c.w_total <= 0.0f) return false;
    float pick = u_lobe * c.w_total;
    float3 wi;
    if (pick < c.w_fuzz) {
        r.lobe = LOBE_FUZZ;
        float rr = sqrtf(ux);
        float sp, cp;
        sincosf(2.0f * PBR_PI * uy, &sp, &cp);
        float dx = rr * cp, dy = rr * sp;
        float dz = sqrtf(fmaxf(0.0f, 1.0f - (dx * dx + dy * dy)));
        float3 ws = normalize(f3(dx - dz * c.fuzz_b, dy, dz * c.fuzz_a));
        wi = align_to_view(ws, wo, true);
    } else if (pick < c.w_fuzz + c.w_coat) {
        r.lobe = LOBE_COAT;
        float3 h = sample_vndf(wo, c.coat_alpha, ux, uy);
        wi = 2.0f * dot(wo, h) * h - wo;
    } else if (pick < c.w_fuzz + c.w_coat + c.w_spec) {
        float ub = (pick - c.w_fuzz - c.w_coat) / fmaxf(1e-6f, c.w_spec);
        if (c.thin_walled) {
            if (ub < reflect_probability(c, 0.0f)) {
                r.lobe = LOBE_SPECULAR;
                float3 h = sample_vndf(wo, c.alpha, ux, uy);
                wi = 2.0f * dot(wo, h) * h - wo;
            } else {
                r.lobe = LOBE_TRANSMISSION;
                float3 h = sample_vndf(wo, c.thin_alpha, ux, uy);
                float3 rf = 2.0f * dot(wo, h) * h - wo;
                wi = f3(rf.x, rf.y, -rf.z);
            }
        } else {
            float3 h = sample_vndf(wo, c.alpha, ux, uy);
            float f = fresnel_dielectric(c.eta, dot(h, wo));
            if (ub < reflect_probability(c, f)) {
                r.lobe = LOBE_SPECULAR;
                wi = 2.0f * dot(wo, h) * h - wo;
            } else {
                r.lobe = LOBE_TRANSMISSION;
                float cc = dot(wo, h);
                float cos2t = 1.0f - (1.0f - cc * cc) / (c.eta * c.eta);
                if (cos2t <= 0.0f) return false;
                wi = (cc / c.eta - sqrtf(cos2t)) * h - wo / c.eta;
            }
        }
    } else {
        r.lobe = LOBE_DIFFUSE;
        float rr = sqrtf(ux);
        float sp, cp;
        sincosf(2.0f * PBR_PI * uy, &sp, &cp);
        wi = f3(rr * cp, rr * sp, sqrtf(1.0f - ux));
    }
    r.wi = wi;
    return true;
}

// Duff et al. frame, :888-909
struct Frame {
    float3 t, b, n;
    __device__ __forceinline__ explicit Frame(float3 nn) : n(nn) {
        float s = nn.z >= 0.0f ? 1.0f : -1.0f;
        float a = -1.0f / (s + nn.z);
        float m = nn.x * nn.y * a;
        t = f3(1.0f + s * nn.x * nn.x * a, s * m, -s * nn.x);
        b = f3(m, s + nn.y * nn.y * a, -nn.y);
    }
    __device__ __forceinline__ float3 to_local(float3 v) const { return f3(dot(v, t), dot(v, b), dot(v, n)); }
    __device__ __forceinline__ float3 to_world(float3 v) const { return v.x * t + v.y * b + v.z * n; }
};

__device__ __forceinline__ float power_heuristic(float p, float q) { return (p * p) / (p * p + q * q); }

}  // namespace cn
