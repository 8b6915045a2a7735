// Test infrastructure (CPU oracle): the OpenPBR closure restated from
// crates/cenote/shaders/openpbr.slang, templated on the scalar type. T=double
// is the FP64 oracle the FP32 kernels' eval/pdf are judged against; T=float
// mirrors the kernels for image-level comparisons. Line citations are into
// openpbr.slang unless stated otherwise.
#pragma once
#include <cstdint>
#include "vec.h"

namespace oracle {

constexpr double PI_D = 3.14159265358979;  // openpbr.slang:40 (the reference's literal)
constexpr uint32_t TEXTURE_NONE = 0xffffffffu;

// The 144-byte material record, field order of material.rs:28-109 /
// openpbr.slang:49-78.
struct Material {
    float base_color[3];
    float base_roughness;
    float emission[3];
    float metalness;
    float specular_weight;
    float specular_roughness;
    float specular_ior;
    float transmission_weight;
    float transmission_color[3];
    float transmission_depth;
    float coat_color[3];
    float coat_weight;
    float coat_roughness;
    float coat_ior;
    float coat_darkening;
    float fuzz_weight;
    float fuzz_color[3];
    float fuzz_roughness;
    float opacity;
    uint32_t thin_walled;
    uint32_t base_color_texture;
    uint32_t specular_roughness_texture;
    uint32_t metalness_texture;
    uint32_t emission_texture;
    uint32_t opacity_texture;
    uint32_t normal_texture;
};
static_assert(sizeof(Material) == 144, "material record is 144 bytes");

// Table layout, openpbr.slang:86-95 / tables.rs:51-80.
constexpr uint32_t TABLE_GGX_E = 0;
constexpr uint32_t TABLE_GGX_E_AVG = 1024;
constexpr uint32_t TABLE_GLASS_E = 1056;
constexpr uint32_t TABLE_GLASS_E_AVG = 5152;
constexpr uint32_t TABLE_GLASS_INV_E = 5408;
constexpr uint32_t TABLE_GLASS_INV_E_AVG = 9504;
constexpr uint32_t TABLE_DIELECTRIC_E = 9760;
constexpr uint32_t TABLE_SHEEN_A = 13856;
constexpr uint32_t TABLE_SHEEN_B = 14880;
constexpr uint32_t TABLE_SHEEN_R = 15904;
constexpr uint32_t TABLE_FLOATS = 16928;

constexpr uint32_t LOBE_DIFFUSE = 0;
constexpr uint32_t LOBE_SPECULAR = 1;
constexpr uint32_t LOBE_TRANSMISSION = 2;
constexpr uint32_t LOBE_COAT = 3;
constexpr uint32_t LOBE_FUZZ = 4;

template <class T>
struct MaterialT {  // the material's float fields in the evaluation precision
    V3<T> base_color;
    T base_roughness;
    V3<T> emission;
    T metalness, specular_weight, specular_roughness, specular_ior, transmission_weight;
    V3<T> transmission_color;
    T transmission_depth;
    V3<T> coat_color;
    T coat_weight, coat_roughness, coat_ior, coat_darkening, fuzz_weight;
    V3<T> fuzz_color;
    T fuzz_roughness, opacity;
    uint32_t thin_walled;
    uint32_t normal_texture;
};

template <class T>
inline MaterialT<T> to_t(const Material& m) {
    auto v = [](const float* f) { return V3<T>(T(f[0]), T(f[1]), T(f[2])); };
    MaterialT<T> r;
    r.base_color = v(m.base_color);
    r.base_roughness = T(m.base_roughness);
    r.emission = v(m.emission);
    r.metalness = T(m.metalness);
    r.specular_weight = T(m.specular_weight);
    r.specular_roughness = T(m.specular_roughness);
    r.specular_ior = T(m.specular_ior);
    r.transmission_weight = T(m.transmission_weight);
    r.transmission_color = v(m.transmission_color);
    r.transmission_depth = T(m.transmission_depth);
    r.coat_color = v(m.coat_color);
    r.coat_weight = T(m.coat_weight);
    r.coat_roughness = T(m.coat_roughness);
    r.coat_ior = T(m.coat_ior);
    r.coat_darkening = T(m.coat_darkening);
    r.fuzz_weight = T(m.fuzz_weight);
    r.fuzz_color = v(m.fuzz_color);
    r.fuzz_roughness = T(m.fuzz_roughness);
    r.opacity = T(m.opacity);
    r.thin_walled = m.thin_walled;
    r.normal_texture = m.normal_texture;
    return r;
}

template <class T>
struct BSDF {
    static constexpr T PI = T(PI_D);
    static constexpr T MIN_SPECULAR_ROUGHNESS = T(0.035);  // :45

    // :97-121 — clamped multilinear reads, first axis fastest.
    static T read1(const float* t, uint32_t off, uint32_t size, T x) {
        T fx = saturate(x) * T(size - 1);
        uint32_t i = std::min(uint32_t(fx), size - 1);
        uint32_t j = std::min(i + 1, size - 1);
        return lerp(T(t[off + i]), T(t[off + j]), fx - T(i));
    }
    static T read2(const float* t, uint32_t off, uint32_t sx, uint32_t sy, T x, T y) {
        T fy = saturate(y) * T(sy - 1);
        uint32_t i = std::min(uint32_t(fy), sy - 1);
        uint32_t j = std::min(i + 1, sy - 1);
        return lerp(read1(t, off + sx * i, sx, x), read1(t, off + sx * j, sx, x), fy - T(i));
    }
    static T read3(const float* t, uint32_t off, uint32_t sx, uint32_t sy, uint32_t sz, T x,
                   T y, T z) {
        T fz = saturate(z) * T(sz - 1);
        uint32_t i = std::min(uint32_t(fz), sz - 1);
        uint32_t j = std::min(i + 1, sz - 1);
        uint32_t plane = sx * sy;
        return lerp(read2(t, off + plane * i, sx, sy, x, y), read2(t, off + plane * j, sx, sy, x, y),
                    fz - T(i));
    }
    static T ior_remap(T eta) { return std::sqrt(std::fabs(eta - T(1)) / (eta + T(1))); }  // :125-127

    // EON diffuse, :134-166.
    static constexpr T FON_A = T(0.5) - T(2) / (T(3) * PI);
    static constexpr T FON_B = T(2) / T(3) - T(28) / (T(15) * PI);
    static T fon_albedo(T mu, T r) {
        T g = T(1) - mu;
        T g_over_pi = g * (T(0.0571085289) +
                           g * (T(0.491881867) + g * (T(-0.332181442) + g * T(0.0714429953))));
        return (T(1) + r * g_over_pi) / (T(1) + FON_A * r);
    }
    static V3<T> eon_brdf(V3<T> rho, T r, V3<T> wi, V3<T> wo) {
        T s = dot(wi, wo) - wi.z * wo.z;
        T s_over_t = s > T(0) ? s / std::max(wi.z, wo.z) : s;
        T A = T(1) / (T(1) + FON_A * r);
        V3<T> single = (rho / PI) * A * (T(1) + r * s_over_t);
        T albedo_i = fon_albedo(wi.z, r);
        T albedo_o = fon_albedo(wo.z, r);
        T albedo_avg = A * (T(1) + FON_B * r);
        V3<T> rho_multi = (rho * rho) * albedo_avg / (V3<T>(T(1)) - rho * (T(1) - albedo_avg));
        T eps = T(1e-7);
        V3<T> multi = (rho_multi / PI) * std::max(eps, T(1) - albedo_o) *
                      std::max(eps, T(1) - albedo_i) / std::max(eps, T(1) - albedo_avg);
        return single + multi;
    }
    static V3<T> sample_cosine_hemisphere(T ux, T uy, T* pdf) {  // :170-175
        T r = std::sqrt(ux);
        T phi = T(2) * PI * uy;
        T z = std::sqrt(T(1) - ux);
        *pdf = z / PI;
        return {r * std::cos(phi), r * std::sin(phi), z};
    }

    // GGX, :179-216.
    static T ggx_d(T alpha, T hz) {
        T a2 = alpha * alpha;
        T denom = hz * hz * (a2 - T(1)) + T(1);
        return hz > T(0) ? a2 / (PI * denom * denom) : T(0);
    }
    static T smith_g1(T alpha, T vz) {
        T a2 = alpha * alpha;
        return T(2) * std::fabs(vz) / (std::fabs(vz) + std::sqrt(vz * vz * (T(1) - a2) + a2));
    }
    static V3<T> sample_vndf(V3<T> wo, T alpha, T ux, T uy) {
        V3<T> wo_std = normalize(V3<T>(wo.x * alpha, wo.y * alpha, wo.z));
        T phi = T(2) * PI * ux;
        T z = std::fma(T(1) - uy, T(1) + wo_std.z, -wo_std.z);
        T sin_theta = std::sqrt(clampv(T(1) - z * z, T(0), T(1)));
        V3<T> c(sin_theta * std::cos(phi), sin_theta * std::sin(phi), z);
        V3<T> h_std = c + wo_std;
        return normalize(V3<T>(h_std.x * alpha, h_std.y * alpha, h_std.z));
    }
    static T vndf_reflect_pdf(T alpha, V3<T> wo, V3<T> h) {
        return smith_g1(alpha, wo.z) * ggx_d(alpha, h.z) / (T(4) * wo.z);
    }

    // Fresnel, :221-277.
    static V3<T> fresnel_schlick(V3<T> f0, T cosine) {
        T m = T(1) - std::fabs(cosine);
        T m2 = m * m;
        return f0 + (T(1) - f0) * m2 * m2 * m;
    }
    static V3<T> fresnel_schlick_average(V3<T> f0) {
        return lerp(f0, V3<T>(T(1)), T(1) / T(21));
    }
    static T fresnel_dielectric(T eta, T cosine) {
        T mu = std::fabs(cosine);
        T sin2 = T(1) - mu * mu;
        T cos2t = T(1) - sin2 / (eta * eta);
        if (cos2t < T(0)) return T(1);
        T t0 = std::sqrt(cos2t);
        T t1 = eta * t0;
        T t2 = eta * mu;
        T rs = (mu - t1) / (mu + t1);
        T rp = (t0 - t2) / (t0 + t2);
        return (rs * rs + rp * rp) / T(2);
    }
    static T fresnel_dielectric_average(T eta) {
        if (eta < T(1)) return T(0.997118) + eta * (T(0.1014) - eta * (T(0.965241) + eta * T(0.130607)));
        return (eta - T(1)) / (T(4.08567) + T(1.00071) * eta);
    }
    static V3<T> fresnel_multi_scatter(V3<T> fss, T e_avg) {
        return fss * e_avg / (V3<T>(T(1)) - fss * (T(1) - e_avg));
    }
    static bool refract_direction(V3<T> wo, V3<T> h, T eta, V3<T>* out) {
        T c = dot(wo, h);
        T cos2t = T(1) - (T(1) - c * c) / (eta * eta);
        if (cos2t <= T(0)) return false;
        *out = (c / eta - std::sqrt(cos2t)) * h - wo / eta;
        return true;
    }

    struct Closure {  // :295-340
        MaterialT<T> m;
        const float* tables;
        T alpha, coat_alpha, eta;
        bool exiting, has_specular;
        T fuzz_a, fuzz_b, fuzz_r, fuzz_atten;
        T coat_e, coat_scale;
        V3<T> base_weight;
        T spec_e;
        V3<T> conductor_scale;
        T dielectric_scale;
        V3<T> glass_scale, glass_tint;
        V3<T> thin_r, thin_t;
        T thin_alpha, thin_scale_r, thin_scale_t, thin_t_share;
        T w_fuzz, w_coat, w_spec, w_diffuse, w_total;
        V3<T> aov_albedo;
    };

    static V3<T> reflection_scale(const float* t, T rough, T mu, V3<T> fss) {  // :348-352
        T e = std::max(T(1e-4), read2(t, TABLE_GGX_E, 32, 32, rough, mu));
        T e_avg = read1(t, TABLE_GGX_E_AVG, 32, rough);
        return T(1) + fresnel_multi_scatter(fss, e_avg) * ((T(1) - e) / e);
    }
    static T dielectric_albedo(const float* t, T rough, T mu, T eta) {  // :357-363
        if (eta < T(1)) return fresnel_dielectric(eta, mu);
        return read3(t, TABLE_DIELECTRIC_E, 16, 16, 16, rough, mu, ior_remap(eta));
    }
    static V3<T> coat_darkening(const MaterialT<T>& m, T rough, T mu, T base_fresnel) {  // :371-384
        T fss_coat = fresnel_dielectric_average(m.coat_ior);
        T k_rough = T(1) - (T(1) - fss_coat) / (m.coat_ior * m.coat_ior);
        T k_smooth = fresnel_dielectric(m.coat_ior, mu);
        T rough_diffuse = lerp(T(1), rough, saturate(m.specular_weight * base_fresnel));
        T base_rough = lerp(rough_diffuse, rough, m.metalness);
        T k = lerp(k_smooth, k_rough, base_rough);
        V3<T> base_albedo = lerp(m.base_color, V3<T>(T(1)), (T(1) - m.metalness) * m.transmission_weight);
        V3<T> darkened = (T(1) - k) / vmax(V3<T>(T(1e-4)), T(1) - base_albedo * k);
        return lerp(V3<T>(T(1)), darkened, m.coat_weight * m.coat_darkening);
    }

    static Closure resolve(const float* t, const MaterialT<T>& m, V3<T> wo, bool exiting) {  // :391-587
        Closure c;
        c.m = m;
        c.tables = t;
        c.exiting = exiting;
        c.has_specular = exiting || m.metalness > T(0) || m.transmission_weight > T(0) ||
                         m.specular_weight > T(0);
        T mu = wo.z;
        T rough = clampv(m.specular_roughness, MIN_SPECULAR_ROUGHNESS, T(1));
        T coat_rough = clampv(m.coat_roughness, MIN_SPECULAR_ROUGHNESS, T(1));
        if (m.coat_weight > T(0) && !exiting) {
            T variance = std::min(T(1), rough * rough * rough * rough +
                                            T(2) * coat_rough * coat_rough * coat_rough * coat_rough);
            rough = lerp(rough, std::sqrt(std::sqrt(variance)), m.coat_weight);
        }
        c.alpha = rough * rough;
        c.coat_alpha = coat_rough * coat_rough;

        T eta_s = std::max(m.specular_ior, T(1e-4));
        if (m.coat_weight > T(0) && !exiting) {
            T eta_bc = m.coat_ior > eta_s ? m.coat_ior / eta_s : eta_s / m.coat_ior;
            eta_s = lerp(eta_s, eta_bc, m.coat_weight);
        }
        T f0 = (eta_s - T(1)) * (eta_s - T(1)) / ((eta_s + T(1)) * (eta_s + T(1)));
        T weight = clampv(m.specular_weight, T(0), f0 > T(1e-6) ? T(1) / f0 : T(0));
        T epsilon = signum(eta_s - T(1)) * std::sqrt(weight * f0);
        T eta = (T(1) + epsilon) / std::max(T(1e-3), T(1) - epsilon);
        if (std::fabs(eta - T(1)) < T(1e-3)) eta = eta < T(1) ? T(1) - T(1e-3) : T(1) + T(1e-3);
        c.eta = exiting ? T(1) / eta : eta;

        c.fuzz_a = T(0);
        c.fuzz_b = T(0);
        c.fuzz_r = T(0);
        c.fuzz_atten = T(1);
        if (m.fuzz_weight > T(0) && !exiting) {
            T fuzz_rough = clampv(m.fuzz_roughness, T(1e-3), T(1));
            T a = read2(t, TABLE_SHEEN_A, 32, 32, mu, fuzz_rough);
            T r = read2(t, TABLE_SHEEN_R, 32, 32, mu, fuzz_rough);
            if (std::fabs(a) >= T(1e-5) && r >= T(1e-5)) {
                c.fuzz_a = a;
                c.fuzz_b = read2(t, TABLE_SHEEN_B, 32, 32, mu, fuzz_rough);
                c.fuzz_r = r;
                c.fuzz_atten = T(1) - m.fuzz_weight * r;
            }
        }

        c.coat_e = T(0);
        c.coat_scale = T(1);
        V3<T> coat_atten(T(1));
        if (m.coat_weight > T(0) && !exiting) {
            c.coat_e = dielectric_albedo(t, coat_rough, mu, m.coat_ior);
            T fss_coat = fresnel_dielectric_average(m.coat_ior);
            c.coat_scale = reflection_scale(t, coat_rough, mu, V3<T>(fss_coat)).x;
            coat_atten = lerp(V3<T>(T(1)), m.coat_color * (T(1) - c.coat_e), m.coat_weight) *
                         coat_darkening(m, rough, mu, f0);
        }
        c.base_weight = c.fuzz_atten * coat_atten;

        c.spec_e = c.has_specular ? dielectric_albedo(t, rough, mu, c.eta) : T(0);
        c.conductor_scale = reflection_scale(t, rough, mu, fresnel_schlick_average(m.base_color));
        c.dielectric_scale = reflection_scale(t, rough, mu, V3<T>(fresnel_dielectric_average(c.eta))).x;

        c.glass_tint = m.transmission_depth == T(0) ? m.transmission_color : V3<T>(T(1));
        T glass_eta = c.eta;
        uint32_t glass_off = TABLE_GLASS_E, glass_avg_off = TABLE_GLASS_E_AVG;
        if (glass_eta < T(1)) {
            glass_eta = T(1) / glass_eta;
            glass_off = TABLE_GLASS_INV_E;
            glass_avg_off = TABLE_GLASS_INV_E_AVG;
        }
        T glass_z = ior_remap(glass_eta);
        T glass_e = std::max(T(1e-4), read3(t, glass_off, 16, 16, 16, rough, mu, glass_z));
        T glass_e_avg = read2(t, glass_avg_off, 16, 16, rough, glass_z);
        c.glass_scale = T(1) + fresnel_multi_scatter(c.glass_tint, glass_e_avg) * ((T(1) - glass_e) / glass_e);

        c.thin_r = V3<T>(T(0));
        c.thin_t = V3<T>(T(0));
        c.thin_alpha = c.alpha;
        c.thin_scale_r = T(1);
        c.thin_scale_t = T(1);
        c.thin_t_share = T(0);
        bool thin = m.thin_walled != 0 && m.transmission_weight > T(0);
        if (thin) {
            T thin_eta = std::max(eta, T(1) / eta);
            T r1 = fresnel_dielectric(thin_eta, mu);
            T t1 = T(1) - r1;
            T cos2t = std::max(T(0), T(1) - (T(1) - mu * mu) / (thin_eta * thin_eta));
            V3<T> absorb = cos2t > T(0) ? vpow(vclamp(m.transmission_color, T(1e-4), T(1)),
                                               V3<T>(T(1) / std::sqrt(cos2t)))
                                        : V3<T>(T(0));
            V3<T> denom = vmax(V3<T>(T(1e-4)), T(1) - absorb * absorb * (r1 * r1));
            c.thin_t = absorb * (t1 * t1) / denom;
            c.thin_r = r1 + c.thin_t * (r1 * absorb);
            T thin_rough = clampv(rough * std::sqrt(T(3.4) * (thin_eta - T(1)) * (thin_eta - T(0.5)) *
                                                    (thin_eta - T(0.5)) / (thin_eta * thin_eta * thin_eta)),
                                  MIN_SPECULAR_ROUGHNESS, T(1));
            c.thin_alpha = thin_rough * thin_rough;
            c.thin_scale_r = reflection_scale(t, rough, mu, V3<T>(T(1))).x;
            c.thin_scale_t = reflection_scale(t, thin_rough, mu, V3<T>(T(1))).x;
            T total = average(c.thin_r) + average(c.thin_t);
            c.thin_t_share = total > T(0) ? average(c.thin_t) / total : T(0);
        }

        T schlick_s = saturate((c.spec_e - f0) / std::max(T(1e-4), T(1) - f0));
        V3<T> metal_e = lerp(m.base_color, V3<T>(T(1)), schlick_s);
        T glass_total = thin ? average(c.thin_r + c.thin_t)
                             : c.spec_e + (T(1) - c.spec_e) * average(c.glass_tint);
        T dielectric_e = lerp(c.spec_e, glass_total, m.transmission_weight);
        T base_avg = average(c.base_weight);
        c.w_fuzz = exiting ? T(0) : m.fuzz_weight * c.fuzz_r * average(m.fuzz_color);
        c.w_coat = exiting ? T(0) : c.fuzz_atten * m.coat_weight * c.coat_e;
        c.w_spec = c.has_specular ? base_avg * lerp(dielectric_e, average(metal_e), m.metalness) : T(0);
        c.w_diffuse = exiting ? T(0)
                              : base_avg * (T(1) - m.metalness) * (T(1) - m.transmission_weight) *
                                    (T(1) - c.spec_e) * average(m.base_color);
        if (exiting) c.w_spec = T(1);
        c.w_total = c.w_fuzz + c.w_coat + c.w_spec + c.w_diffuse;

        V3<T> glass_color = thin ? c.thin_r + c.thin_t : V3<T>(c.spec_e) + (T(1) - c.spec_e) * c.glass_tint;
        if (exiting) {
            c.aov_albedo = glass_color;
        } else {
            V3<T> dielectric_color = lerp(V3<T>(c.spec_e), glass_color, m.transmission_weight);
            V3<T> spec_color = c.has_specular ? lerp(dielectric_color, metal_e, m.metalness) : V3<T>(T(0));
            c.aov_albedo = m.fuzz_weight * c.fuzz_r * m.fuzz_color +
                           V3<T>(c.fuzz_atten * m.coat_weight * c.coat_e) +
                           c.base_weight * (spec_color + (T(1) - m.metalness) * (T(1) - m.transmission_weight) *
                                                             (T(1) - c.spec_e) * m.base_color);
        }
        return c;
    }

    static T aov_record_fraction(const Closure& c, uint32_t lobe) {  // :596-608
        T alpha;
        if (lobe == LOBE_COAT) alpha = c.coat_alpha;
        else if (lobe == LOBE_SPECULAR) alpha = c.alpha;
        else if (lobe == LOBE_TRANSMISSION) alpha = c.m.thin_walled != 0 ? c.thin_alpha : c.alpha;
        else return T(1);
        return saturate(std::sqrt(alpha) / T(0.15));
    }
    static V3<T> aov_pass_tint(const Closure& c, uint32_t lobe) {  // :614-622
        if (lobe == LOBE_TRANSMISSION) return c.glass_tint;
        if (lobe == LOBE_SPECULAR) return lerp(V3<T>(T(1)), c.m.base_color, c.m.metalness);
        return V3<T>(T(1));
    }

    static T sheen_density(const Closure& c, V3<T> w) {  // :629-636
        T a = c.fuzz_a, b = c.fuzz_b;
        T len_sqr = (a * w.x + b * w.z) * (a * w.x + b * w.z) + (a * w.y) * (a * w.y) + w.z * w.z;
        T ratio = a / len_sqr;
        return std::max(w.z, T(0)) * ratio * ratio / PI;
    }
    static V3<T> align_to_view(V3<T> v, V3<T> wo, bool inverse) {  // :639-647
        T len = std::sqrt(wo.x * wo.x + wo.y * wo.y);
        if (len < T(1e-6)) return v;
        T cos_phi = wo.x / len;
        T sin_phi = (inverse ? -wo.y : wo.y) / len;
        return {cos_phi * v.x + sin_phi * v.y, cos_phi * v.y - sin_phi * v.x, v.z};
    }
    static T reflection_core(T alpha, V3<T> wi, V3<T> wo, V3<T> h) {  // :650-653
        return ggx_d(alpha, h.z) * smith_g1(alpha, wo.z) * smith_g1(alpha, wi.z) / (T(4) * wo.z * wi.z);
    }
    static V3<T> base_reflection(const Closure& c, V3<T> wi, V3<T> wo, V3<T> h) {  // :660-677
        T core = reflection_core(c.alpha, wi, wo, h);
        T cos_vh = dot(h, wo);
        T fd = fresnel_dielectric(c.eta, cos_vh);
        if (c.exiting) return core * fd * c.glass_scale;
        V3<T> conductor = fresnel_schlick(c.m.base_color, cos_vh) * c.conductor_scale;
        V3<T> dielectric = lerp(V3<T>(fd * c.dielectric_scale), fd * c.glass_scale, c.m.transmission_weight);
        if (c.m.thin_walled != 0)
            dielectric = lerp(V3<T>(fd * c.dielectric_scale), c.thin_r * c.thin_scale_r, c.m.transmission_weight);
        return core * lerp(dielectric, conductor, c.m.metalness);
    }

    static V3<T> eval(const Closure& c, V3<T> wi, V3<T> wo) {  // :681-744
        if (wo.z <= T(0) || wi.z == T(0)) return V3<T>(T(0));
        const MaterialT<T>& m = c.m;
        if (wi.z < T(0)) {
            T glass_share = c.exiting ? T(1) : (T(1) - m.metalness) * m.transmission_weight;
            if (glass_share <= T(0) || (c.exiting && m.thin_walled != 0)) return V3<T>(T(0));
            if (m.thin_walled != 0) {
                V3<T> flipped(wi.x, wi.y, -wi.z);
                V3<T> h = normalize(flipped + wo);
                T core = reflection_core(c.thin_alpha, flipped, wo, h);
                return c.base_weight * glass_share * c.thin_t * c.thin_scale_t * core;
            }
            V3<T> hu = wo + c.eta * wi;
            T len2 = dot(hu, hu);
            if (len2 < T(1e-9)) return V3<T>(T(0));
            V3<T> h = hu / std::sqrt(len2);
            h = h.z >= T(0) ? h : -h;
            T cos_vh = dot(h, wo);
            T cos_lh = dot(h, wi);
            if (cos_vh <= T(0) || cos_lh >= T(0)) return V3<T>(T(0));
            T f = fresnel_dielectric(c.eta, cos_vh);
            T core = ggx_d(c.alpha, h.z) * smith_g1(c.alpha, wo.z) * smith_g1(c.alpha, wi.z) * cos_vh *
                     (c.eta * c.eta) * std::fabs(cos_lh) / (wo.z * std::fabs(wi.z) * len2);
            return c.base_weight * glass_share * (T(1) - f) * c.glass_tint * c.glass_scale * core;
        }
        V3<T> result(T(0));
        if (c.fuzz_r > T(0)) {
            T density = sheen_density(c, align_to_view(wi, wo, false));
            result = result + m.fuzz_weight * m.fuzz_color * c.fuzz_r * density / wi.z;
        }
        V3<T> h = normalize(wi + wo);
        if (m.coat_weight > T(0) && !c.exiting) {
            T coat_f = fresnel_dielectric(m.coat_ior, dot(h, wo));
            result = result + V3<T>(c.fuzz_atten * m.coat_weight * coat_f * c.coat_scale *
                                    reflection_core(c.coat_alpha, wi, wo, h));
        }
        V3<T> base(T(0));
        if (c.has_specular) base = base_reflection(c, wi, wo, h);
        if (!c.exiting)
            base = base + (T(1) - m.metalness) * (T(1) - m.transmission_weight) * (T(1) - c.spec_e) *
                              eon_brdf(m.base_color, m.base_roughness, wi, wo);
        return result + c.base_weight * base;
    }

    static T reflect_probability(const Closure& c, T fresnel) {  // :748-752
        T glass_share = c.exiting ? T(1) : (T(1) - c.m.metalness) * c.m.transmission_weight;
        T transmit = c.m.thin_walled != 0 ? c.thin_t_share : T(1) - fresnel;
        return T(1) - glass_share * transmit;
    }

    static T pdf(const Closure& c, V3<T> wi, V3<T> wo) {  // :756-808
        if (wo.z <= T(0) || wi.z == T(0) || c.w_total <= T(0)) return T(0);
        if (wi.z < T(0)) {
            if (c.w_spec <= T(0)) return T(0);
            T p = T(0);
            if (c.m.thin_walled != 0) {
                V3<T> flipped(wi.x, wi.y, -wi.z);
                V3<T> h = normalize(flipped + wo);
                p = vndf_reflect_pdf(c.thin_alpha, wo, h) * (T(1) - reflect_probability(c, T(0)));
            } else {
                V3<T> hu = wo + c.eta * wi;
                T len2 = dot(hu, hu);
                if (len2 < T(1e-9)) return T(0);
                V3<T> h = hu / std::sqrt(len2);
                h = h.z >= T(0) ? h : -h;
                T cos_vh = dot(h, wo);
                T cos_lh = dot(h, wi);
                if (cos_vh <= T(0) || cos_lh >= T(0)) return T(0);
                T f = fresnel_dielectric(c.eta, cos_vh);
                T vndf = smith_g1(c.alpha, wo.z) * ggx_d(c.alpha, h.z) * cos_vh / wo.z;
                T jac = (c.eta * c.eta) * std::fabs(cos_lh) / len2;
                p = vndf * jac * (T(1) - reflect_probability(c, f));
            }
            return c.w_spec * p / c.w_total;
        }
        V3<T> h = normalize(wi + wo);
        T p = T(0);
        if (c.w_fuzz > T(0)) p += c.w_fuzz * sheen_density(c, align_to_view(wi, wo, false));
        if (c.w_coat > T(0)) p += c.w_coat * vndf_reflect_pdf(c.coat_alpha, wo, h);
        if (c.w_spec > T(0)) {
            T f = fresnel_dielectric(c.eta, dot(h, wo));
            p += c.w_spec * vndf_reflect_pdf(c.alpha, wo, h) * reflect_probability(c, f);
        }
        if (c.w_diffuse > T(0)) p += c.w_diffuse * wi.z / PI;
        return p / c.w_total;
    }

    struct Sample {
        V3<T> wi;
        T pdf;
        uint32_t lobe;
    };

    static Sample sample(const Closure& c, V3<T> wo, T u_lobe, T ux, T uy) {  // :821-884
        Sample r;
        r.wi = V3<T>(T(0), T(0), T(1));
        r.pdf = T(0);
        r.lobe = LOBE_DIFFUSE;
        if (c.w_total <= T(0)) return r;
        T pick = u_lobe * c.w_total;
        V3<T> wi(T(0));
        if (pick < c.w_fuzz) {
            r.lobe = LOBE_FUZZ;
            T rr = std::sqrt(ux);
            T phi = T(2) * PI * uy;
            T dx = rr * std::cos(phi), dy = rr * std::sin(phi);
            T dz = std::sqrt(std::max(T(0), T(1) - (dx * dx + dy * dy)));
            V3<T> wi_std = normalize(V3<T>(dx - dz * c.fuzz_b, dy, dz * c.fuzz_a));
            wi = align_to_view(wi_std, wo, true);
        } else if (pick < c.w_fuzz + c.w_coat) {
            r.lobe = LOBE_COAT;
            V3<T> h = sample_vndf(wo, c.coat_alpha, ux, uy);
            wi = T(2) * dot(wo, h) * h - wo;
        } else if (pick < c.w_fuzz + c.w_coat + c.w_spec) {
            T u_branch = (pick - c.w_fuzz - c.w_coat) / std::max(T(1e-6), c.w_spec);
            if (c.m.thin_walled != 0) {
                if (u_branch < reflect_probability(c, T(0))) {
                    r.lobe = LOBE_SPECULAR;
                    V3<T> h = sample_vndf(wo, c.alpha, ux, uy);
                    wi = T(2) * dot(wo, h) * h - wo;
                } else {
                    r.lobe = LOBE_TRANSMISSION;
                    V3<T> h = sample_vndf(wo, c.thin_alpha, ux, uy);
                    V3<T> refl = T(2) * dot(wo, h) * h - wo;
                    wi = V3<T>(refl.x, refl.y, -refl.z);
                }
            } else {
                V3<T> h = sample_vndf(wo, c.alpha, ux, uy);
                T f = fresnel_dielectric(c.eta, dot(h, wo));
                if (u_branch < reflect_probability(c, f)) {
                    r.lobe = LOBE_SPECULAR;
                    wi = T(2) * dot(wo, h) * h - wo;
                } else {
                    r.lobe = LOBE_TRANSMISSION;
                    V3<T> refr;
                    if (!refract_direction(wo, h, c.eta, &refr)) return r;
                    wi = refr;
                }
            }
        } else {
            r.lobe = LOBE_DIFFUSE;
            T p;
            wi = sample_cosine_hemisphere(ux, uy, &p);
        }
        r.wi = wi;
        r.pdf = pdf(c, wi, wo);
        return r;
    }
};

// Duff et al. orthonormal frame, openpbr.slang:888-909.
template <class T>
struct Frame {
    V3<T> t, b, n;
    explicit Frame(V3<T> nn) : n(nn) {
        T s = nn.z >= T(0) ? T(1) : T(-1);
        T a = T(-1) / (s + nn.z);
        T m = nn.x * nn.y * a;
        t = V3<T>(T(1) + s * nn.x * nn.x * a, s * m, -s * nn.x);
        b = V3<T>(m, s + nn.y * nn.y * a, -nn.y);
    }
    V3<T> to_local(V3<T> v) const { return {dot(v, t), dot(v, b), dot(v, n)}; }
    V3<T> to_world(V3<T> v) const { return v.x * t + v.y * b + v.z * n; }
};

template <class T>
inline T power_heuristic(T p, T q) {  // lights.slang:42-44
    return (p * p) / (p * p + q * q);
}

}  // namespace oracle
