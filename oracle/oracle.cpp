// Test infrastructure (CPU oracle): scene assembly and the per-pixel path
// tracer that restates cenote's wavefront stage by stage, plus the C entry
// points the Python tests call through ctypes. It is the checker and the
// timed CPU baseline; the shipped library never links or calls it.
//
// Stage order per bounce follows crates/cenote/src/wavefront.rs:727-828:
// intersect → shade_miss | shade_surface → trace_shadow, with the pixel's
// radiance adds in that order, so an FP32 oracle render and a kernel render
// of the same (pixel, sample) take the same path unless rounding diverges.
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "lights_env.h"
#include "openpbr.h"
#include "rng.h"
#include "textures.h"
#include "trace.h"

using namespace oracle;

namespace {

constexpr uint32_t MEDIUM_NONE = 0xffffff;     // pathstate.slang:188
constexpr uint32_t RAY_MASK_CAMERA = 0x01;     // scene/mod.rs:54-57
constexpr uint32_t RAY_MASK_ALL = 0xff;
constexpr uint32_t TRANSPARENT_CAP = 8;        // intersect.slang:199
constexpr uint32_t ROULETTE_START = 3;         // shade_surface.slang:53

using BF = BSDF<float>;
using V4 = float[4];

struct Instance {
    float o2w[3][4];
    float w2o[3][4];
    std::vector<float> positions, normals, uvs;
    std::vector<uint32_t> indices;
    Material material;
    uint32_t light = LIGHT_NONE;  // first light record of an emissive instance
    bool camera_visible = true;
};

struct Scene {
    std::vector<Instance> inst;
    std::vector<LightRecord> lights;
    uint32_t light_count = 0;
    EnvTables env;
    float select_prob = 0.0f;
    Bvh bvh;
    std::vector<float> tables;
    V3f cam_pos, cam_look, cam_upv;       // Camera (scene/mod.rs:392-407)
    V3f cam_right, cam_up, cam_fwd;       // basis for the current target, scene/mod.rs:448-460
    float vfov = 40.0f, aperture = 0.0f, focus = 1.0f;
    std::vector<Texture> textures;  // the bindless table, material slot order
};

// glam's Mat4::transform_point3 on the top three rows: ((x·p.x + y·p.y) + z·p.z) + w.
V3f transform_point(const float m[3][4], V3f p) {
    return {m[0][0] * p.x + m[0][1] * p.y + m[0][2] * p.z + m[0][3],
            m[1][0] * p.x + m[1][1] * p.y + m[1][2] * p.z + m[1][3],
            m[2][0] * p.x + m[2][1] * p.y + m[2][2] * p.z + m[2][3]};
}

// Inverse of an affine 3×4 in double, rounded to f32.
void invert_affine(const float m[3][4], float out[3][4]) {
    double a[3][3], t[3];
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) a[r][c] = m[r][c];
        t[r] = m[r][3];
    }
    double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
                 a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                 a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    double inv[3][3];
    inv[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) / det;
    inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
    inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
    inv[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) / det;
    inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
    inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
    inv[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) / det;
    inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
    inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) out[r][c] = float(inv[r][c]);
        out[r][3] = float(-(inv[r][0] * t[0] + inv[r][1] * t[1] + inv[r][2] * t[2]));
    }
}

V3f mat_color(const float* f) { return {f[0], f[1], f[2]}; }

// ---- textures (textures.slang:24-82, scene.slang:31-64) ---------------------

struct F2v {
    float x, y;
};

F2v interpolate_uv(const Instance& m, uint32_t prim, float b1, float b2) {
    const float* uv0 = &m.uvs[2 * m.indices[3 * prim]];
    const float* uv1 = &m.uvs[2 * m.indices[3 * prim + 1]];
    const float* uv2 = &m.uvs[2 * m.indices[3 * prim + 2]];
    return {uv0[0] + b1 * (uv1[0] - uv0[0]) + b2 * (uv2[0] - uv0[0]),
            uv0[1] + b1 * (uv1[1] - uv0[1]) + b2 * (uv2[1] - uv0[1])};
}

void sample_texture(const Scene& s, uint32_t index, F2v uv, float out[4]) { s.textures[index].sample(uv.x, uv.y, out); }

// Linear Rec.709 -> ACEScg, rows-dot-vector (textures.slang:37-45).
V3f sample_color(const Scene& s, uint32_t index, F2v uv) {
    float t[4];
    sample_texture(s, index, uv, t);
    return {0.613097400f * t[0] + 0.339523140f * t[1] + 0.047379450f * t[2],
            0.070193730f * t[0] + 0.916353900f * t[1] + 0.013452399f * t[2],
            0.020615594f * t[0] + 0.109569780f * t[1] + 0.869814660f * t[2]};
}

float sample_scalar(const Scene& s, uint32_t index, F2v uv) {
    float t[4];
    sample_texture(s, index, uv, t);
    return t[0];
}

V3f sample_normal(const Scene& s, uint32_t index, F2v uv) {
    float t[4];
    sample_texture(s, index, uv, t);
    float x = t[0] * 2.0f - 1.0f, y = t[1] * 2.0f - 1.0f;
    return {x, y, std::sqrt(std::max(1.0f - (x * x + y * y), 0.0f))};
}

bool textured(const Material& m) {
    return m.base_color_texture != TEXTURE_NONE || m.specular_roughness_texture != TEXTURE_NONE ||
           m.metalness_texture != TEXTURE_NONE || m.emission_texture != TEXTURE_NONE;
}

Material resolve_material(const Scene& s, Material m, F2v uv) {  // textures.slang:70-82
    if (m.base_color_texture != TEXTURE_NONE) wr3(m.base_color, sample_color(s, m.base_color_texture, uv));
    if (m.specular_roughness_texture != TEXTURE_NONE)
        m.specular_roughness = sample_scalar(s, m.specular_roughness_texture, uv);
    if (m.metalness_texture != TEXTURE_NONE) m.metalness = sample_scalar(s, m.metalness_texture, uv);
    if (m.emission_texture != TEXTURE_NONE)
        wr3(m.emission, mat_color(m.emission) * sample_color(s, m.emission_texture, uv));
    return m;
}

float opacity_at(const Scene& s, uint32_t inst, uint32_t prim, float b1, float b2) {  // scene.slang:56-64
    const Instance& in = s.inst[inst];
    float opacity = in.material.opacity;
    if (in.material.opacity_texture != TEXTURE_NONE)
        opacity *= sample_scalar(s, in.material.opacity_texture, interpolate_uv(in, prim, b1, b2));
    return opacity;
}

// ---- kernels, restated ----------------------------------------------------

struct Hit {
    uint32_t instance, primitive;
    float b1, b2;
};

// Closest committed hit with stochastic opacity (intersect.slang:47-88).
bool intersect(const Scene& s, V3f org, V3f dir, uint32_t mask, uint32_t pixel, uint32_t sample,
               uint32_t bounce, Hit* hit) {
    RayPre r = ray_pre(org, dir);
    float best_t = 1e30f;
    uint64_t best_key = ~0ull;
    bool found = false;
    uint32_t crossings = 0;
    s.bvh.walk(r, 1e30f, [&](uint32_t i, float tmax) {
        const Tri& t = s.bvh.tris[i];
        if (!(t.mask & mask)) return tmax;
        float tt, b1, b2;
        if (!intersect_tri(r, t, tmax, &tt, &b1, &b2)) return tmax;
        uint64_t key = hit_key(t.instance, t.primitive);
        if (!(tt < best_t || (tt == best_t && key < best_key))) return tmax;
        if (!t.opaque) {
            float opacity = opacity_at(s, t.instance, t.primitive, b1, b2);
            bool commit = crossings >= TRANSPARENT_CAP || hash_uniform(pixel, sample, bounce, crossings) < opacity;
            crossings++;
            if (!commit) return tmax;
        }
        best_t = tt;
        best_key = key;
        hit->instance = t.instance;
        hit->primitive = t.primitive;
        hit->b1 = b1;
        hit->b2 = b2;
        found = true;
        return tt;
    });
    return found;
}

// trace_shadow.slang:29-72: closest hit by identity, multiplicative
// attenuation through fractional-opacity occluders. Returns the attenuation,
// or -1 when the connection is occluded.
float trace_shadow(const Scene& s, V3f org, V3f dir, float tmax, uint32_t light, uint32_t prim) {
    RayPre r = ray_pre(org, dir);
    float best_t = 1e30f;
    uint64_t best_key = ~0ull;
    bool found = false;
    uint32_t committed_inst = 0, committed_prim = 0;
    float atten = 1.0f;
    bool dead = false;
    s.bvh.walk(r, tmax, [&](uint32_t i, float tm) {
        if (dead) return -1.0f;
        const Tri& t = s.bvh.tris[i];
        float tt, b1, b2;
        if (!intersect_tri(r, t, tm, &tt, &b1, &b2)) return tm;
        uint64_t key = hit_key(t.instance, t.primitive);
        if (!(tt < best_t || (tt == best_t && key < best_key))) return tm;
        bool target = t.instance == light && t.primitive == prim;
        if (!t.opaque && !target) {
            atten *= 1.0f - opacity_at(s, t.instance, t.primitive, b1, b2);
            if (atten < 1e-4f) { dead = true; return -1.0f; }
            return tm;
        }
        best_t = tt;
        best_key = key;
        committed_inst = t.instance;
        committed_prim = t.primitive;
        found = true;
        return tt;
    });
    if (dead) return -1.0f;
    if (!found || (committed_inst == light && committed_prim == prim)) return atten;
    return -1.0f;
}

V3f fetch3(const std::vector<float>& a, uint32_t v) { return {a[3 * v], a[3 * v + 1], a[3 * v + 2]}; }

struct Spawn {
    V3f position, below, normal, shading;
    bool front_face;
};

// shade_surface.slang:96-181 (van Antwerpen's offsets).
Spawn spawn_point(const Instance& m, const Hit& hit, V3f ray_dir) {
    uint32_t base = 3 * hit.primitive;
    V3f v0 = fetch3(m.positions, m.indices[base]);
    V3f v1 = fetch3(m.positions, m.indices[base + 1]);
    V3f v2 = fetch3(m.positions, m.indices[base + 2]);
    const auto& o2w = m.o2w;
    const auto& w2o = m.w2o;
    V3f e1 = v1 - v0, e2 = v2 - v0;
    V3f obj_p = v0 + vfma(V3f(hit.b1), e1, hit.b2 * e2);
    V3f obj_n = cross(e1, e2);
    V3f wp(o2w[0][3] + std::fma(o2w[0][0], obj_p.x, std::fma(o2w[0][1], obj_p.y, o2w[0][2] * obj_p.z)),
           o2w[1][3] + std::fma(o2w[1][0], obj_p.x, std::fma(o2w[1][1], obj_p.y, o2w[1][2] * obj_p.z)),
           o2w[2][3] + std::fma(o2w[2][0], obj_p.x, std::fma(o2w[2][1], obj_p.y, o2w[2][2] * obj_p.z)));
    V3f r0(w2o[0][0], w2o[0][1], w2o[0][2]), r1(w2o[1][0], w2o[1][1], w2o[1][2]), r2(w2o[2][0], w2o[2][1], w2o[2][2]);
    V3f wn = r0 * obj_n.x + r1 * obj_n.y + r2 * obj_n.z;
    float wscale = 1.0f / std::sqrt(dot(wn, wn));
    wn = wn * wscale;
    const float c0 = 5.9604644775390625e-8f;
    const float c1 = 1.788139769587360206060111522674560546875e-7f;
    const float c2 = 1.19209317972490680404007434844970703125e-7f;
    V3f ext3 = vabs(e1) + vabs(e2) + vabs(e1 - e2);
    float extent = std::max(std::max(ext3.x, ext3.y), ext3.z);
    V3f obj_err = vfma(V3f(c0), vabs(v0), V3f(c1 * extent));
    V3f o0(o2w[0][0], o2w[0][1], o2w[0][2]), o1(o2w[1][0], o2w[1][1], o2w[1][2]), o2(o2w[2][0], o2w[2][1], o2w[2][2]);
    V3f ap = vabs(obj_p);
    V3f wld_err = vfma(V3f(c1), V3f(dot(vabs(o0), ap), dot(vabs(o1), ap), dot(vabs(o2), ap)),
                       c2 * vabs(V3f(o2w[0][3], o2w[1][3], o2w[2][3])));
    V3f awp = vabs(wp);
    obj_err = vfma(V3f(c2),
                   V3f(dot(vabs(r0), awp) + std::fabs(w2o[0][3]), dot(vabs(r1), awp) + std::fabs(w2o[1][3]),
                       dot(vabs(r2), awp) + std::fabs(w2o[2][3])),
                   obj_err);
    float wld_off = dot(wld_err, vabs(wn));
    float obj_off = dot(obj_err, vabs(obj_n));
    wld_off = std::fma(wscale, obj_off, wld_off);
    Spawn sp;
    sp.front_face = dot(wn, ray_dir) < 0.0f;
    if (dot(wn, ray_dir) > 0.0f) wn = -wn;
    V3f n0 = fetch3(m.normals, m.indices[base]);
    V3f n1 = fetch3(m.normals, m.indices[base + 1]);
    V3f n2 = fetch3(m.normals, m.indices[base + 2]);
    V3f obj_s = n0 + hit.b1 * (n1 - n0) + hit.b2 * (n2 - n0);
    V3f sh = normalize(r0 * obj_s.x + r1 * obj_s.y + r2 * obj_s.z);
    if (dot(sh, wn) < 0.0f) sh = -sh;
    sp.position = vfma(V3f(wld_off), wn, wp);
    sp.below = vfma(V3f(-wld_off), wn, wp);
    sp.normal = wn;
    sp.shading = sh;
    return sp;
}

// shade_surface.slang:183-231: the shading normal under a tangent-space
// normal map, tangent frame from the triangle's positions and UVs.
V3f mapped_shading_normal(const Scene& s, const Instance& m, const Hit& hit, F2v uv, uint32_t map,
                          const Spawn& sp) {
    uint32_t base = 3 * hit.primitive;
    uint32_t i0 = m.indices[base], i1 = m.indices[base + 1], i2 = m.indices[base + 2];
    float du1 = m.uvs[2 * i1] - m.uvs[2 * i0], dv1 = m.uvs[2 * i1 + 1] - m.uvs[2 * i0 + 1];
    float du2 = m.uvs[2 * i2] - m.uvs[2 * i0], dv2 = m.uvs[2 * i2 + 1] - m.uvs[2 * i0 + 1];
    float det = du1 * dv2 - dv1 * du2;
    if (std::fabs(det) < 1e-12f) return sp.shading;
    V3f e1 = fetch3(m.positions, i1) - fetch3(m.positions, i0);
    V3f e2 = fetch3(m.positions, i2) - fetch3(m.positions, i0);
    const auto& o = m.o2w;
    V3f we1(dot(V3f(o[0][0], o[0][1], o[0][2]), e1), dot(V3f(o[1][0], o[1][1], o[1][2]), e1),
            dot(V3f(o[2][0], o[2][1], o[2][2]), e1));
    V3f we2(dot(V3f(o[0][0], o[0][1], o[0][2]), e2), dot(V3f(o[1][0], o[1][1], o[1][2]), e2),
            dot(V3f(o[2][0], o[2][1], o[2][2]), e2));
    V3f dpdu = (dv2 * we1 - dv1 * we2) / det;
    V3f dpdv = (du1 * we2 - du2 * we1) / det;
    V3f tangent = dpdu - sp.shading * dot(sp.shading, dpdu);
    float len2 = dot(tangent, tangent);
    if (!(len2 > 1e-20f)) return sp.shading;
    tangent = tangent * (1.0f / std::sqrt(len2));
    V3f bitangent = cross(sp.shading, tangent);
    if (dot(bitangent, dpdv) < 0.0f) bitangent = -bitangent;
    V3f t = sample_normal(s, map, uv);
    V3f mapped = normalize(t.x * tangent + t.y * bitangent + t.z * sp.shading);
    if (dot(mapped, sp.normal) < 0.0f) mapped = -mapped;
    return mapped;
}

// raygen.slang:47-62
void concentric_disk(float ux, float uy, float* dx, float* dy) {
    float ox = 2.0f * ux - 1.0f, oy = 2.0f * uy - 1.0f;
    if (ox == 0.0f && oy == 0.0f) { *dx = *dy = 0.0f; return; }
    float r, theta;
    if (std::fabs(ox) > std::fabs(oy)) {
        r = ox;
        theta = (PI_F / 4.0f) * (oy / ox);
    } else {
        r = oy;
        theta = (PI_F / 2.0f) - (PI_F / 4.0f) * (ox / oy);
    }
    *dx = r * std::cos(theta);
    *dy = r * std::sin(theta);
}

struct RayCounts {
    uint64_t extension = 0, shadow = 0;
};

// One sample's denoiser guides (pathstate.slang:82-106): albedo and normal
// (xyz), camera-plane depth of the first hit (+inf on a miss).
struct Guides {
    float albedo[4] = {0, 0, 0, 0};
    float normal[4] = {0, 0, 0, 0};
    float depth = 0.0f;
    void record(V3f w, V3f a, V3f n) {  // shade_surface.slang:59-63
        albedo[0] += w.x * a.x; albedo[1] += w.y * a.y; albedo[2] += w.z * a.z;
        normal[0] += w.x * n.x; normal[1] += w.y * n.y; normal[2] += w.z * n.z;
    }
};

// One sample of one pixel: raygen, then the bounce loop. Returns RGBA.
void trace_path(const Scene& s, uint32_t width, uint32_t height, uint32_t pixel, uint32_t sample,
                uint32_t max_bounces, uint32_t light_sampling, float out[4], RayCounts& counts,
                Guides* aov = nullptr) {
    float rad[4] = {0, 0, 0, 0};
    // raygen.slang:66-112 with the basis of wavefront.rs:633-675
    V3f right = s.cam_right, up = s.cam_up, fwd = s.cam_fwd;
    if (s.aperture > 0.0f) {
        right = right * s.focus;
        up = up * s.focus;
        fwd = fwd * s.focus;
    }
    F2 jit = sample_2d(pixel, sample, CAMERA_JITTER);
    float xyx = float(pixel % width) + jit.x, xyy = float(pixel / width) + jit.y;
    float uvx = xyx / float(width), uvy = xyy / float(height);
    float ndcx = 2.0f * uvx - 1.0f, ndcy = 1.0f - 2.0f * uvy;
    V3f target = fwd + ndcx * right + ndcy * up;
    V3f origin = s.cam_pos;
    V3f dir = normalize(target);
    if (s.aperture > 0.0f) {
        F2 ul = sample_2d(pixel, sample, CAMERA_LENS);
        float dx, dy;
        concentric_disk(ul.x, ul.y, &dx, &dy);
        dx *= s.aperture;
        dy *= s.aperture;
        V3f off = dx * normalize(right) + dy * normalize(up);
        origin = origin + off;
        dir = normalize(target - off);
    }
    // ORACLE_ULP_NUDGE (sensitivity experiments only): 1 moves every camera
    // ray's direction by one ulp in x, 2 every ray's, the size of the
    // rounding differences between two correct FP32 implementations.
    static const int nudge = std::getenv("ORACLE_ULP_NUDGE") ? std::atoi(std::getenv("ORACLE_ULP_NUDGE")) : 0;
    if (nudge == 1) dir.x = std::nextafter(dir.x, 2.0f);
    float dir_w = dot(dir, normalize(fwd));
    V3f guide(1.0f);  // the open feature throughput; a camera ray's is 1
    V3f thr(1.0f);
    float thr_w = 0.0f;
    uint32_t medium = MEDIUM_NONE;

    const float* tables = s.tables.data();
    for (uint32_t bounce = 0; bounce < max_bounces; ++bounce) {
        Hit hit;
        counts.extension++;
        if (nudge == 2) dir.x = std::nextafter(dir.x, 2.0f);
        bool found = intersect(s, origin, dir, bounce == 0 ? RAY_MASK_CAMERA : RAY_MASK_ALL, pixel, sample,
                               bounce, &hit);
        if (!found) {  // shade_miss.slang:29-75
            float weight = 1.0f;
            if (thr_w > 0.0f) {
                if (light_sampling == LIGHT_SAMPLING_NEE) weight = 0.0f;
                else if (light_sampling == LIGHT_SAMPLING_MIS)
                    weight = power_heuristic(thr_w, s.select_prob * env_pdf(s.env, dir));
            }
            if (aov) {  // shade_miss.slang:52-66
                if (thr_w == 0.0f) aov->depth += INFINITY;
                aov->albedo[0] += guide.x; aov->albedo[1] += guide.y; aov->albedo[2] += guide.z;
            }
            V3f c = thr * env_radiance(s.env, dir) * weight;
            rad[0] += c.x; rad[1] += c.y; rad[2] += c.z; rad[3] += 1.0f;
            break;
        }
        // shade_surface.slang:235-521
        const Instance& mesh = s.inst[hit.instance];
        F2v uv{0.0f, 0.0f};
        const bool maps = textured(mesh.material) || mesh.material.normal_texture != TEXTURE_NONE;
        if (maps) uv = interpolate_uv(mesh, hit.primitive, hit.b1, hit.b2);
        const Material mat = textured(mesh.material) ? resolve_material(s, mesh.material, uv) : mesh.material;
        Spawn spawn = spawn_point(mesh, hit, dir);
        if (medium != MEDIUM_NONE) {
            const Material& interior = s.inst[medium].material;
            if (interior.transmission_depth > 0.0f) {
                V3f sigma = -vlog(vclamp(mat_color(interior.transmission_color), 1e-4f, 1.0f)) /
                            interior.transmission_depth;
                thr = thr * vexp(-sigma * length(origin - spawn.position));
            }
        }
        V3f contribution(0.0f);
        if (mesh.light != LIGHT_NONE && spawn.front_face) {
            float weight = 1.0f;
            if (thr_w > 0.0f) {
                if (light_sampling == LIGHT_SAMPLING_NEE) weight = 0.0f;
                else if (light_sampling == LIGHT_SAMPLING_MIS) {
                    V3f delta = spawn.position - origin;
                    float cos_light = std::fabs(dot(spawn.normal, dir));
                    float nee_pdf = (1.0f - s.select_prob) * s.lights[mesh.light + hit.primitive].pdf *
                                    dot(delta, delta) / cos_light;
                    weight = power_heuristic(thr_w, nee_pdf);
                }
            }
            contribution = thr * mat_color(mat.emission) * weight;
        }
        V3f shading = spawn.shading;
        if (mat.normal_texture != TEXTURE_NONE)
            shading = mapped_shading_normal(s, mesh, hit, uv, mat.normal_texture, spawn);
        Frame<float> frame(shading);
        V3f wo = frame.to_local(-dir);
        MaterialT<float> mt = to_t<float>(mat);
        BF::Closure closure = BF::resolve(tables, mt, wo, medium == hit.instance);
        V3f aov_alb(0.0f);
        if (aov) {  // shade_surface.slang:322-340
            if (bounce == 0) aov->depth += length(origin - spawn.position) * dir_w;
            aov_alb = vclamp(closure.aov_albedo, 0.0f, 1.0f);
        }
        auto record_open = [&](V3f w) {
            if (aov && any_gt0(w)) aov->record(w, aov_alb, shading);
        };

        bool shadow_live = false;
        V3f sh_org, sh_dir, sh_contrib;
        float sh_tmax = 1e30f;
        uint32_t sh_light = LIGHT_NONE, sh_prim = 0;
        bool terminal = false, cont = false;

        if (bounce + 1 >= max_bounces) {
            record_open(guide);
            rad[0] += contribution.x; rad[1] += contribution.y; rad[2] += contribution.z; rad[3] += 1.0f;
            break;
        }
        float env_prob = s.select_prob;
        if (light_sampling != LIGHT_SAMPLING_BSDF && (s.light_count > 0 || env_prob > 0.0f)) {
            float u_light = sample_1d(pixel, sample, bounce_dimension(bounce, NEE_LIGHT));
            F2 u_point = sample_2d(pixel, sample, bounce_dimension(bounce, NEE_POINT));
            V3f unshadowed(0.0f);
            if (u_light < env_prob) {
                EnvSample cand = env_sample(s.env, u_point.x, u_point.y);
                V3f wl = frame.to_local(cand.direction);
                bool through = dot(cand.direction, spawn.normal) < 0.0f;
                if (cand.pdf > 0.0f && wl.z != 0.0f && (wl.z < 0.0f) == through) {
                    float nee_pdf = env_prob * cand.pdf;
                    float scatter_pdf = BF::pdf(closure, wl, wo);
                    float w = light_sampling == LIGHT_SAMPLING_MIS ? power_heuristic(nee_pdf, scatter_pdf) : 1.0f;
                    unshadowed = thr * cand.radiance * BF::eval(closure, wl, wo) * std::fabs(wl.z) * (w / nee_pdf);
                    sh_org = through ? spawn.below : spawn.position;
                    sh_light = LIGHT_NONE;
                    sh_prim = 0;
                    sh_dir = cand.direction;
                    sh_tmax = 1e30f;
                }
            } else {
                float u_list = (u_light - env_prob) / (1.0f - env_prob);
                LightConnection cand = sample_lights(s.lights.data(), s.light_count, u_list, u_point.x,
                                                     u_point.y, spawn.position);
                if (!cand.delta) {  // a textured emitter evaluates its map at the sampled point
                    const Instance& em = s.inst[cand.instance];
                    if (em.material.emission_texture != TEXTURE_NONE)
                        cand.radiance = cand.radiance *
                                        sample_color(s, em.material.emission_texture,
                                                     interpolate_uv(em, cand.primitive, cand.bary_x, cand.bary_y));
                }
                V3f wl = frame.to_local(cand.direction);
                bool through = dot(cand.direction, spawn.normal) < 0.0f;
                if (cand.pdf > 0.0f && wl.z != 0.0f && (wl.z < 0.0f) == through) {
                    float nee_pdf = (1.0f - env_prob) * cand.pdf;
                    float w = !cand.delta && light_sampling == LIGHT_SAMPLING_MIS
                                  ? power_heuristic(nee_pdf, BF::pdf(closure, wl, wo))
                                  : 1.0f;
                    unshadowed = thr * cand.radiance * BF::eval(closure, wl, wo) * std::fabs(wl.z) * (w / nee_pdf);
                    sh_org = through ? spawn.below : spawn.position;
                    sh_light = cand.instance;
                    sh_prim = cand.primitive;
                    sh_dir = cand.direction;
                    sh_tmax = cand.tmax;
                }
            }
            if (any_gt0(unshadowed)) {
                shadow_live = true;
                sh_contrib = unshadowed;
            }
        }
        float u_lobe = sample_1d(pixel, sample, bounce_dimension(bounce, BSDF_LOBE));
        F2 u = sample_2d(pixel, sample, bounce_dimension(bounce, BSDF_DIR));
        BF::Sample sc = BF::sample(closure, wo, u_lobe, u.x, u.y);
        V3f wi_world = frame.to_world(sc.wi);
        V3f scattered(0.0f);
        if (sc.pdf > 0.0f && sc.wi.z != 0.0f && (sc.wi.z > 0.0f) == (dot(wi_world, spawn.normal) > 0.0f))
            scattered = thr * BF::eval(closure, sc.wi, wo) * (std::fabs(sc.wi.z) / sc.pdf);
        float survival = std::max(scattered.x, std::max(scattered.y, scattered.z));
        if (survival <= 0.0f) {
            terminal = true;
        } else if (bounce >= ROULETTE_START) {
            survival = std::min(1.0f, survival);
            if (sample_1d(pixel, sample, bounce_dimension(bounce, RR)) >= survival) terminal = true;
            else scattered = scattered / survival;
        }
        if (terminal) {
            record_open(guide);
            rad[0] += contribution.x; rad[1] += contribution.y; rad[2] += contribution.z; rad[3] += 1.0f;
        } else {
            if (aov) {  // shade_surface.slang:488-503
                float rec = BF::aov_record_fraction(closure, sc.lobe);
                if (rec > 0.0f) record_open(guide * rec);
                guide = guide * (1.0f - rec) * BF::aov_pass_tint(closure, sc.lobe);
            }
            if (sc.lobe == LOBE_TRANSMISSION && mat.thin_walled == 0)
                medium = medium == hit.instance ? MEDIUM_NONE : hit.instance;
            bool transmitted = sc.wi.z < 0.0f;
            origin = transmitted ? spawn.below : spawn.position;
            dir = wi_world;
            thr = scattered;
            thr_w = sc.pdf;
            cont = true;
            if (any_gt0(contribution)) {
                rad[0] += contribution.x; rad[1] += contribution.y; rad[2] += contribution.z;
            }
        }
        if (shadow_live) {
            counts.shadow++;
            float att = trace_shadow(s, sh_org, sh_dir, sh_tmax, sh_light, sh_prim);
            if (att >= 0.0f) {
                V3f c = sh_contrib * att;
                rad[0] += c.x; rad[1] += c.y; rad[2] += c.z;
            }
        }
        if (!cont) break;
    }
    for (int i = 0; i < 4; ++i) out[i] = rad[i];
}

bool finite4(const float* v) {
    for (int i = 0; i < 4; ++i)
        if (!std::isfinite(v[i])) return false;
    return true;
}

}  // namespace

// ---- C entry points -------------------------------------------------------

extern "C" {

struct oracle_object {  // mirrors cenote_object in include/cenote_c.h
    const float* positions;
    const float* normals;
    const float* uvs;
    const uint32_t* indices;
    uint32_t vertex_count;
    uint32_t triangle_count;
    float transform[12];
    Material material;
    uint32_t camera_visible;
    uint32_t pad;
};

struct oracle_camera {
    float position[3], look_at[3], up[3];
    float vfov_degrees, aperture_radius, focus_distance;
};

struct oracle_delta_light {
    uint32_t kind;
    float anchor[3];
    float emission[3];
};

void oracle_camera_basis(const oracle_camera* cam, float aspect, float* right, float* up, float* fwd);

struct oracle_texture {  // mirrors cenote_texture in include/cenote_c.h
    uint32_t format, width, height, pad;
    const void* data;
};

// Returns null when a texture cannot be decoded or a material names a slot
// past the table.
void* oracle_scene_create(const oracle_object* objects, uint32_t n, const oracle_camera* cam,
                          uint32_t env_w, uint32_t env_h, const float* env_texels,
                          const oracle_delta_light* deltas, uint32_t n_deltas, const float* bsdf_tables,
                          const oracle_texture* textures, uint32_t n_textures) {
    Scene* s = new Scene();
    s->textures.resize(n_textures);
    for (uint32_t k = 0; k < n_textures; ++k)
        if (!s->textures[k].decode(textures[k].format, textures[k].width, textures[k].height, textures[k].data)) {
            delete s;
            return nullptr;
        }
    for (uint32_t i = 0; i < n; ++i) {
        const Material& m = objects[i].material;
        for (uint32_t slot : {m.base_color_texture, m.specular_roughness_texture, m.metalness_texture,
                              m.emission_texture, m.opacity_texture, m.normal_texture})
            if (slot != TEXTURE_NONE && slot >= n_textures) {
                delete s;
                return nullptr;
            }
    }
    s->tables.assign(bsdf_tables, bsdf_tables + TABLE_FLOATS);
    std::vector<TriangleLight> tri_lights;
    std::vector<Tri> tris;
    for (uint32_t i = 0; i < n; ++i) {
        const oracle_object& o = objects[i];
        Instance in;
        std::memcpy(in.o2w, o.transform, sizeof in.o2w);
        invert_affine(in.o2w, in.w2o);
        in.positions.assign(o.positions, o.positions + 3 * o.vertex_count);
        in.normals.assign(o.normals, o.normals + 3 * o.vertex_count);
        in.uvs.assign(o.uvs, o.uvs + 2 * o.vertex_count);
        in.indices.assign(o.indices, o.indices + 3 * o.triangle_count);
        in.material = o.material;
        in.camera_visible = o.camera_visible != 0;
        V3f em = mat_color(o.material.emission);
        bool emissive = em.x != 0.0f || em.y != 0.0f || em.z != 0.0f;
        bool opaque = o.material.opacity >= 1.0f && o.material.opacity_texture == TEXTURE_NONE;
        for (uint32_t t = 0; t < o.triangle_count; ++t) {
            V3f c[3];
            for (int k = 0; k < 3; ++k) c[k] = transform_point(in.o2w, fetch3(in.positions, in.indices[3 * t + k]));
            Tri tri{c[0], c[1], c[2], i, t, in.camera_visible ? RAY_MASK_ALL : (RAY_MASK_ALL & ~RAY_MASK_CAMERA),
                    opaque ? 1u : 0u};
            tris.push_back(tri);
            if (emissive) tri_lights.push_back({{c[0], c[1], c[2]}, em, i, t});
        }
        s->inst.push_back(std::move(in));
    }
    std::vector<DeltaLight> dl;
    for (uint32_t i = 0; i < n_deltas; ++i) dl.push_back({deltas[i].kind, rd3(deltas[i].anchor), rd3(deltas[i].emission)});
    s->lights = build_lights(tri_lights, dl);
    s->light_count = uint32_t(s->lights.size());
    // GeometryRecord.light: index of the instance's first triangle record
    // (scene/mod.rs:514-519).
    for (size_t k = 0; k < tri_lights.size(); ++k) {
        Instance& in = s->inst[tri_lights[k].instance];
        if (in.light == LIGHT_NONE) in.light = uint32_t(k);
    }
    s->env.width = env_w;
    s->env.height = env_h;
    s->env.texels.assign(env_texels, env_texels + size_t(4) * env_w * env_h);
    build_env_tables(s->env);
    s->select_prob = select_probability(s->env.power, total_light_power(tri_lights, dl));
    s->bvh.build(std::move(tris));
    s->cam_pos = rd3(cam->position);
    s->cam_look = rd3(cam->look_at);
    s->cam_upv = rd3(cam->up);
    s->vfov = cam->vfov_degrees;
    s->aperture = cam->aperture_radius;
    s->focus = cam->focus_distance;
    return s;
}

// Camera::basis (scene/mod.rs:448-460) for a target aspect ratio.
void oracle_camera_basis(const oracle_camera* cam, float aspect, float* right, float* up, float* fwd) {
    V3f pos = rd3(cam->position), look = rd3(cam->look_at), upv = rd3(cam->up);
    V3f d = look - pos;
    V3f f = d * (1.0f / length(d));
    V3f c = cross(f, upv);
    V3f r = c * (1.0f / length(c));
    V3f u = cross(r, f);
    float half_h = std::tan(cam->vfov_degrees * (3.14159265358979323846f / 180.0f) / 2.0f);
    wr3(right, r * half_h * aspect);
    wr3(up, u * half_h);
    wr3(fwd, f);
}

void oracle_scene_destroy(void* p) { delete static_cast<Scene*>(p); }

uint32_t oracle_scene_light_count(void* p) { return static_cast<Scene*>(p)->light_count; }
void oracle_scene_lights(void* p, LightRecord* out) {
    auto* s = static_cast<Scene*>(p);
    std::memcpy(out, s->lights.data(), s->lights.size() * sizeof(LightRecord));
}
float oracle_scene_select_prob(void* p) { return static_cast<Scene*>(p)->select_prob; }
double oracle_scene_env_power(void* p) { return static_cast<Scene*>(p)->env.power; }
void oracle_scene_env_tables(void* p, float* marginal, float* conditional, float* pdfs) {
    auto* s = static_cast<Scene*>(p);
    std::memcpy(marginal, s->env.marginal.data(), s->env.marginal.size() * 4);
    std::memcpy(conditional, s->env.conditional.data(), s->env.conditional.size() * 4);
    std::memcpy(pdfs, s->env.pdfs.data(), s->env.pdfs.size() * 4);
}

// Accumulate samples [sample_begin, sample_begin + sample_count) into
// sum_rgba (w·h·4 floats, added to what is there) with the film's
// non-finite guard (accumulate.slang:38-44), over `threads` host threads.
// The guide sums (albedo/normal w·h·4, depth w·h) are accumulated alongside
// when the pointers are non-null, each with its own guard (accumulate.slang:49-67).
void oracle_render(void* p, uint32_t width, uint32_t height, uint32_t sample_begin, uint32_t sample_count,
                   uint32_t max_bounces, uint32_t light_sampling, uint32_t threads, float* sum_rgba,
                   uint64_t* ray_counts, float* albedo_sum, float* normal_sum, float* depth_sum) {
    Scene* s = static_cast<Scene*>(p);
    oracle_camera cam;
    wr3(cam.position, s->cam_pos);
    wr3(cam.look_at, s->cam_look);
    wr3(cam.up, s->cam_upv);
    cam.vfov_degrees = s->vfov;
    float r[3], u[3], f[3];
    oracle_camera_basis(&cam, float(width) / float(height), r, u, f);
    s->cam_right = rd3(r);
    s->cam_up = rd3(u);
    s->cam_fwd = rd3(f);
    std::atomic<uint32_t> next{0};
    std::atomic<uint64_t> ext{0}, shd{0};
    auto work = [&]() {
        RayCounts rc;
        for (;;) {
            uint32_t row = next.fetch_add(1);
            if (row >= height) break;
            for (uint32_t x = 0; x < width; ++x) {
                uint32_t pixel = row * width + x;
                float* dst = sum_rgba + size_t(4) * pixel;
                for (uint32_t k = 0; k < sample_count; ++k) {
                    float v[4];
                    Guides g;
                    trace_path(*s, width, height, pixel, sample_begin + k, max_bounces, light_sampling, v, rc,
                               albedo_sum ? &g : nullptr);
                    if (finite4(v))
                        for (int c = 0; c < 4; ++c) dst[c] += v[c];
                    if (albedo_sum) {
                        if (finite4(g.albedo))
                            for (int c = 0; c < 4; ++c) albedo_sum[size_t(4) * pixel + c] += g.albedo[c];
                        if (finite4(g.normal))
                            for (int c = 0; c < 4; ++c) normal_sum[size_t(4) * pixel + c] += g.normal[c];
                        depth_sum[pixel] += std::isnan(g.depth) ? 0.0f : g.depth;
                    }
                }
            }
        }
        ext += rc.extension;
        shd += rc.shadow;
    };
    if (threads <= 1) {
        work();
    } else {
        std::vector<std::thread> pool;
        for (uint32_t t = 0; t < threads; ++t) pool.emplace_back(work);
        for (auto& t : pool) t.join();
    }
    if (ray_counts) {
        ray_counts[0] = ext.load();
        ray_counts[1] = shd.load();
    }
}

// ---- probes ----------------------------------------------------------------

// Decode a texture to linear RGBA floats (w·h·4); 0 on success.
int oracle_texture_decode(uint32_t format, uint32_t w, uint32_t h, const void* data, float* out) {
    Texture t;
    if (!t.decode(format, w, h, data)) return -1;
    std::memcpy(out, t.texels.data(), t.texels.size() * 4);
    return 0;
}

// n taps at uv (n·2): mode 0 the filtered texel, 1 sampleColor, 2
// sampleScalar, 3 sampleNormal (the modes of cenote_probe_texture).
int oracle_texture_sample(uint32_t format, uint32_t w, uint32_t h, const void* data, uint32_t mode, const float* uv,
                          uint32_t n, float* out) {
    Scene s;
    s.textures.resize(1);
    if (!s.textures[0].decode(format, w, h, data)) return -1;
    for (uint32_t i = 0; i < n; ++i) {
        F2v c{uv[2 * i], uv[2 * i + 1]};
        float* o = out + 4 * size_t(i);
        o[0] = o[1] = o[2] = o[3] = 0.0f;
        if (mode == 1) {
            V3f v = sample_color(s, 0, c);
            wr3(o, v);
        } else if (mode == 2) {
            o[0] = sample_scalar(s, 0, c);
        } else if (mode == 3) {
            wr3(o, sample_normal(s, 0, c));
        } else {
            sample_texture(s, 0, c, o);
        }
    }
    return 0;
}

void oracle_sampler(uint32_t pixel, uint32_t dimension, uint32_t count, float* points, float* values) {
    for (uint32_t i = 0; i < count; ++i) {
        F2 p = sample_2d(pixel, i, dimension);
        points[2 * i] = p.x;
        points[2 * i + 1] = p.y;
        values[i] = sample_1d(pixel, i, dimension);
    }
}

float oracle_hash_uniform(uint32_t pixel, uint32_t sample, uint32_t bounce, uint32_t crossing) {
    return hash_uniform(pixel, sample, bounce, crossing);
}

// FP64 closure evaluation for n (wo, wi) pairs: f (3 doubles) and pdf.
void oracle_bsdf_eval(const Material* m, const float* tables, const float* wo, const float* wi,
                      uint32_t n, uint32_t exiting, double* f_out, double* pdf_out) {
    using BD = BSDF<double>;
    MaterialT<double> md = to_t<double>(*m);
    for (uint32_t i = 0; i < n; ++i) {
        V3<double> o(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
        V3<double> w(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        BD::Closure c = BD::resolve(tables, md, o, exiting != 0);
        V3<double> f = BD::eval(c, w, o);
        f_out[3 * i] = f.x;
        f_out[3 * i + 1] = f.y;
        f_out[3 * i + 2] = f.z;
        pdf_out[i] = BD::pdf(c, w, o);
    }
}

// FP64 closure sampling: u = (u_lobe, u.x, u.y) per entry.
void oracle_bsdf_sample(const Material* m, const float* tables, const float* wo, const float* u, uint32_t n,
                        uint32_t exiting, double* wi_out, double* pdf_out, uint32_t* lobe_out) {
    using BD = BSDF<double>;
    MaterialT<double> md = to_t<double>(*m);
    for (uint32_t i = 0; i < n; ++i) {
        V3<double> o(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
        BD::Closure c = BD::resolve(tables, md, o, exiting != 0);
        BD::Sample s = BD::sample(c, o, u[3 * i], u[3 * i + 1], u[3 * i + 2]);
        wi_out[3 * i] = s.wi.x;
        wi_out[3 * i + 1] = s.wi.y;
        wi_out[3 * i + 2] = s.wi.z;
        pdf_out[i] = s.pdf;
        lobe_out[i] = s.lobe;
    }
}

// Alias-table build for explicit light lists (the reference's own tests).
uint32_t oracle_build_lights(const float* tri_corners, const float* tri_emission, const uint32_t* tri_ids,
                             uint32_t n_tris, const oracle_delta_light* deltas, uint32_t n_deltas,
                             LightRecord* out, double* total_power) {
    std::vector<TriangleLight> tl;
    for (uint32_t i = 0; i < n_tris; ++i)
        tl.push_back({{rd3(tri_corners + 9 * i), rd3(tri_corners + 9 * i + 3), rd3(tri_corners + 9 * i + 6)},
                      rd3(tri_emission + 3 * i), tri_ids[2 * i], tri_ids[2 * i + 1]});
    std::vector<DeltaLight> dl;
    for (uint32_t i = 0; i < n_deltas; ++i) dl.push_back({deltas[i].kind, rd3(deltas[i].anchor), rd3(deltas[i].emission)});
    auto recs = build_lights(tl, dl);
    if (out) std::memcpy(out, recs.data(), recs.size() * sizeof(LightRecord));
    if (total_power) *total_power = total_light_power(tl, dl);
    return uint32_t(recs.size());
}

void oracle_env_tables(uint32_t w, uint32_t h, const float* texels, float* marginal, float* conditional,
                       float* pdfs, double* power) {
    EnvTables e;
    e.width = w;
    e.height = h;
    e.texels.assign(texels, texels + size_t(4) * w * h);
    build_env_tables(e);
    std::memcpy(marginal, e.marginal.data(), e.marginal.size() * 4);
    std::memcpy(conditional, e.conditional.data(), e.conditional.size() * 4);
    std::memcpy(pdfs, e.pdfs.data(), e.pdfs.size() * 4);
    *power = e.power;
}

// Environment sampling probe: n uniform pairs → direction, pdf, (row, col).
void oracle_env_sample(void* p, const float* u, uint32_t n, float* dir, float* pdf, uint32_t* rc) {
    Scene* s = static_cast<Scene*>(p);
    for (uint32_t i = 0; i < n; ++i) {
        EnvSample e = env_sample(s->env, u[2 * i], u[2 * i + 1]);
        wr3(dir + 3 * i, e.direction);
        pdf[i] = e.pdf;
        rc[2 * i] = e.row;
        rc[2 * i + 1] = e.col;
    }
}

void oracle_env_pdf(void* p, const float* dirs, uint32_t n, float* pdf) {
    Scene* s = static_cast<Scene*>(p);
    for (uint32_t i = 0; i < n; ++i) pdf[i] = env_pdf(s->env, rd3(dirs + 3 * i));
}

// Closest-hit probe over the scene's world-space triangles with ray mask ALL:
// hits[4·i] = (instance, primitive, b1 bits, b2 bits), t[i]; instance
// 0xffffffff on a miss.
void oracle_intersect(void* p, const float* org, const float* dir, uint32_t n, uint32_t* hits, float* t_out) {
    Scene* s = static_cast<Scene*>(p);
    for (uint32_t i = 0; i < n; ++i) {
        RayPre r = ray_pre(rd3(org + 3 * i), rd3(dir + 3 * i));
        float best_t = 1e30f;
        uint64_t best_key = ~0ull;
        Hit h{LIGHT_NONE, 0, 0, 0};
        s->bvh.walk(r, 1e30f, [&](uint32_t k, float tmax) {
            const Tri& t = s->bvh.tris[k];
            float tt, b1, b2;
            if (!intersect_tri(r, t, tmax, &tt, &b1, &b2)) return tmax;
            uint64_t key = hit_key(t.instance, t.primitive);
            if (!(tt < best_t || (tt == best_t && key < best_key))) return tmax;
            best_t = tt;
            best_key = key;
            h = {t.instance, t.primitive, b1, b2};
            return tt;
        });
        hits[4 * i] = h.instance;
        hits[4 * i + 1] = h.primitive;
        std::memcpy(&hits[4 * i + 2], &h.b1, 4);
        std::memcpy(&hits[4 * i + 3], &h.b2, 4);
        t_out[i] = h.instance == LIGHT_NONE ? -1.0f : best_t;
    }
}

// Shadow probe: attenuation (≥ 0) or -1 when occluded.
void oracle_shadow(void* p, const float* org, const float* dir, const float* tmax, const uint32_t* target,
                   uint32_t n, float* out) {
    Scene* s = static_cast<Scene*>(p);
    for (uint32_t i = 0; i < n; ++i)
        out[i] = trace_shadow(*s, rd3(org + 3 * i), rd3(dir + 3 * i), tmax[i], target[2 * i], target[2 * i + 1]);
}

}  // extern "C"
