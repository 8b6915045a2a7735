// Material textures on the device: the bindless table of
// crates/cenote/shaders/textures.slang:20-82 as an array of CUDA texture
// objects (one level, bilinear, repeat addressing, sRGB storage decoded by the
// texture unit per texel; BC1/BC4/BC5 blocks decoded by the hardware), UV
// interpolation and opacity taps (scene.slang:31-64), and the normal-mapped
// shading frame (shade_surface.slang:183-231).
#pragma once
#include "records.h"
#include "vecmath.cuh"

namespace cn {

__device__ __forceinline__ float4 sample_texture(const DeviceScene& s, uint32_t index, float2 uv) {
    return tex2D<float4>(static_cast<cudaTextureObject_t>(__ldg(s.textures + index)), uv.x, uv.y);
}

// Linear Rec.709 -> ACEScg, rows-dot-vector (textures.slang:37-45).
__device__ __forceinline__ float3 sample_color(const DeviceScene& s, uint32_t index, float2 uv) {
    float4 t = sample_texture(s, index, uv);
    return f3(0.613097400f * t.x + 0.339523140f * t.y + 0.047379450f * t.z,
              0.070193730f * t.x + 0.916353900f * t.y + 0.013452399f * t.z,
              0.020615594f * t.x + 0.109569780f * t.y + 0.869814660f * t.z);
}

__device__ __forceinline__ float sample_scalar(const DeviceScene& s, uint32_t index, float2 uv) {
    return sample_texture(s, index, uv).x;
}

__device__ __forceinline__ float3 sample_normal(const DeviceScene& s, uint32_t index, float2 uv) {
    float4 t = sample_texture(s, index, uv);
    float x = t.x * 2.0f - 1.0f, y = t.y * 2.0f - 1.0f;
    return f3(x, y, sqrtf(fmaxf(1.0f - (x * x + y * y), 0.0f)));
}

// scene.slang:31-37, from the instance's own index and UV streams.
__device__ __forceinline__ float2 interpolate_uv(const float* uvs, const uint32_t* indices, uint32_t prim, float b1,
                                                 float b2) {
    uint32_t i0 = __ldg(indices + 3 * prim), i1 = __ldg(indices + 3 * prim + 1), i2 = __ldg(indices + 3 * prim + 2);
    float2 u0 = __ldg(reinterpret_cast<const float2*>(uvs) + i0);
    float2 u1 = __ldg(reinterpret_cast<const float2*>(uvs) + i1);
    float2 u2 = __ldg(reinterpret_cast<const float2*>(uvs) + i2);
    return make_float2(u0.x + b1 * (u1.x - u0.x) + b2 * (u2.x - u0.x), u0.y + b1 * (u1.y - u0.y) + b2 * (u2.y - u0.y));
}

__device__ __forceinline__ float2 interpolate_uv(const DeviceScene& s, uint32_t inst, uint32_t prim, float b1,
                                                 float b2) {
    const GeomRecord* g = s.geometry + inst;
    const float* uvs = reinterpret_cast<const float*>(__ldg(reinterpret_cast<const unsigned long long*>(&g->uvs)));
    const uint32_t* idx =
        reinterpret_cast<const uint32_t*>(__ldg(reinterpret_cast<const unsigned long long*>(&g->indices)));
    return interpolate_uv(uvs, idx, prim, b1, b2);
}

// The slots resolveMaterial replaces (textures.slang:70-82): base colour,
// specular roughness, metalness, emission. Opacity and normal maps resolve
// where they are used.
__device__ __forceinline__ bool has_parameter_maps(const Material& m) {
    return (m.base_color_texture & m.specular_roughness_texture & m.metalness_texture & m.emission_texture) !=
           TEXTURE_NONE;
}

// The mapped values of one hit. Kept out of line with its inputs and result
// by value (as are the other map paths below): an untextured scene never
// calls it, and neither inlining it nor handing it the material by reference
// (which moves the material to local memory) may cost the shading kernel.
struct MapTaps {
    float3 base_color, emission;
    float roughness, metalness;
};

static __device__ __noinline__ MapTaps read_maps(const DeviceScene& s, uint32_t base_map, uint32_t rough_map,
                                                 uint32_t metal_map, uint32_t emission_map_slot, float2 uv) {
    MapTaps t;
    t.base_color = base_map != TEXTURE_NONE ? sample_color(s, base_map, uv) : f3(0.0f);
    t.roughness = rough_map != TEXTURE_NONE ? sample_scalar(s, rough_map, uv) : 0.0f;
    t.metalness = metal_map != TEXTURE_NONE ? sample_scalar(s, metal_map, uv) : 0.0f;
    t.emission = emission_map_slot != TEXTURE_NONE ? sample_color(s, emission_map_slot, uv) : f3(1.0f);
    return t;
}

// textures.slang:70-82: replaced slots take the texel, emission multiplies it.
__device__ __forceinline__ void resolve_material(const DeviceScene& s, Material& m, float2 uv) {
    MapTaps t = read_maps(s, m.base_color_texture, m.specular_roughness_texture, m.metalness_texture,
                          m.emission_texture, uv);
    if (m.base_color_texture != TEXTURE_NONE) {
        m.base_color[0] = t.base_color.x;
        m.base_color[1] = t.base_color.y;
        m.base_color[2] = t.base_color.z;
    }
    if (m.specular_roughness_texture != TEXTURE_NONE) m.specular_roughness = t.roughness;
    if (m.metalness_texture != TEXTURE_NONE) m.metalness = t.metalness;
    if (m.emission_texture != TEXTURE_NONE) {
        m.emission[0] *= t.emission.x;
        m.emission[1] *= t.emission.y;
        m.emission[2] *= t.emission.z;
    }
}

// scene.slang:56-64: a candidate's opacity, its map evaluated at the candidate.
static __device__ __noinline__ float opacity_map(const DeviceScene& s, uint32_t map, uint32_t inst, uint32_t prim, float b1,
                                          float b2) {
    return sample_scalar(s, map, interpolate_uv(s, inst, prim, b1, b2));
}

__device__ __forceinline__ float opacity_at(const DeviceScene& s, uint32_t inst, uint32_t prim, float b1, float b2) {
    const Material* m = s.materials + inst;
    float opacity = __ldg(&m->opacity);
    uint32_t map = __ldg(&m->opacity_texture);
    if (map != TEXTURE_NONE) opacity *= opacity_map(s, map, inst, prim, b1, b2);
    return opacity;
}

// A textured emitter's map at a sampled light point (shade_surface.slang:405-418).
static __device__ __noinline__ float3 emission_map(const DeviceScene& s, uint32_t map, uint32_t inst, uint32_t prim, float b1,
                                            float b2) {
    return sample_color(s, map, interpolate_uv(s, inst, prim, b1, b2));
}

// shade_surface.slang:183-231: tangent frame per hit from the triangle's
// positions and UVs; degenerate parameterisations keep the unmapped normal;
// the result is flipped to the face the ray struck.
static __device__ __noinline__ float3 mapped_shading_normal(const DeviceScene& s, uint32_t inst, uint32_t prim,
                                                            float2 uv, uint32_t map, float3 shading, float3 normal) {
    const GeomRecord& g = s.geometry[inst];
    uint32_t i0 = __ldg(g.indices + 3 * prim), i1 = __ldg(g.indices + 3 * prim + 1), i2 = __ldg(g.indices + 3 * prim + 2);
    const float2* uvs = reinterpret_cast<const float2*>(g.uvs);
    float2 u0 = __ldg(uvs + i0), u1 = __ldg(uvs + i1), u2 = __ldg(uvs + i2);
    float du1 = u1.x - u0.x, dv1 = u1.y - u0.y, du2 = u2.x - u0.x, dv2 = u2.y - u0.y;
    float det = du1 * dv2 - dv1 * du2;
    if (fabsf(det) < 1e-12f) return shading;
    float3 p0 = f3(__ldg(g.positions + 3 * i0), __ldg(g.positions + 3 * i0 + 1), __ldg(g.positions + 3 * i0 + 2));
    float3 p1 = f3(__ldg(g.positions + 3 * i1), __ldg(g.positions + 3 * i1 + 1), __ldg(g.positions + 3 * i1 + 2));
    float3 p2 = f3(__ldg(g.positions + 3 * i2), __ldg(g.positions + 3 * i2 + 1), __ldg(g.positions + 3 * i2 + 2));
    float3 e1 = p1 - p0, e2 = p2 - p0;
    float3 r0 = f3(g.o2w[0][0], g.o2w[0][1], g.o2w[0][2]), r1 = f3(g.o2w[1][0], g.o2w[1][1], g.o2w[1][2]),
           r2 = f3(g.o2w[2][0], g.o2w[2][1], g.o2w[2][2]);
    float3 we1 = f3(dot(r0, e1), dot(r1, e1), dot(r2, e1));
    float3 we2 = f3(dot(r0, e2), dot(r1, e2), dot(r2, e2));
    float3 dpdu = (dv2 * we1 - dv1 * we2) / det;
    float3 dpdv = (du1 * we2 - du2 * we1) / det;
    float3 tangent = dpdu - shading * dot(shading, dpdu);
    float len2 = dot(tangent, tangent);
    if (!(len2 > 1e-20f)) return shading;
    tangent = tangent * rsqrtf(len2);
    float3 bitangent = cross(shading, tangent);
    if (dot(bitangent, dpdv) < 0.0f) bitangent = -bitangent;
    float3 t = sample_normal(s, map, uv);
    float3 mapped = normalize(t.x * tangent + t.y * bitangent + t.z * shading);
    if (dot(mapped, normal) < 0.0f) mapped = -mapped;
    return mapped;
}

}  // namespace cn
