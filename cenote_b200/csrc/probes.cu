// Probe kernels: the test entry points that expose one device function at a
// time for parity checks — the sampler dump of crates/cenote/shaders/rng_test.slang,
// closure eval/pdf/sample, closest-hit and shadow queries, and environment
// sampling. They run the same device code the wavefront kernels inline.
#include <cuda_runtime.h>

#include "lights_env.cuh"
#include "openpbr.cuh"
#include "sampler.cuh"
#include "shadow.cuh"
#include "textures.cuh"
#include "traverse.cuh"
#include "trqueue.cuh"

namespace cn {
namespace {

__global__ void k_probe_sampler(uint32_t pixel, uint32_t dim, uint32_t count, float2* points, float* values) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    points[i] = sample_2d(pixel, i, dim);
    values[i] = sample_1d(pixel, i, dim);
}

__global__ void k_probe_bsdf(const float* tables, Material m, const float3* wo, const float3* wi, uint32_t n,
                             uint32_t exiting, float3* f, float* pdf) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Closure c = resolve_closure(tables, m, wo[i], exiting != 0);
    f[i] = eval_bsdf(c, wi[i], wo[i]);
    pdf[i] = bsdf_pdf(c, wi[i], wo[i]);
}

__global__ void k_probe_bsdf_sample(const float* tables, Material m, const float3* wo, const float3* u, uint32_t n,
                                    uint32_t exiting, float3* wi, float* pdf, uint32_t* lobe) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Closure c = resolve_closure(tables, m, wo[i], exiting != 0);
    BsdfSample s = sample_bsdf(c, wo[i], u[i].x, u[i].y, u[i].z);
    wi[i] = s.wi;
    pdf[i] = s.pdf;
    lobe[i] = s.lobe;
}

__global__ void k_probe_intersect(DeviceScene scene, const float3* org, const float3* dir, uint32_t n, uint4* hits,
                                  float* tout, uint32_t* flag) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Ray ray = make_ray(org[i], dir[i]);
    float tmax = 1e30f;
    uint32_t bi = LIGHT_NONE, bp = 0;
    float b1s = 0.0f, b2s = 0.0f;
    bool ok = traverse(scene, ray, tmax, [&](uint32_t, float4 a, float4 b, float4 c, float& tm) {
        float t, b1, b2;
        if (!tri_hit(ray, a, b, c, tm, t, b1, b2)) return false;
        uint32_t inst = __float_as_uint(a.w), prim = __float_as_uint(b.w);
        if (!(t < tm || (t == tm && (inst < bi || (inst == bi && prim < bp))))) return false;
        tm = t;
        bi = inst;
        bp = prim;
        b1s = b1;
        b2s = b2;
        return false;
    });
    if (!ok) atomicOr(flag, 1u);
    hits[i] = make_uint4(bi, bp, __float_as_uint(b1s), __float_as_uint(b2s));
    tout[i] = bi == LIGHT_NONE ? -1.0f : tmax;
}

// The queued closest-hit walk (trqueue.cuh) over n rays: each warp walks its
// own contiguous share of the rays, refilling idle lanes as the wavefront
// kernel does.
struct ProbeSource {
    const float3* org;
    const float3* dir;
    uint4* hits;
    float* tout;
    uint32_t cursor, end;  // the warp's next ray and the end of its share (warp-uniform)
    __device__ __forceinline__ uint32_t next(bool live, bool& drained) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !live);
        const uint32_t lane = threadIdx.x & 31u;
        const uint32_t i = cursor + __popc(idle & ((1u << lane) - 1u));
        cursor += __popc(idle);
        if (cursor >= end) drained = true;
        return (!live && i < end) ? i : ~0u;
    }
    __device__ __forceinline__ void ray(uint32_t i, float3& o, float3& d) const {
        o = org[i];
        d = dir[i];
    }
    __device__ __forceinline__ void emit(uint32_t i, uint4 h, float t) const {
        hits[i] = h;
        tout[i] = h.x == LIGHT_NONE ? -1.0f : t;
    }
    __device__ __forceinline__ void step(bool, uint32_t, uint32_t, float) const {}
    __device__ __forceinline__ uint32_t want_idle(bool drained) const { return drained ? 32u : 8u; }
};

constexpr uint32_t PROBE_RAYS_PER_WARP = 256;

__global__ void __launch_bounds__(128) k_probe_intersect_queued(DeviceScene scene, const float3* org,
                                                                const float3* dir, uint32_t n, uint4* hits,
                                                                float* tout, uint32_t* flag) {
    __shared__ TriQueueSmem tqs[4];
    const uint32_t warp = blockIdx.x * 4u + (threadIdx.x >> 5);
    const uint32_t begin = warp * PROBE_RAYS_PER_WARP;
    if (begin >= n) return;  // whole warps only
    ProbeSource src{org, dir, hits, tout, begin, min(n, begin + PROBE_RAYS_PER_WARP)};
    bool overflow = false;
    queued_closest<false>(scene, tqs[threadIdx.x >> 5], src, RAY_MASK_ALL, overflow, nullptr, nullptr);
    if (overflow) atomicOr(flag, 1u);
}

// The queued shadow walk (trqueue.cuh, queued_any) over n queries of an
// all-opaque scene, each warp walking its own contiguous share with refills;
// out[i] = 1 when visible, -1 when occluded (k_probe_shadow's encoding).
struct ProbeShadowSource {
    const DeviceScene& scene;
    const float3* org;
    const float3* dir;
    const float* tmaxs;
    const uint2* targets;
    float* out;
    uint32_t* flag;
    uint32_t cursor, end;  // the warp's next query and the end of its share (warp-uniform)
    __device__ __forceinline__ uint32_t next(bool live, bool& drained) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !live);
        const uint32_t i = cursor + __popc(idle & ((1u << (threadIdx.x & 31u)) - 1u));
        cursor += __popc(idle);
        if (cursor >= end) drained = true;
        return (!live && i < end) ? i : ~0u;
    }
    __device__ __forceinline__ uint32_t leaf_of(uint32_t i) const {
        const uint32_t light = targets[i].x, lprim = targets[i].y;
        if (light == LIGHT_NONE) return 0xffffffffu;
        const uint32_t first = scene.geometry[light].light;
        return first != LIGHT_NONE ? scene.light_leaf[first + lprim] : 0xffffffffu;
    }
    __device__ __forceinline__ bool begin(uint32_t i, Ray& ray, AnyQuery& a) const {
        ray = make_ray(org[i], dir[i]);
        const uint32_t light = targets[i].x, leaf = leaf_of(i);
        a.occluded = false;
        a.light = light;
        a.lprim = targets[i].y;
        a.tm = tmaxs[i];
        a.leaf = 0xffffffffu;
        if (light != LIGHT_NONE && leaf == 0xffffffffu) return false;
        if (leaf < scene.tri_count) {
            const float4* tp = scene.tris + 3u * leaf;
            float t, b1, b2;
            if (tri_hit(ray, __ldg(tp), __ldg(tp + 1), __ldg(tp + 2), tmaxs[i], t, b1, b2)) {
                a.tm = t;
                a.leaf = leaf;
            }
        }
        return true;
    }
    template <int S>
    __device__ __forceinline__ void closest(uint32_t i, uint2* stack) const {
        const float a = shadow_query<false, S>(scene, make_ray(org[i], dir[i]), tmaxs[i], targets[i].x, targets[i].y,
                                               leaf_of(i), stack);
        if (a == -2.0f) atomicOr(flag, 1u);
        out[i] = a < 0.0f ? -1.0f : a;
    }
    __device__ __forceinline__ void emit(uint32_t i, bool visible) const { out[i] = visible ? 1.0f : -1.0f; }
    __device__ __forceinline__ uint32_t want_idle(bool drained) const { return drained ? 32u : 8u; }
};

__global__ void __launch_bounds__(128) k_probe_shadow_queued(DeviceScene scene, const float3* org, const float3* dir,
                                                             const float* tmaxs, const uint2* targets, uint32_t n,
                                                             float* out, uint32_t* flag) {
    __shared__ TriQueueSmem tqs[4];
    const uint32_t warp = blockIdx.x * 4u + (threadIdx.x >> 5);
    const uint32_t begin = warp * PROBE_RAYS_PER_WARP;
    if (begin >= n) return;  // whole warps only
    ProbeShadowSource src{scene, org, dir, tmaxs, targets, out, flag, begin, min(n, begin + PROBE_RAYS_PER_WARP)};
    bool overflow = false;
    queued_any<false>(scene, tqs[threadIdx.x >> 5], src, overflow, nullptr, nullptr);
    if (overflow) atomicOr(flag, 1u);
}

__global__ void k_probe_shadow(DeviceScene scene, const float3* org, const float3* dir, const float* tmaxs,
                               const uint2* targets, uint32_t n, float* out, uint32_t* flag) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Ray ray = make_ray(org[i], dir[i]);
    uint32_t light = targets[i].x, lprim = targets[i].y;
    // The leaf of an emissive target comes from its light record, as in the
    // wavefront (GeometryRecord.light + primitive).
    uint32_t leaf = 0xffffffffu;
    if (light != LIGHT_NONE) {
        uint32_t first = scene.geometry[light].light;
        if (first != LIGHT_NONE) leaf = scene.light_leaf[first + lprim];
    }
    uint2 stack[TRAVERSAL_STACK];
    float a = shadow_query(scene, ray, tmaxs[i], light, lprim, leaf, stack);
    if (a == -2.0f) atomicOr(flag, 1u);
    out[i] = a < 0.0f ? -1.0f : a;
}

__global__ void k_probe_env_sample(DeviceScene scene, const float2* u, uint32_t n, float3* dir, float* pdf,
                                   uint2* rc) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    EnvSample s = env_sample(scene, u[i]);
    dir[i] = s.direction;
    pdf[i] = s.pdf;
    rc[i] = make_uint2(s.row, s.col);
}

__global__ void k_probe_env_pdf(DeviceScene scene, const float3* d, uint32_t n, float* pdf) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pdf[i] = env_pdf(scene, d[i]);
}

// One raw tap per UV of a bindless slot (mode 0: the texel as filtered;
// 1: sampleColor; 2: sampleScalar in x; 3: sampleNormal).
__global__ void k_probe_texture(DeviceScene scene, uint32_t index, uint32_t mode, const float2* uv, uint32_t n,
                                float4* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 r;
    if (mode == 1) {
        float3 c = sample_color(scene, index, uv[i]);
        r = make_float4(c.x, c.y, c.z, 0.0f);
    } else if (mode == 2) {
        r = make_float4(sample_scalar(scene, index, uv[i]), 0.0f, 0.0f, 0.0f);
    } else if (mode == 3) {
        float3 c = sample_normal(scene, index, uv[i]);
        r = make_float4(c.x, c.y, c.z, 0.0f);
    } else {
        r = sample_texture(scene, index, uv[i]);
    }
    out[i] = r;
}

inline int blocks(uint32_t n) { return int((n + 127) / 128); }

}  // namespace

void probe_sampler(uint32_t pixel, uint32_t dim, uint32_t count, float2* points, float* values, cudaStream_t s) {
    k_probe_sampler<<<blocks(count), 128, 0, s>>>(pixel, dim, count, points, values);
}
void probe_bsdf(const float* tables, const Material& m, const float3* wo, const float3* wi, uint32_t n,
                uint32_t exiting, float3* f, float* pdf, cudaStream_t s) {
    k_probe_bsdf<<<blocks(n), 128, 0, s>>>(tables, m, wo, wi, n, exiting, f, pdf);
}
void probe_bsdf_sample(const float* tables, const Material& m, const float3* wo, const float3* u, uint32_t n,
                       uint32_t exiting, float3* wi, float* pdf, uint32_t* lobe, cudaStream_t s) {
    k_probe_bsdf_sample<<<blocks(n), 128, 0, s>>>(tables, m, wo, u, n, exiting, wi, pdf, lobe);
}
void probe_intersect(const DeviceScene& scene, const float3* org, const float3* dir, uint32_t n, uint4* hits, float* t,
                     uint32_t* flag, cudaStream_t s) {
    k_probe_intersect<<<blocks(n), 128, 0, s>>>(scene, org, dir, n, hits, t, flag);
}
void probe_intersect_queued(const DeviceScene& scene, const float3* org, const float3* dir, uint32_t n, uint4* hits,
                            float* t, uint32_t* flag, cudaStream_t s) {
    const uint32_t grid = (n + 4u * PROBE_RAYS_PER_WARP - 1u) / (4u * PROBE_RAYS_PER_WARP);
    k_probe_intersect_queued<<<grid, 128, 0, s>>>(scene, org, dir, n, hits, t, flag);
}
void probe_shadow(const DeviceScene& scene, const float3* org, const float3* dir, const float* tmax,
                  const uint2* targets, uint32_t n, float* out, uint32_t* flag, cudaStream_t s) {
    k_probe_shadow<<<blocks(n), 128, 0, s>>>(scene, org, dir, tmax, targets, n, out, flag);
}
void probe_shadow_queued(const DeviceScene& scene, const float3* org, const float3* dir, const float* tmax,
                         const uint2* targets, uint32_t n, float* out, uint32_t* flag, cudaStream_t s) {
    const uint32_t grid = (n + 4u * PROBE_RAYS_PER_WARP - 1u) / (4u * PROBE_RAYS_PER_WARP);
    k_probe_shadow_queued<<<grid, 128, 0, s>>>(scene, org, dir, tmax, targets, n, out, flag);
}
void probe_env_sample(const DeviceScene& scene, const float2* u, uint32_t n, float3* dir, float* pdf, uint2* rc,
                      cudaStream_t s) {
    k_probe_env_sample<<<blocks(n), 128, 0, s>>>(scene, u, n, dir, pdf, rc);
}
void probe_env_pdf(const DeviceScene& scene, const float3* d, uint32_t n, float* pdf, cudaStream_t s) {
    k_probe_env_pdf<<<blocks(n), 128, 0, s>>>(scene, d, n, pdf);
}
void probe_texture(const DeviceScene& scene, uint32_t index, uint32_t mode, const float2* uv, uint32_t n, float4* out,
                   cudaStream_t s) {
    k_probe_texture<<<blocks(n), 128, 0, s>>>(scene, index, mode, uv, n, out);
}

}  // namespace cn
