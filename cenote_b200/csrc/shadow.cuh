// The shadow-ray query of crates/cenote/shaders/trace_shadow.slang:29-72 as
// an any-hit walk. The reference commits the closest hit and calls the
// connection visible iff that hit is the target (instance, primitive) or
// nothing. Equivalently: intersect the target triangle first with the same
// watertight arithmetic the walk uses; if it is hit at t_target, any opaque
// non-target hit nearer than it (ties by the (instance, primitive) key)
// occludes; if it is missed (or the connection has no target: environment
// and delta lights), any opaque hit within tmax occludes. Either way the first
// occluder found ends the walk. Fractional-opacity occluders multiply their
// transparency in, as the reference's candidate loop does.
#pragma once
#include "records.h"
#include "textures.cuh"
#include "traverse.cuh"

namespace cn {

// The query's state, resumable step by step (a persistent kernel retires and
// starts queries per lane; see Walk).
struct ShadowQuery {
    Walk w;
    float atten, t_target, tm;
    uint32_t light, lprim, leaf, best_inst, best_prim;
    bool occluded, have_t, closest_fallback;
};

__device__ __forceinline__ void shadow_begin(const DeviceScene& scene, const Ray& ray, float tmax, uint32_t light,
                                             uint32_t lprim, uint32_t leaf, ShadowQuery& q) {
    q.atten = 1.0f;
    q.occluded = false;
    q.have_t = false;
    q.t_target = tmax;
    q.light = light;
    q.lprim = lprim;
    q.leaf = leaf;
    if (leaf != 0xffffffffu && leaf < scene.tri_count) {
        const float4* tp = scene.tris + 3u * leaf;
        float t, b1, b2;
        if (tri_hit(ray, __ldg(tp), __ldg(tp + 1), __ldg(tp + 2), tmax, t, b1, b2)) {
            q.have_t = true;
            q.t_target = t;
        }
    }
    q.closest_fallback = light != LIGHT_NONE && leaf == 0xffffffffu;
    q.best_inst = LIGHT_NONE;
    q.best_prim = 0;
    q.tm = q.t_target;
    walk_begin(q.w, ray);
}

template <bool COUNT = false, int S = TRAVERSAL_STACK>
__device__ __forceinline__ int shadow_step(const DeviceScene& scene, const Ray& ray, ShadowQuery& q, uint2* stack,
                                           uint32_t* visits = nullptr, uint32_t* tests = nullptr) {
    if (scene.node_count == 0) return WALK_DONE;
    return walk_step<COUNT, S>(scene, ray, q.tm, q.w, stack, [&](uint32_t ti, float4 a, float4 b, float4 c, float& tcur) {
        if (q.have_t && ti == q.leaf) return false;  // the target itself
        float t, b1, b2;
        if (!tri_hit(ray, a, b, c, tcur, t, b1, b2)) return false;
        uint32_t inst = __float_as_uint(a.w), prim = __float_as_uint(b.w);
        bool target = inst == q.light && prim == q.lprim;
        if (q.closest_fallback) {
            // No leaf index for the target: the reference's closest-hit walk.
            if (!(t < tcur || (t == tcur && (inst < q.best_inst || (inst == q.best_inst && prim < q.best_prim)))))
                return false;
        } else if (q.have_t && t == q.t_target && !(inst < q.light || (inst == q.light && prim < q.lprim))) {
            return false;  // the target wins the tie
        }
        if (!(__float_as_uint(c.w) & TRI_OPAQUE) && !target) {
            q.atten *= 1.0f - opacity_at(scene, inst, prim, b1, b2);
            if (q.atten < 1e-4f) {
                q.occluded = true;
                return true;
            }
            return false;
        }
        if (!q.closest_fallback) {
            q.occluded = true;  // an opaque occluder nearer than the target (or any, without one)
            return true;
        }
        tcur = t;
        q.best_inst = inst;
        q.best_prim = prim;
        return false;
    }, visits, tests);
}

// The attenuation (>= 0) when visible, -1 when occluded.
__device__ __forceinline__ float shadow_result(const ShadowQuery& q) {
    if (q.occluded) return -1.0f;
    if (q.closest_fallback && !(q.best_inst == LIGHT_NONE || (q.best_inst == q.light && q.best_prim == q.lprim)))
        return -1.0f;
    return q.atten;
}

// The whole query for one ray: the attenuation (>= 0) when visible, -1 when
// occluded, -2 when a traversal bound was exceeded. `stack` holds S entries.
template <bool COUNT = false, int S = TRAVERSAL_STACK>
__device__ __forceinline__ float shadow_query(const DeviceScene& scene, const Ray& ray, float tmax, uint32_t light,
                                              uint32_t lprim, uint32_t leaf, uint2* stack, uint32_t* visits = nullptr,
                                              uint32_t* tests = nullptr) {
    ShadowQuery q;
    shadow_begin(scene, ray, tmax, light, lprim, leaf, q);
    for (;;) {
        int st = shadow_step<COUNT, S>(scene, ray, q, stack, visits, tests);
        if (st == WALK_OVERFLOW) return -2.0f;
        if (st == WALK_DONE) return shadow_result(q);
    }
}

}  // namespace cn
