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

// Returns the attenuation (>= 0) when visible, -1 when occluded, -2 when a
// traversal bound was exceeded.
template <bool COUNT = false>
__device__ __forceinline__ float shadow_query(const DeviceScene& scene, const Ray& ray, float tmax, uint32_t light,
                                              uint32_t lprim, uint32_t leaf, uint32_t* visits = nullptr,
                                              uint32_t* tests = nullptr) {
    float atten = 1.0f;
    bool occluded = false;
    bool have_t = false;
    float t_target = tmax;
    if (leaf != 0xffffffffu && leaf < scene.tri_count) {
        const float4* tp = scene.tris + 3u * leaf;
        float t, b1, b2;
        if (tri_hit(ray, __ldg(tp), __ldg(tp + 1), __ldg(tp + 2), tmax, t, b1, b2)) {
            have_t = true;
            t_target = t;
        }
    }
    const bool closest_fallback = light != LIGHT_NONE && leaf == 0xffffffffu;
    uint32_t best_inst = LIGHT_NONE, best_prim = 0;
    float tm = t_target;
    bool ok = traverse<COUNT>(scene, ray, tm, [&](uint32_t ti, float4 a, float4 b, float4 c, float& tcur) {
        if (have_t && ti == leaf) return false;  // the target itself
        float t, b1, b2;
        if (!tri_hit(ray, a, b, c, tcur, t, b1, b2)) return false;
        uint32_t inst = __float_as_uint(a.w), prim = __float_as_uint(b.w);
        bool target = inst == light && prim == lprim;
        if (closest_fallback) {
            // No leaf index for the target: the reference's closest-hit walk.
            if (!(t < tcur || (t == tcur && (inst < best_inst || (inst == best_inst && prim < best_prim))))) return false;
        } else if (have_t && t == t_target &&
                   !(inst < light || (inst == light && prim < lprim))) {
            return false;  // the target wins the tie
        }
        if (!(__float_as_uint(c.w) & TRI_OPAQUE) && !target) {
            atten *= 1.0f - opacity_at(scene, inst, prim, b1, b2);
            if (atten < 1e-4f) {
                occluded = true;
                return true;
            }
            return false;
        }
        if (!closest_fallback) {
            occluded = true;  // an opaque occluder nearer than the target (or any, without one)
            return true;
        }
        tcur = t;
        best_inst = inst;
        best_prim = prim;
        return false;
    }, visits, tests);
    if (!ok) return -2.0f;
    if (occluded) return -1.0f;
    if (closest_fallback && !(best_inst == LIGHT_NONE || (best_inst == light && best_prim == lprim))) return -1.0f;
    return atten;
}

}  // namespace cn
