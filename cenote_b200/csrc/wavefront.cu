// The wavefront engine's kernels for sm_100a.
//
// Stage order per wave follows crates/cenote/src/wavefront.rs:727-828 —
// raygen, then per bounce intersect → shade (miss | surface) → shadow — and
// each stage's arithmetic follows its Slang kernel (raygen.slang,
// intersect.slang, shade_miss.slang, shade_surface.slang, trace_shadow.slang).
// The B200 shape differs from the reference's:
//  * a wave may carry several samples of every pixel (path = s·count + pixel),
//    so one launch fills all 148 SMs even at small resolutions; radiance is
//    path-owned and the film adds samples in ascending order, which keeps the
//    result bitwise identical to one-sample waves;
//  * there is no indirect dispatch: the traversal and shading kernels are
//    persistent grids (a multiple of the SM count) whose warps pull 32 work
//    items at a time from a per-stage counter, so a stage costs one launch
//    whatever its queue length and load-balances divergent rays;
//  * queue pushes are warp-aggregated (one atomic per warp, ballot + popc);
//  * miss and surface shading share one kernel — a path is in exactly one of
//    the two, so the per-path write stays single and ordered.
#include "wavefront.h"

#include "guide.h"
#include "lights_env.cuh"
#include "openpbr.cuh"
#include "sampler.cuh"
#include "shadow.cuh"
#include "textures.cuh"
#include "traverse.cuh"
#include "trqueue.cuh"

namespace cn {

namespace {

constexpr int BLOCK = 128;

// Minimum resident 128-thread blocks per SM for the shading kernel: the
// register cap that trades spills against occupancy (6 → 80 registers; with
// material-sorted waves of 30-60 M paths, 6 measured 2 % faster than 5 on the
// textured terrain and level on the chart; 4 and uncapped were slower).
#ifndef CN_SHADE_MIN_BLOCKS
#define CN_SHADE_MIN_BLOCKS 6
#endif
// The same for the variant with the coat, fuzz, transmission and thin-wall
// lobes, which needs more registers than the layer-free one: 4 (128
// registers, 82 / 152 bytes of spills per thread instead of 374 / 908 at 80)
// shades the terrain in 86.2 ms per frame against 87.2 at 6 and 89.0 at 5
// (two runs each); the layer-free variant keeps 6.
#ifndef CN_SHADE_LAYERED_MIN_BLOCKS
#define CN_SHADE_LAYERED_MIN_BLOCKS 4
#endif
// The same for the traversal kernels (8 → 64 registers), and for the
// closest-hit walks alone (which spill a little at 64 registers).
#ifndef CN_TRAV_MIN_BLOCKS
#define CN_TRAV_MIN_BLOCKS 8
#endif
#ifndef CN_ISECT_MIN_BLOCKS
#define CN_ISECT_MIN_BLOCKS CN_TRAV_MIN_BLOCKS
#endif

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Fetch the next 32 work items for this warp; every lane gets the same base.
__device__ __forceinline__ uint32_t warp_fetch(uint32_t* counter) {
    uint32_t base = 0;
    if (lane_id() == 0) base = atomicAdd(counter, 32u);
    return __shfl_sync(0xffffffffu, base, 0);
}

// Warp-aggregated append: returns this lane's slot, or ~0u if !pred. Must be
// called by all 32 lanes together.
__device__ __forceinline__ uint32_t warp_push(uint32_t* counter, bool pred) {
    uint32_t mask = __ballot_sync(0xffffffffu, pred);
    if (mask == 0) return ~0u;
    uint32_t leader = __ffs(mask) - 1u;
    uint32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(counter, uint32_t(__popc(mask)));
    base = __shfl_sync(0xffffffffu, base, leader);
    return pred ? base + __popc(mask & ((1u << lane_id()) - 1u)) : ~0u;
}

__device__ __forceinline__ void flag_overflow(uint32_t* counters) { atomicOr(counters + CTR_OVERFLOW, 1u); }

// The material-sort key of a closest hit at distance t along path `path`'s
// ray (SORT_LAYERS splits the key range). Layer-free hits take their
// instance, or with pool.sort_location the Morton index of the 32 x 32 cell
// of the scene's x/z extent their point lies in: their next rays then leave
// nearby points together, which the next walk's caches reward on some scenes
// (the autotuner decides).
__device__ __forceinline__ uint32_t material_key(const DeviceScene& s, const PathPool& pool, uint32_t inst,
                                                 uint32_t path, float t) {
    if (inst == LIGHT_NONE) return 0u;
    if (__ldg(s.instance_layers + inst)) return SORT_LAYERS + inst % (SORT_BINS - SORT_LAYERS);
    if (!pool.sort_location) return 1u + inst % (SORT_LAYERS - 1u);
    const float4 o = pool.org[path], d = pool.dir[path];
    const float fx = (o.x + t * d.x - s.bbox_min[0]) * s.bbox_inv, fz = (o.z + t * d.z - s.bbox_min[2]) * s.bbox_inv;
    const uint32_t cx = min(31u, uint32_t(fmaxf(fx, 0.0f) * 32.0f)), cz = min(31u, uint32_t(fmaxf(fz, 0.0f) * 32.0f));
    uint32_t m = 0u;
    for (uint32_t b = 0; b < 5u; ++b) m |= (((cx >> b) & 1u) << (2u * b)) | (((cz >> b) & 1u) << (2u * b + 1u));
    return 1u + m % (SORT_LAYERS - 1u);
}

// Instrumented launches: one 64-bit add per warp for the traversal tallies.
__device__ __forceinline__ void flush_counts(uint32_t* counters, uint32_t visits, uint32_t tests) {
    for (int o = 16; o > 0; o >>= 1) {
        visits += __shfl_xor_sync(0xffffffffu, visits, o);
        tests += __shfl_xor_sync(0xffffffffu, tests, o);
    }
    if (lane_id() == 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(counters + CTR_VISITS), (unsigned long long)visits);
        atomicAdd(reinterpret_cast<unsigned long long*>(counters + CTR_TESTS), (unsigned long long)tests);
    }
}

// Paths entering bounce `bounce`: the wave's camera paths (n0, or when n0
// is 0 the count raygen left in CTR_RAYS, as a replayed graph's waves do),
// then the previous bounce's pushes.
__device__ __forceinline__ uint32_t bounce_paths(const PathPool& pool, uint32_t bounce, uint32_t n0) {
    return min(bounce == 0 && n0 != 0 ? n0 : pool.counters[CTR_RAYS + bounce], pool.capacity);
}

// ---- raygen (raygen.slang:47-112) ----------------------------------------------

__device__ __forceinline__ float2 concentric_disk(float2 u) {
    float ox = 2.0f * u.x - 1.0f, oy = 2.0f * u.y - 1.0f;
    if (ox == 0.0f && oy == 0.0f) return make_float2(0.0f, 0.0f);
    float r, th;
    if (fabsf(ox) > fabsf(oy)) {
        r = ox;
        th = (ENV_PI / 4.0f) * (oy / ox);
    } else {
        r = oy;
        th = (ENV_PI / 2.0f) - (ENV_PI / 4.0f) * (ox / oy);
    }
    float s, c;
    sincosf(th, &s, &c);
    return make_float2(r * c, r * s);
}

// One camera path: path slot p traces `sample` of `pixel` of a width x height
// image with the camera's basis.
__device__ __forceinline__ void raygen_path(const PathPool& pool, uint32_t p, uint32_t pixel, uint32_t sample,
                                            uint32_t width, uint32_t height, float3 cam_pos, float3 cam_right,
                                            float3 cam_up, float3 cam_fwd, float aperture) {
    float2 j = sample_2d(pixel, sample, CAMERA_JITTER);
    float xx = float(pixel % width) + j.x, yy = float(pixel / width) + j.y;
    float ux = xx / float(width), uy = yy / float(height);
    float nx = 2.0f * ux - 1.0f, ny = 1.0f - 2.0f * uy;
    float3 target = cam_fwd + nx * cam_right + ny * cam_up;
    float3 org = cam_pos;
    float3 dir = normalize(target);
    if (aperture > 0.0f) {
        float2 d = concentric_disk(sample_2d(pixel, sample, CAMERA_LENS));
        d.x *= aperture;
        d.y *= aperture;
        float3 off = d.x * normalize(cam_right) + d.y * normalize(cam_up);
        org = org + off;
        dir = normalize(target - off);
    }
    pool.org[p] = f4(org, 0.0f);
    pool.dir[p] = f4(dir, dot(dir, normalize(cam_fwd)));
    pool.thr[p] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    pool.ps[p] = make_uint2(pixel, sample);
    pool.state[p] = MEDIUM_NONE;
    pool.rad[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (pool.guide_rec) pool.guide_rec[p] = ~0u;
    if (pool.aov_albedo) {
        pool.aov_albedo[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        pool.aov_normal[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        pool.aov_depth[p] = 0.0f;
    }
}

__global__ void __launch_bounds__(BLOCK) k_raygen(PathPool pool, WaveParams wp) {
    uint32_t n = wp.pixel_count * wp.samples;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        uint32_t s = p / wp.pixel_count;
        uint32_t pixel = wp.pixel_base + wave_pixel(p - s * wp.pixel_count, wp.tile_width);
        uint32_t sample = wp.sample_base + s + (wp.sample_offset ? __ldg(wp.sample_offset) : 0u);
        raygen_path(pool, p, pixel, sample, wp.width, wp.height, wp.cam_pos, wp.cam_right, wp.cam_up, wp.cam_fwd,
                    wp.aperture);
    }
}

// The segment of a multi-job wave that holds item `x` (a path, or with
// `by_pixel` an accumulate item): the last whose first item is at most x.
__device__ __forceinline__ uint32_t find_segment(const WaveSegment* segs, uint32_t nseg, uint32_t x, bool by_pixel) {
    uint32_t lo = 0, hi = nseg;  // answer in [lo, hi)
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t first = by_pixel ? __ldg(&segs[mid].pixel_start) : __ldg(&segs[mid].start);
        if (first <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Camera paths of a multi-job wave: each path takes its job's image size,
// camera and sample index from its segment, so it is the path a standalone
// render of that job traces for the same (pixel, sample). With `hdr` (a
// replayed graph) the segment and path counts come from it, and the path
// count goes to CTR_RAYS for the kernels that follow.
__global__ void __launch_bounds__(BLOCK) k_raygen_segments(PathPool pool, const WaveSegment* __restrict__ segs,
                                                           uint32_t nseg, uint32_t n, const uint32_t* hdr) {
    if (hdr) {
        nseg = __ldg(hdr);
        n = __ldg(hdr + 1);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) pool.counters[CTR_RAYS] = n;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const WaveSegment& g = segs[find_segment(segs, nseg, p, false)];
        const uint32_t q = p - g.start;
        const uint32_t s = q / g.pixel_count;
        raygen_path(pool, p, g.pixel_base + (q - s * g.pixel_count), g.sample_base + s, g.width, g.height,
                    g.cam_pos, g.cam_right, g.cam_up, g.cam_fwd, g.aperture);
    }
}

// ---- intersect (intersect.slang:47-88) -------------------------------------------

// Dynamic ray fetching (Aila & Laine, HPG 2009): a lane whose ray finishes
// does not wait for the warp's slowest ray. Each warp walks until at least
// CN_REFILL_IDLE of its lanes are idle, then takes that many new rays with
// one atomic and resumes; once the queue is drained it runs its last rays out.
#ifndef CN_REFILL_IDLE
#define CN_REFILL_IDLE 8
#endif

__device__ __forceinline__ uint32_t lanemask_lt() { return (1u << lane_id()) - 1u; }

// Hand the warp's idle lanes their next work items: returns this lane's item
// index (or ~0u) and sets `drained` (warp-uniform) once the queue is used up.
__device__ __forceinline__ uint32_t refill(uint32_t* counter, uint32_t count, bool live, bool& drained) {
    uint32_t idle = __ballot_sync(0xffffffffu, !live);
    if (idle == 0) return ~0u;
    uint32_t base = 0;
    if (lane_id() == 0) base = atomicAdd(counter, uint32_t(__popc(idle)));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base + uint32_t(__popc(idle)) >= count) drained = true;
    if (live) return ~0u;
    uint32_t i = base + __popc(idle & lanemask_lt());
    return i < count ? i : ~0u;
}

// Traversal kernels come in launch variants: B threads per block (the same
// registers per thread: CN_TRAV_MIN_BLOCKS * 128 / B blocks per SM) and S
// stack entries per lane (16 halves a lane's local-memory stack, for trees
// whose node groups need fewer). Every variant walks the same tree to the
// same hits.
template <bool COUNT, int B = BLOCK, int S = TRAVERSAL_STACK>
__global__ void __launch_bounds__(B, CN_ISECT_MIN_BLOCKS * BLOCK / B)
    k_intersect(DeviceScene scene, PathPool pool, uint32_t bounce, uint32_t n0) {
    extern __shared__ uint4 top_levels[];
    stage_top_levels(scene, top_levels, min(pool.top_nodes, TOP_NODES_MAX));  // as the launch sized it
    uint32_t visits = 0, tests = 0;
    const uint32_t count = bounce_paths(pool, bounce, n0);
    const uint32_t* queue = pool.queue[bounce & 1u];
    const uint32_t mask = bounce == 0 ? RAY_MASK_CAMERA : RAY_MASK_ALL;
    uint32_t* fetch = pool.counters + CTR_FETCH_ISECT + bounce;
    uint2 stack[S];
    Walk w;
    Ray ray;
    float tmax = 1e30f, best_b1 = 0.0f, best_b2 = 0.0f;
    uint32_t path = 0, best_inst = LIGHT_NONE, best_prim = 0, crossings = 0, pixel = 0, sample = 0;
    uint32_t qi = 0;          // the ray's queue position (the material sort's key slot)
    bool live = false, drained = false, finished = false;
    // Material sort (when this bounce sorts): each finished ray's key goes to
    // its queue slot and into the key counts, one atomic per distinct key per
    // warp. Called where the whole warp is converged.
    auto flush_keys = [&]() {
        if (!pool.sort_keys) return;
        if (__ballot_sync(0xffffffffu, finished) == 0u) return;
        const uint32_t key = finished ? material_key(scene, pool, best_inst, path, tmax) : 0xffffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, key);
        if (finished) {
            pool.sort_keys[qi] = key;
            if (lane_id() == uint32_t(__ffs(peers) - 1)) atomicAdd(pool.sort_bins + key, uint32_t(__popc(peers)));
        }
        finished = false;
    };
    auto visit = [&](uint32_t, float4 a, float4 b, float4 c, float& tm) {
        uint32_t flags = __float_as_uint(c.w);
        if (!(flags & mask)) return false;
        float t, b1, b2;
        if (!tri_hit(ray, a, b, c, tm, t, b1, b2)) return false;
        uint32_t inst = __float_as_uint(a.w), prim = __float_as_uint(b.w);
        if (!(t < tm || (t == tm && (inst < best_inst || (inst == best_inst && prim < best_prim))))) return false;
        if (!(flags & TRI_OPAQUE)) {
            float opacity = opacity_at(scene, inst, prim, b1, b2);
            bool commit = crossings >= TRANSPARENT_CAP || hash_uniform(pixel, sample, bounce, crossings) < opacity;
            crossings++;
            if (!commit) return false;
        }
        tm = t;
        best_inst = inst;
        best_prim = prim;
        best_b1 = b1;
        best_b2 = b2;
        return false;
    };
    for (;;) {
        if (!drained) {
            uint32_t i = refill(fetch, count, live, drained);
            if (i != ~0u) {
                qi = i;
                path = bounce == 0 ? i : queue[i];
                float4 o = pool.org[path], d = pool.dir[path];
                ray = make_ray(xyz(o), xyz(d));
                tmax = 1e30f;
                best_inst = LIGHT_NONE;
                best_prim = 0;
                best_b1 = best_b2 = 0.0f;
                crossings = 0;
                if (scene.has_nonopaque) {
                    uint2 ps = pool.ps[path];
                    pixel = ps.x;
                    sample = ps.y;
                }
                walk_begin(w, ray);
                live = true;
                if (scene.node_count == 0) {
                    pool.hit[path] = make_uint4(LIGHT_NONE, 0u, 0u, 0u);
                    live = false;
                    finished = true;
                }
            }
        }
        flush_keys();
        if (!__any_sync(0xffffffffu, live)) {
            if (drained) break;
            continue;
        }
        // Walk until enough lanes are idle to refill (all of them once drained).
        const uint32_t want_idle = drained ? 32u : (pool.refill_idle ? pool.refill_idle : uint32_t(CN_REFILL_IDLE));
        for (;;) {
            if (live) {
                int st = walk_step<COUNT, S>(scene, ray, tmax, w, stack, visit, &visits, &tests);
                if (st != WALK_CONTINUE) {
                    if (st == WALK_OVERFLOW) flag_overflow(pool.counters);
                    pool.hit[path] =
                        make_uint4(best_inst, best_prim, __float_as_uint(best_b1), __float_as_uint(best_b2));
                    live = false;
                    finished = true;
                }
            }
            flush_keys();
            if (uint32_t(__popc(__ballot_sync(0xffffffffu, !live))) >= want_idle) break;
        }
    }
    if (COUNT) flush_counts(pool.counters, visits, tests);
}

// The closest-hit stage for scenes whose triangles are all opaque: the same
// persistent, refilling grid as k_intersect, with the triangle tests shared
// by the warp through its triangle queue (trqueue.cuh). Hits are bitwise
// those of k_intersect.
struct IsectSource {
    const PathPool& pool;
    const DeviceScene* scene;
    const uint32_t* queue;
    uint32_t* fetch;
    uint32_t count, bounce;
    __device__ __forceinline__ uint32_t path_of(uint32_t i) const { return bounce == 0 ? i : queue[i]; }
    __device__ __forceinline__ uint32_t next(bool live, bool& drained) { return refill(fetch, count, live, drained); }
    __device__ __forceinline__ void ray(uint32_t i, float3& o, float3& d) const {
        const uint32_t path = path_of(i);
        o = xyz(pool.org[path]);
        d = xyz(pool.dir[path]);
    }
    __device__ __forceinline__ void emit(uint32_t i, uint4 hit, float) const { pool.hit[path_of(i)] = hit; }
    // Material sort: each finished ray's key goes to its queue slot and into
    // the key counts, one atomic per distinct key per warp.
    __device__ __forceinline__ void step(bool finished, uint32_t i, uint32_t inst, float t) const {
        if (!pool.sort_keys) return;
        if (__ballot_sync(0xffffffffu, finished) == 0u) return;
        const uint32_t key = finished ? material_key(*scene, pool, inst, path_of(i), t) : 0xffffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, key);
        if (finished) {
            pool.sort_keys[i] = key;
            if (lane_id() == uint32_t(__ffs(peers) - 1)) atomicAdd(pool.sort_bins + key, uint32_t(__popc(peers)));
        }
    }
    __device__ __forceinline__ uint32_t want_idle(bool drained) const {
        return drained ? 32u : (pool.refill_idle ? pool.refill_idle : uint32_t(CN_REFILL_IDLE));
    }
};

template <bool COUNT, int B = BLOCK, int S = TRAVERSAL_STACK>
__global__ void __launch_bounds__(B, CN_ISECT_MIN_BLOCKS * BLOCK / B)
    k_intersect_queued(DeviceScene scene, PathPool pool, uint32_t bounce, uint32_t n0) {
    extern __shared__ uint4 top_levels[];
    __shared__ TriQueueSmem tqs[B / 32];
    stage_top_levels(scene, top_levels, min(pool.top_nodes, TOP_NODES_MAX));
    uint32_t visits = 0, tests = 0;
    IsectSource src{pool, &scene, pool.queue[bounce & 1u], pool.counters + CTR_FETCH_ISECT + bounce,
                    bounce_paths(pool, bounce, n0), bounce};
    bool overflow = false;
    queued_closest<COUNT, IsectSource, S>(scene, tqs[threadIdx.x >> 5], src,
                                          bounce == 0 ? RAY_MASK_CAMERA : RAY_MASK_ALL, overflow,
                          &visits, &tests);
    if (overflow) flag_overflow(pool.counters);
    if (COUNT) flush_counts(pool.counters, visits, tests);
}

// ---- shade: shade_miss.slang:29-75 and shade_surface.slang:235-521 -----------------

struct Spawn {
    float3 position, below, normal, shading;
    bool front;
};

__device__ __forceinline__ float3 fetch3(const float* a, uint32_t v) {
    return f3(__ldg(a + 3 * v), __ldg(a + 3 * v + 1), __ldg(a + 3 * v + 2));
}

// shade_surface.slang:96-181 (van Antwerpen's rigorous spawn offsets).
__device__ __forceinline__ Spawn spawn_point(const GeomRecord& g, uint32_t prim, float b1, float b2, float3 rd) {
    uint32_t i0 = __ldg(g.indices + 3 * prim), i1 = __ldg(g.indices + 3 * prim + 1), i2 = __ldg(g.indices + 3 * prim + 2);
    float3 v0 = fetch3(g.positions, i0), v1 = fetch3(g.positions, i1), v2 = fetch3(g.positions, i2);
    float3 e1 = v1 - v0, e2 = v2 - v0;
    float3 op = v0 + fma3(f3(b1), e1, b2 * e2);
    float3 on = cross(e1, e2);
    float3 r0 = f3(g.o2w[0][0], g.o2w[0][1], g.o2w[0][2]), r1 = f3(g.o2w[1][0], g.o2w[1][1], g.o2w[1][2]),
           r2 = f3(g.o2w[2][0], g.o2w[2][1], g.o2w[2][2]);
    float3 tw = f3(g.o2w[0][3], g.o2w[1][3], g.o2w[2][3]);
    float3 wp = f3(tw.x + fmaf(r0.x, op.x, fmaf(r0.y, op.y, r0.z * op.z)),
                   tw.y + fmaf(r1.x, op.x, fmaf(r1.y, op.y, r1.z * op.z)),
                   tw.z + fmaf(r2.x, op.x, fmaf(r2.y, op.y, r2.z * op.z)));
    float3 w0 = f3(g.w2o[0][0], g.w2o[0][1], g.w2o[0][2]), w1 = f3(g.w2o[1][0], g.w2o[1][1], g.w2o[1][2]),
           w2 = f3(g.w2o[2][0], g.w2o[2][1], g.w2o[2][2]);
    float3 wn = w0 * on.x + w1 * on.y + w2 * on.z;
    float wscale = rsqrtf(dot(wn, wn));
    wn = wn * wscale;
    const float c0 = 5.9604644775390625e-8f;
    const float c1 = 1.788139769587360206060111522674560546875e-7f;
    const float c2 = 1.19209317972490680404007434844970703125e-7f;
    float3 ext3 = fabs3(e1) + fabs3(e2) + fabs3(e1 - e2);
    float extent = fmaxf(fmaxf(ext3.x, ext3.y), ext3.z);
    float3 oerr = fma3(f3(c0), fabs3(v0), f3(c1 * extent));
    float3 aop = fabs3(op);
    float3 werr = fma3(f3(c1), f3(dot(fabs3(r0), aop), dot(fabs3(r1), aop), dot(fabs3(r2), aop)), c2 * fabs3(tw));
    float3 awp = fabs3(wp);
    oerr = fma3(f3(c2),
                f3(dot(fabs3(w0), awp) + fabsf(g.w2o[0][3]), dot(fabs3(w1), awp) + fabsf(g.w2o[1][3]),
                   dot(fabs3(w2), awp) + fabsf(g.w2o[2][3])),
                oerr);
    float woff = dot(werr, fabs3(wn));
    float ooff = dot(oerr, fabs3(on));
    woff = fmaf(wscale, ooff, woff);
    Spawn sp;
    sp.front = dot(wn, rd) < 0.0f;
    if (dot(wn, rd) > 0.0f) wn = -wn;
    float3 n0 = fetch3(g.normals, i0), n1 = fetch3(g.normals, i1), n2 = fetch3(g.normals, i2);
    float3 os = n0 + b1 * (n1 - n0) + b2 * (n2 - n0);
    float3 sh = normalize(w0 * os.x + w1 * os.y + w2 * os.z);
    if (dot(sh, wn) < 0.0f) sh = -sh;
    sp.position = fma3(f3(woff), wn, wp);
    sp.below = fma3(f3(-woff), wn, wp);
    sp.normal = wn;
    sp.shading = sh;
    return sp;
}

__device__ __forceinline__ void load_material(const Material* rec, Material& m) {
    const uint4* src = reinterpret_cast<const uint4*>(rec);
    uint4* dst = reinterpret_cast<uint4*>(&m);
#pragma unroll
    for (int k = 0; k < int(sizeof(Material) / 16); ++k) dst[k] = __ldg(src + k);
}

// shade_surface.slang:59-63: the open guides record this surface.
__device__ __forceinline__ void record_guides(const PathPool& pool, uint32_t path, float3 w, float3 albedo, float3 n) {
    float4 a = pool.aov_albedo[path], b = pool.aov_normal[path];
    pool.aov_albedo[path] = make_float4(a.x + w.x * albedo.x, a.y + w.y * albedo.y, a.z + w.z * albedo.z, a.w);
    pool.aov_normal[path] = make_float4(b.x + w.x * n.x, b.y + w.y * n.y, b.z + w.z * n.z, b.w);
}

__device__ __forceinline__ float luminance(float3 c) { return 0.2722287f * c.x + 0.6740818f * c.y + 0.0536895f * c.z; }

// The path's open training record learns the radiance gathered so far (the
// next vertex's snapshot; everything after it is the record's target).
__device__ __forceinline__ void close_record(const PathPool& pool, uint32_t path, float4 rad) {
    uint32_t rec = pool.guide_rec[path];
    if (rec != ~0u) {
        reinterpret_cast<guide::Record*>(pool.sink->records)[rec].q2.w = luminance(xyz(rad));
        pool.guide_rec[path] = ~0u;
    }
}

// LAYERS false: the scene has no material with coat, fuzz, transmission or
// thin walls, so those weights are the constant zero here and the compiler
// drops their lobes (fewer registers and spills: shading 15 % faster on the
// material chart). The arithmetic is the same but for the compiler's choice
// of fused multiply-adds once the zeros fold: films agree within 2 ulps.
template <bool AOV, bool GUIDE, bool LAYERS>
__global__ void __launch_bounds__(BLOCK, LAYERS ? CN_SHADE_LAYERED_MIN_BLOCKS : CN_SHADE_MIN_BLOCKS)
    k_shade(DeviceScene scene, PathPool pool, uint32_t bounce,
                                                 uint32_t max_bounces, uint32_t light_sampling, uint32_t n0,
                                                 uint32_t part) {
    // part 0: the whole bounce; on a sorted bounce, 1: the misses and
    // layer-free hits (keys below SORT_LAYERS), 2: the layered hits.
    uint32_t count = bounce_paths(pool, bounce, n0);
    uint32_t first = 0;
    if (part != 0) {
        const uint32_t split = min(pool.sort_bins[SORT_LAYERS - 1u], count);  // the end of the layer-free keys
        if (part == 1) count = split;
        else first = split;
    }
    const uint32_t* queue = pool.queue[bounce & 1u];
    uint32_t* next_queue = pool.queue[(bounce + 1u) & 1u];
    uint32_t* fetch = pool.counters + (part == 2 ? CTR_FETCH_SHADE_LAYERS : CTR_FETCH_SHADE) + bounce;
    for (;;) {
        uint32_t base = first + warp_fetch(fetch);
        if (base >= count) break;
        uint32_t i = base + lane_id();
        bool push_ray = false, push_shadow = false;
        uint32_t path = 0;
        ShadowRay sr;
        if (i < count) {
            path = pool.order ? pool.order[i] : (bounce == 0 ? i : queue[i]);
            uint4 h = pool.hit[path];
            float4 d4 = pool.dir[path];
            float3 dir = xyz(d4);
            float4 t4 = pool.thr[path];
            float3 thr = xyz(t4);
            float4 rad = pool.rad[path];
            if (GUIDE) close_record(pool, path, rad);
            if (h.x == LIGHT_NONE) {
                // shade_miss.slang:29-75
                float weight = 1.0f;
                if (t4.w > 0.0f) {
                    if (light_sampling == CENOTE_LIGHT_SAMPLING_NEE) weight = 0.0f;
                    else if (light_sampling == CENOTE_LIGHT_SAMPLING_MIS)
                        weight = power_heuristic(t4.w, scene.select_prob * env_pdf(scene, dir));
                }
                if (AOV) {
                    // shade_miss.slang:52-66: depth +inf on a camera ray; the
                    // open guides record the environment as white albedo.
                    const bool camera_ray = t4.w == 0.0f;
                    if (camera_ray) pool.aov_depth[path] += __int_as_float(0x7f800000);
                    float3 guide = camera_ray ? f3(1.0f) : xyz(pool.aov_guide[path]);
                    float4 a = pool.aov_albedo[path];
                    pool.aov_albedo[path] = make_float4(a.x + guide.x, a.y + guide.y, a.z + guide.z, a.w);
                }
                float3 c = thr * env_radiance(scene, dir) * weight;
                pool.rad[path] = make_float4(rad.x + c.x, rad.y + c.y, rad.z + c.z, rad.w + 1.0f);
            } else {
                const uint32_t inst = h.x, prim = h.y;
                const float b1 = __uint_as_float(h.z), b2 = __uint_as_float(h.w);
                uint2 ps = pool.ps[path];
                const uint32_t pixel = ps.x, sample = ps.y;
                float3 origin = xyz(pool.org[path]);
                // The instance record is read field by field where used (all
                // lanes of a sorted warp mostly share it, so the reads hit L1):
                // a register copy of its 144 bytes made the kernel spill more.
                const GeomRecord& g = scene.geometry[inst];
                Material mat;
                load_material(scene.materials + inst, mat);
                if (!LAYERS) {
                    mat.coat_weight = 0.0f;
                    mat.fuzz_weight = 0.0f;
                    mat.transmission_weight = 0.0f;
                    mat.thin_walled = 0u;
                }
                // Textured parameters resolve once at the hit's UV
                // (shade_surface.slang:249-252).
                const bool normal_map = mat.normal_texture != TEXTURE_NONE;
                float2 uv = make_float2(0.0f, 0.0f);
                if (has_parameter_maps(mat) || normal_map) {
                    uv = interpolate_uv(g.uvs, g.indices, prim, b1, b2);
                    resolve_material(scene, mat, uv);
                }
                Spawn sp = spawn_point(g, prim, b1, b2, dir);
                if (normal_map)
                    sp.shading = mapped_shading_normal(scene, inst, prim, uv, mat.normal_texture, sp.shading, sp.normal);
                uint32_t medium = bounce == 0 ? MEDIUM_NONE : (pool.state[path] & 0xffffffu);
                if (medium != MEDIUM_NONE) {
                    const Material& in = scene.materials[medium];
                    float depth = __ldg(&in.transmission_depth);
                    if (depth > 0.0f) {
                        float3 tc = f3(__ldg(&in.transmission_color[0]), __ldg(&in.transmission_color[1]),
                                       __ldg(&in.transmission_color[2]));
                        float3 sigma = -log3(clamp3(tc, 1e-4f, 1.0f)) / depth;
                        thr = thr * exp3(-sigma * length(origin - sp.position));
                    }
                }
                float3 contribution = f3(0.0f);
                if (g.light != LIGHT_NONE && sp.front) {
                    float weight = 1.0f;
                    if (t4.w > 0.0f) {
                        if (light_sampling == CENOTE_LIGHT_SAMPLING_NEE) weight = 0.0f;
                        else if (light_sampling == CENOTE_LIGHT_SAMPLING_MIS) {
                            float3 delta = sp.position - origin;
                            float cl = fabsf(dot(sp.normal, dir));
                            float lp = __ldg(&scene.lights[g.light + prim].pdf);
                            float nee = (1.0f - scene.select_prob) * lp * dot(delta, delta) / cl;
                            weight = power_heuristic(t4.w, nee);
                        }
                    }
                    contribution = thr * ld3(mat.emission) * weight;
                }
                Frame frame(sp.shading);
                float3 wo = frame.to_local(-dir);
                Closure cl = resolve_closure(scene.bsdf_tables, mat, wo, medium == inst);
                // The learned guide's share of the one-sample MIS with BSDF
                // sampling: none on near-specular vertices, where the BSDF is the
                // better proposal and a broad mixture would waste its samples.
                float g_alpha = 0.0f;
                const float* g_out = nullptr;
                if (GUIDE) {
                    g_out = pool.guide_out + size_t(path) * guide::OUT_ACT;
                    if (cl.w_diffuse + cl.w_fuzz > 0.0f || cl.alpha > 0.05f) g_alpha = pool.sink->fraction;
                }
                // Guides (shade_surface.slang:322-340): camera rays are fully
                // open; the first hit records camera-plane depth.
                float3 guide = f3(0.0f), aov_alb = f3(0.0f);
                if (AOV) {
                    guide = bounce == 0 ? f3(1.0f) : xyz(pool.aov_guide[path]);
                    if (bounce == 0) pool.aov_depth[path] += length(origin - sp.position) * d4.w;
                    aov_alb = saturate3(cl.aov_albedo);
                }
                if (bounce + 1 >= max_bounces) {
                    if (AOV && any_pos(guide)) record_guides(pool, path, guide, aov_alb, sp.shading);
                    pool.rad[path] = make_float4(rad.x + contribution.x, rad.y + contribution.y, rad.z + contribution.z,
                                                 rad.w + 1.0f);
                } else {
                    // Next-event estimation (shade_surface.slang:363-446): one candidate,
                    // the environment or a light from the list, then one shared
                    // eval/pdf of the closure for it.
                    const float env_prob = scene.select_prob;
                    if (light_sampling != CENOTE_LIGHT_SAMPLING_BSDF && (scene.light_count > 0 || env_prob > 0.0f)) {
                        float u_light = sample_1d(pixel, sample, bounce_dim(bounce, NEE_LIGHT));
                        float2 u_point = sample_2d(pixel, sample, bounce_dim(bounce, NEE_POINT));
                        float3 cdir, crad;
                        float cpdf, nee, ctmax = 1e30f;
                        bool cdelta = false;
                        uint32_t clight = LIGHT_NONE, cprim = 0, cleaf = 0xffffffffu;
                        if (u_light < env_prob) {
                            EnvSample cand = env_sample(scene, u_point);
                            cdir = cand.direction;
                            crad = cand.radiance;
                            cpdf = cand.pdf;
                            nee = env_prob * cand.pdf;
                        } else {
                            float u_list = (u_light - env_prob) / (1.0f - env_prob);
                            LightConn cand = sample_lights(scene.lights, scene.light_count, u_list, u_point, sp.position);
                            if (!cand.delta) {
                                // A textured emitter evaluates its map at the sampled point
                                // (shade_surface.slang:405-418).
                                uint32_t em = __ldg(&scene.materials[cand.instance].emission_texture);
                                if (em != TEXTURE_NONE)
                                    cand.radiance = cand.radiance * emission_map(scene, em, cand.instance,
                                                                                 cand.primitive, cand.b1, cand.b2);
                            }
                            cdir = cand.direction;
                            crad = cand.radiance;
                            cpdf = cand.pdf;
                            nee = (1.0f - env_prob) * cand.pdf;
                            cdelta = cand.delta;
                            clight = cand.instance;
                            cprim = cand.primitive;
                            ctmax = cand.tmax;
                            if (!cand.delta) cleaf = __ldg(scene.light_leaf + cand.record);
                        }
                        float3 wl = frame.to_local(cdir);
                        bool through = dot(cdir, sp.normal) < 0.0f;
                        if (cpdf > 0.0f && wl.z != 0.0f && (wl.z < 0.0f) == through) {
                            // A delta light has no competing BSDF strategy: weight 1.
                            bool mis = !cdelta && light_sampling == CENOTE_LIGHT_SAMPLING_MIS;
                            EvalPdf ep = eval_pdf(cl, wl, wo);
                            float p_scatter = ep.pdf;
                            if (GUIDE && g_alpha > 0.0f)
                                p_scatter = g_alpha * guide::mixture_pdf_act(g_out, cdir) + (1.0f - g_alpha) * ep.pdf;
                            float w = mis ? power_heuristic(nee, p_scatter) : 1.0f;
                            float3 unshadowed = thr * crad * ep.f * fabsf(wl.z) * (w / nee);
                            if (any_pos(unshadowed)) {
                                float3 sorg = through ? sp.below : sp.position;
                                push_shadow = true;
                                sr.org[0] = sorg.x; sr.org[1] = sorg.y; sr.org[2] = sorg.z;
                                sr.tmax = ctmax;
                                sr.dir[0] = cdir.x; sr.dir[1] = cdir.y; sr.dir[2] = cdir.z;
                                sr.path = path;
                                sr.contrib[0] = unshadowed.x; sr.contrib[1] = unshadowed.y; sr.contrib[2] = unshadowed.z;
                                sr.light = clight;
                                sr.primitive = cprim;
                                sr.leaf = cleaf;
                            }
                        }
                    }
                    float u_lobe = sample_1d(pixel, sample, bounce_dim(bounce, BSDF_LOBE));
                    float2 u = sample_2d(pixel, sample, bounce_dim(bounce, BSDF_DIR));
                    BsdfSample sc;
                    float3 fsc = f3(0.0f);
                    bool have;
                    if (GUIDE && g_alpha > 0.0f && u_lobe < g_alpha) {
                        // A direction from the guide's mixture (the pick's leftover
                        // chooses the lobe); lobe labels follow the hemisphere.
                        float3 d = guide::mixture_sample_act(g_out, u_lobe / g_alpha, u.x, u.y);
                        sc.wi = frame.to_local(d);
                        sc.pdf = 0.0f;
                        sc.lobe = sc.wi.z < 0.0f ? LOBE_TRANSMISSION : LOBE_DIFFUSE;
                        have = true;
                    } else {
                        const float ub = g_alpha > 0.0f ? (u_lobe - g_alpha) / (1.0f - g_alpha) : u_lobe;
                        have = sample_bsdf_dir(cl, wo, ub, u.x, u.y, sc);
                    }
                    if (have) {
                        EvalPdf ep = eval_pdf(cl, sc.wi, wo);
                        sc.pdf = ep.pdf;
                        fsc = ep.f;
                        if (GUIDE && g_alpha > 0.0f)
                            sc.pdf = g_alpha * guide::mixture_pdf_act(g_out, frame.to_world(sc.wi)) + (1.0f - g_alpha) * ep.pdf;
                    }
                    float3 wiw = frame.to_world(sc.wi);
                    float3 scattered = f3(0.0f);
                    if (sc.pdf > 0.0f && sc.wi.z != 0.0f && (sc.wi.z > 0.0f) == (dot(wiw, sp.normal) > 0.0f))
                        scattered = thr * fsc * (fabsf(sc.wi.z) / sc.pdf);
                    float survival = max3(scattered);
                    bool terminal = false;
                    if (survival <= 0.0f) {
                        terminal = true;
                    } else if (bounce >= ROULETTE_START) {
                        survival = fminf(1.0f, survival);
                        if (sample_1d(pixel, sample, bounce_dim(bounce, RR)) >= survival) terminal = true;
                        else scattered = scattered / survival;
                    }
                    if (terminal) {
                        if (AOV && any_pos(guide)) record_guides(pool, path, guide, aov_alb, sp.shading);
                        pool.rad[path] = make_float4(rad.x + contribution.x, rad.y + contribution.y,
                                                     rad.z + contribution.z, rad.w + 1.0f);
                    } else {
                        if (AOV) {
                            // shade_surface.slang:488-503: the sampled lobe splits the
                            // open guides between this surface and the scattered ray.
                            float rec = aov_record_fraction(cl, sc.lobe);
                            if (rec > 0.0f && any_pos(guide)) record_guides(pool, path, guide * rec, aov_alb, sp.shading);
                            pool.aov_guide[path] = f4(guide * (1.0f - rec) * aov_pass_tint(cl, sc.lobe), 0.0f);
                        }
                        if (sc.lobe == LOBE_TRANSMISSION && mat.thin_walled == 0)
                            medium = medium == inst ? MEDIUM_NONE : inst;
                        pool.org[path] = f4(sc.wi.z < 0.0f ? sp.below : sp.position, 0.0f);
                        pool.dir[path] = f4(wiw, 0.0f);
                        pool.thr[path] = f4(scattered, sc.pdf);
                        pool.state[path] = (sc.lobe << 24) | (medium & 0xffffffu);
                        push_ray = true;
                        if (GUIDE && g_alpha > 0.0f && pool.sink->records &&
                            hash_uniform(pixel, sample, bounce, 0x6a09u) < pool.sink->rate) {
                            uint32_t idx = atomicAdd(pool.sink->count, 1u);
                            if (idx < pool.sink->capacity) {
                                guide::Record rc;
                                rc.q0 = f4(sp.position, sc.pdf);
                                rc.q1 = f4(sp.normal, luminance(scattered));
                                rc.q2 = f4(-dir, -1.0f);
                                rc.q3 = f4(wiw, __uint_as_float(path));
                                reinterpret_cast<guide::Record*>(pool.sink->records)[idx] = rc;
                                pool.guide_rec[path] = idx;
                            }
                        }
                        if (any_pos(contribution))
                            pool.rad[path] =
                                make_float4(rad.x + contribution.x, rad.y + contribution.y, rad.z + contribution.z, rad.w);
                    }
                }
            }
        }
        uint32_t slot = warp_push(pool.counters + CTR_RAYS + bounce + 1, push_ray);
        if (push_ray) {
            if (slot < pool.capacity) next_queue[slot] = path;
            else flag_overflow(pool.counters);
        }
        uint32_t sslot = warp_push(pool.counters + CTR_SHADOWS + bounce, push_shadow);
        if (push_shadow) {
            if (sslot < pool.capacity) {
                float4* dst = reinterpret_cast<float4*>(pool.shadows + sslot);
                const float4* src = reinterpret_cast<const float4*>(&sr);
                dst[0] = src[0];
                dst[1] = src[1];
                dst[2] = src[2];
                dst[3] = src[3];
            } else {
                flag_overflow(pool.counters);
            }
        }
    }
}

// ---- trace_shadow (trace_shadow.slang:29-72) ----------------------------------------

template <bool COUNT, int B = BLOCK, int S = TRAVERSAL_STACK>
__global__ void __launch_bounds__(B, CN_TRAV_MIN_BLOCKS * BLOCK / B)
    k_shadow(DeviceScene scene, PathPool pool, uint32_t bounce) {
    extern __shared__ uint4 top_levels[];
    stage_top_levels(scene, top_levels, min(pool.top_nodes, TOP_NODES_MAX));  // as the launch sized it
    const uint32_t count = min(pool.counters[CTR_SHADOWS + bounce], pool.capacity);
    uint32_t* fetch = pool.counters + CTR_FETCH_SHADOW + bounce;
    uint32_t visits = 0, tests = 0;
    uint2 stack[S];
    ShadowQuery q;
    Ray ray;
    float3 contrib = f3(0.0f);
    uint32_t path = 0;
    bool live = false, drained = false;
    for (;;) {
        if (!drained) {
            uint32_t i = refill(fetch, count, live, drained);
            if (i != ~0u) {
                const float4* rec = reinterpret_cast<const float4*>(pool.shadows + i);
                float4 q0 = rec[0], q1 = rec[1], q2 = rec[2], q3 = rec[3];
                path = __float_as_uint(q1.w);
                contrib = xyz(q2);
                ray = make_ray(xyz(q0), xyz(q1));
                shadow_begin(scene, ray, q0.w, __float_as_uint(q2.w), __float_as_uint(q3.x), __float_as_uint(q3.y), q);
                live = true;
            }
        }
        if (!__any_sync(0xffffffffu, live)) {
            if (drained) break;
            continue;
        }
        const uint32_t want_idle = drained ? 32u : (pool.refill_idle ? pool.refill_idle : uint32_t(CN_REFILL_IDLE));
        for (;;) {
            if (live) {
                int st = shadow_step<COUNT, S>(scene, ray, q, stack, &visits, &tests);
                if (st == WALK_OVERFLOW) {
                    flag_overflow(pool.counters);
                    live = false;
                } else if (st == WALK_DONE) {
                    float atten = shadow_result(q);
                    if (atten >= 0.0f) {
                        float4 r = pool.rad[path];
                        pool.rad[path] = make_float4(r.x + contrib.x * atten, r.y + contrib.y * atten,
                                                     r.z + contrib.z * atten, r.w);
                    }
                    live = false;
                }
            }
            if (uint32_t(__popc(__ballot_sync(0xffffffffu, !live))) >= want_idle) break;
        }
    }
    if (COUNT) flush_counts(pool.counters, visits, tests);
}

// The shadow stage for scenes whose triangles are all opaque: k_shadow's
// persistent, refilling grid with the triangle tests shared by the warp
// through its triangle queue (trqueue.cuh). Radiance is bitwise k_shadow's.
struct ShadowSource {
    const DeviceScene& scene;
    const PathPool& pool;
    uint32_t* fetch;
    uint32_t count;
    __device__ __forceinline__ uint32_t next(bool live, bool& drained) { return refill(fetch, count, live, drained); }
    __device__ __forceinline__ bool begin(uint32_t i, Ray& ray, AnyQuery& a) const {
        const float4* rec = reinterpret_cast<const float4*>(pool.shadows + i);
        const float4 q0 = rec[0], q1 = rec[1], q2 = rec[2], q3 = rec[3];
        ray = make_ray(xyz(q0), xyz(q1));
        const uint32_t light = __float_as_uint(q2.w), leaf = __float_as_uint(q3.y);
        a.occluded = false;
        a.light = light;
        a.lprim = __float_as_uint(q3.x);
        a.tm = q0.w;
        a.leaf = 0xffffffffu;
        if (light != LIGHT_NONE && leaf == 0xffffffffu) return false;  // no leaf: the closest-hit query
        if (leaf < scene.tri_count) {
            const float4* tp = scene.tris + 3u * leaf;
            float t, b1, b2;
            if (tri_hit(ray, __ldg(tp), __ldg(tp + 1), __ldg(tp + 2), q0.w, t, b1, b2)) {
                a.tm = t;
                a.leaf = leaf;
            }
        }
        return true;
    }
    __device__ __forceinline__ void add(uint32_t i, float atten) const {
        const float4* rec = reinterpret_cast<const float4*>(pool.shadows + i);
        const uint32_t path = __float_as_uint(rec[1].w);
        const float4 c = rec[2], r = pool.rad[path];
        pool.rad[path] = make_float4(r.x + c.x * atten, r.y + c.y * atten, r.z + c.z * atten, r.w);
    }
    template <int S>
    __device__ __forceinline__ void closest(uint32_t i, uint2* stack) const {
        const float4* rec = reinterpret_cast<const float4*>(pool.shadows + i);
        const float4 q0 = rec[0], q1 = rec[1], q2 = rec[2], q3 = rec[3];
        const float atten = shadow_query<false, S>(scene, make_ray(xyz(q0), xyz(q1)), q0.w, __float_as_uint(q2.w),
                                                   __float_as_uint(q3.x), __float_as_uint(q3.y), stack);
        if (atten == -2.0f) flag_overflow(pool.counters);
        else if (atten >= 0.0f) add(i, atten);
    }
    __device__ __forceinline__ void emit(uint32_t i, bool visible) const {
        if (visible) add(i, 1.0f);
    }
    __device__ __forceinline__ uint32_t want_idle(bool drained) const {
        return drained ? 32u : (pool.refill_idle ? pool.refill_idle : uint32_t(CN_REFILL_IDLE));
    }
};

template <bool COUNT, int B = BLOCK, int S = TRAVERSAL_STACK>
__global__ void __launch_bounds__(B, CN_TRAV_MIN_BLOCKS * BLOCK / B)
    k_shadow_queued(DeviceScene scene, PathPool pool, uint32_t bounce) {
    extern __shared__ uint4 top_levels[];
    __shared__ TriQueueSmem tqs[B / 32];
    stage_top_levels(scene, top_levels, min(pool.top_nodes, TOP_NODES_MAX));
    uint32_t visits = 0, tests = 0;
    ShadowSource src{scene, pool, pool.counters + CTR_FETCH_SHADOW + bounce,
                     min(pool.counters[CTR_SHADOWS + bounce], pool.capacity)};
    bool overflow = false;
    queued_any<COUNT, ShadowSource, S>(scene, tqs[threadIdx.x >> 5], src, overflow, &visits, &tests);
    if (overflow) flag_overflow(pool.counters);
    if (COUNT) flush_counts(pool.counters, visits, tests);
}

// ---- film --------------------------------------------------------------------------

__device__ __forceinline__ bool finite4(float4 v) {
    return isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && isfinite(v.w);
}

__device__ __forceinline__ float4 add4(float4 a, float4 b) {
    return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}

// accumulate.slang:38-67, all samples of a wave in ascending order.
template <bool AOV>
__global__ void k_accumulate(PathPool pool, FilmTargets film, uint32_t pixel_base, uint32_t count, uint32_t tile_width,
                             uint32_t samples, uint32_t reset) {
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < count; p += gridDim.x * blockDim.x) {
        const uint32_t px = pixel_base + wave_pixel(p, tile_width);
        float4 acc = reset ? zero : film.sum[px];
        float4 alb = zero, nrm = zero;
        float dep = 0.0f;
        if (AOV && !reset) {
            alb = film.albedo[px];
            nrm = film.normal[px];
            dep = film.depth[px];
        }
        for (uint32_t s = 0; s < samples; ++s) {
            const size_t q = size_t(s) * count + p;
            float4 v = pool.rad[q];
            if (!finite4(v)) v = zero;
            acc = (reset && s == 0) ? v : add4(acc, v);
            if (AOV) {
                float4 a = pool.aov_albedo[q], n = pool.aov_normal[q];
                float d = pool.aov_depth[q];
                if (!finite4(a)) a = zero;
                if (!finite4(n)) n = zero;
                if (isnan(d)) d = 0.0f;
                alb = (reset && s == 0) ? a : add4(alb, a);
                nrm = (reset && s == 0) ? n : add4(nrm, n);
                dep = (reset && s == 0) ? d : dep + d;
            }
        }
        film.sum[px] = acc;
        if (AOV) {
            film.albedo[px] = alb;
            film.normal[px] = nrm;
            film.depth[px] = dep;
        }
    }
}

// A multi-job wave's radiance into each job's beauty sums: one thread per
// (segment, pixel), adding the segment's samples in ascending order, as a
// standalone render of the job adds them.
__global__ void k_accumulate_segments(PathPool pool, const WaveSegment* __restrict__ segs, uint32_t nseg,
                                      uint32_t items, const uint32_t* hdr) {
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (hdr) {
        nseg = __ldg(hdr);
        items = __ldg(hdr + 2);
    }
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < items; x += gridDim.x * blockDim.x) {
        const WaveSegment& g = segs[find_segment(segs, nseg, x, true)];
        const uint32_t p = x - g.pixel_start, px = g.pixel_base + p;
        float4 acc = g.reset ? zero : g.film[px];
        for (uint32_t s = 0; s < g.samples; ++s) {
            float4 v = pool.rad[g.start + s * g.pixel_count + p];
            if (!finite4(v)) v = zero;
            acc = (g.reset && s == 0) ? v : add4(acc, v);
        }
        g.film[px] = acc;
    }
}

__global__ void k_resolve(const float4* __restrict__ sum, float4* __restrict__ avg, uint32_t n, float samples) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        float4 v = sum[p];
        avg[p] = make_float4(v.x / samples, v.y / samples, v.z / samples, v.w / samples);
    }
}

// The display transform of crates/cenote/shaders/tonemap.slang:16-99 into
// packed RGBA8: exposure, ACEScg -> linear Rec.709, Stephen Hill's analytic
// RRT+ODT fit (BakingLab; its published matrices and rational curve), sRGB
// transfer, round to 8 bits (R in the low byte). Each matrix row is summed
// left to right.
__device__ __forceinline__ float3 mat3_row_sum(const float m[3][3], float3 v) {
    return f3((m[0][0] * v.x + m[0][1] * v.y) + m[0][2] * v.z, (m[1][0] * v.x + m[1][1] * v.y) + m[1][2] * v.z,
              (m[2][0] * v.x + m[2][1] * v.y) + m[2][2] * v.z);
}

__device__ __forceinline__ uint32_t quantize8(float c) {
    return uint32_t(rintf(fminf(fmaxf(c, 0.0f), 1.0f) * 255.0f));
}

__device__ __forceinline__ float srgb_encode(float c) {
    return c <= 0.0031308f ? 12.92f * c : 1.055f * powf(c, 1.0f / 2.4f) - 0.055f;
}

__global__ void k_tonemap(const float4* __restrict__ avg, uint32_t* __restrict__ out, uint32_t n, float exposure) {
    const float SRGB_FROM_ACESCG[3][3] = {{1.705050993f, -0.621792121f, -0.083258872f},
                                          {-0.130256418f, 1.140804737f, -0.010548319f},
                                          {-0.024003357f, -0.128968976f, 1.152972333f}};
    const float IN[3][3] = {{0.59719f, 0.35458f, 0.04823f}, {0.07600f, 0.90834f, 0.01566f}, {0.02840f, 0.13383f, 0.83777f}};
    const float OUT[3][3] = {{1.60475f, -0.53108f, -0.07367f}, {-0.10208f, 1.10813f, -0.00605f},
                             {-0.00327f, -0.07276f, 1.07602f}};
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        float4 a = avg[p];
        float3 v = mat3_row_sum(IN, mat3_row_sum(SRGB_FROM_ACESCG, f3(a.x * exposure, a.y * exposure, a.z * exposure)));
        float3 num = v * (v + f3(0.0245786f)) - f3(0.000090537f);
        float3 den = v * (0.983729f * v + f3(0.4329510f)) + f3(0.238081f);
        float3 d = saturate3(mat3_row_sum(OUT, num / den));
        out[p] = quantize8(srgb_encode(d.x)) | quantize8(srgb_encode(d.y)) << 8 | quantize8(srgb_encode(d.z)) << 16 |
                 255u << 24;
    }
}

__global__ void k_resolve1(const float* __restrict__ sum, float* __restrict__ avg, uint32_t n, float samples) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) avg[p] = sum[p] / samples;
}

__global__ void k_copy_rad(const float4* __restrict__ rad, float4* __restrict__ out, uint32_t base, uint32_t count,
                           uint32_t tile_width) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < count; p += gridDim.x * blockDim.x)
        out[base + wave_pixel(p, tile_width)] = rad[p];
}

// ---- material sort -----------------------------------------------------------------
// Shading in key order keeps a warp on one material: one closure path, one
// set of textures, neighbouring vertices. k_intersect writes each ray's key
// and counts it (one atomic per distinct key per warp, __match_any_sync) as
// the ray finishes, the counts become offsets in one block, and the scatter
// hands each key's paths consecutive slots.

__device__ __forceinline__ uint32_t sort_count(const PathPool& pool, uint32_t bounce, uint32_t n0) {
    return bounce_paths(pool, bounce, n0);
}

// One block of 1024 threads: exclusive prefix sums of the SORT_BINS counts.
__global__ void __launch_bounds__(1024) k_sort_scan(uint32_t* bins) {
    constexpr uint32_t PER = SORT_BINS / 1024u;
    __shared__ uint32_t warp_sums[32];
    uint32_t v[PER], local = 0;
#pragma unroll
    for (uint32_t k = 0; k < PER; ++k) {
        v[k] = bins[threadIdx.x * PER + k];
        local += v[k];
    }
    uint32_t incl = local;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane_id() >= uint32_t(o)) incl += y;
    }
    if (lane_id() == 31u) warp_sums[threadIdx.x >> 5] = incl;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t w = warp_sums[threadIdx.x], wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane_id() >= uint32_t(o)) wi += y;
        }
        warp_sums[threadIdx.x] = wi - w;
    }
    __syncthreads();
    uint32_t run = warp_sums[threadIdx.x >> 5] + incl - local;
#pragma unroll
    for (uint32_t k = 0; k < PER; ++k) {
        bins[threadIdx.x * PER + k] = run;
        run += v[k];
    }
}

__global__ void __launch_bounds__(BLOCK) k_sort_scatter(PathPool pool, uint32_t bounce, uint32_t n0) {
    const uint32_t count = sort_count(pool, bounce, n0);
    const uint32_t* queue = pool.queue[bounce & 1u];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < count; base += stride) {
        const uint32_t i = base + lane_id();
        const bool valid = i < count;
        const uint32_t key = valid ? pool.sort_keys[i] : 0xffffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, key);
        const uint32_t leader = uint32_t(__ffs(peers) - 1);
        uint32_t slot = 0;
        if (valid && lane_id() == leader) slot = atomicAdd(pool.sort_bins + key, uint32_t(__popc(peers)));
        slot = __shfl_sync(0xffffffffu, slot, leader);
        if (valid) pool.order[slot + __popc(peers & ((1u << lane_id()) - 1u))] = bounce == 0 ? i : queue[i];
    }
}

// Fold one wave's queue counters into the renderer's running totals:
// tally[0] += extension rays, tally[1] += shadow rays, tally[2] |= overflow.
__global__ void k_tally(const uint32_t* counters, unsigned long long* tally, uint32_t n0, uint32_t max_bounces) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned long long rays = n0 ? n0 : counters[CTR_RAYS], shadows = 0;
    for (uint32_t b = 1; b < max_bounces; ++b) rays += counters[CTR_RAYS + b];
    for (uint32_t b = 0; b < max_bounces; ++b) shadows += counters[CTR_SHADOWS + b];
    tally[0] += rays;
    tally[1] += shadows;
    tally[2] |= counters[CTR_OVERFLOW];
    tally[3] += *reinterpret_cast<const unsigned long long*>(counters + CTR_VISITS);
    tally[4] += *reinterpret_cast<const unsigned long long*>(counters + CTR_TESTS);
    tally[5] += *reinterpret_cast<const unsigned long long*>(counters + CTR_HITS);
}

// One warp-aggregated 64-bit add per warp of the rays of bounce `bounce`
// whose closest hit is a surface.
__global__ void k_count_hits(PathPool pool, uint32_t bounce, uint32_t n0) {
    const uint32_t count = bounce_paths(pool, bounce, n0);
    const uint32_t* queue = pool.queue[bounce & 1u];
    unsigned long long hits = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint32_t path = bounce == 0 ? i : queue[i];
        hits += pool.hit[path].x != LIGHT_NONE ? 1u : 0u;
    }
    for (int o = 16; o > 0; o >>= 1) hits += __shfl_xor_sync(0xffffffffu, hits, o);
    if (lane_id() == 0 && hits)
        atomicAdd(reinterpret_cast<unsigned long long*>(pool.counters + CTR_HITS), hits);
}

}  // namespace

namespace {
__global__ void k_advance(uint32_t* counter, uint32_t n) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *counter += n;
}
}  // namespace

void launch_advance(uint32_t* counter, uint32_t n, cudaStream_t stream) { k_advance<<<1, 32, 0, stream>>>(counter, n); }

void launch_tally(const PathPool& pool, unsigned long long* tally, uint32_t n0, uint32_t max_bounces,
                  cudaStream_t stream) {
    k_tally<<<1, 32, 0, stream>>>(pool.counters, tally, n0, max_bounces);
}

void launch_count_hits(const PathPool& pool, uint32_t bounce, uint32_t n0, cudaStream_t stream) {
    k_count_hits<<<1184, BLOCK, 0, stream>>>(pool, bounce, n0);
}

// The traversal launch variants (block size, stack entries); index =
// PathPool::trav_variant, the grids in LaunchShape::trav.
template <int V> struct TravVariant;
template <> struct TravVariant<0> { static constexpr int B = 128, S = 32; };
template <> struct TravVariant<1> { static constexpr int B = 128, S = 16; };
template <> struct TravVariant<2> { static constexpr int B = 256, S = 32; };
template <> struct TravVariant<3> { static constexpr int B = 256, S = 16; };

// Resident blocks per SM of kernel `k` with `block` threads and `smem`
// dynamic shared memory, times the SM count.
template <class K>
int grid_for(K k, int block, size_t smem, int sms) {
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, block, smem);
    return sms * (occ > 0 ? occ : 1);
}

template <int V>
void trav_grids(LaunchShape& ls, int sms) {
    constexpr int B = TravVariant<V>::B, S = TravVariant<V>::S;
    const size_t top = TOP_NODES_MAX * 80u;
    ls.trav[V][TRAV_ISECT] = grid_for(k_intersect<false, B, S>, B, top, sms);
    // The queued kernels' own shared memory leaves fewer blocks room for the
    // staged top levels: size their grids for the launch's dynamic memory.
    ls.trav[V][TRAV_ISECT_QUEUED] = grid_for(k_intersect_queued<false, B, S>, B, 0, sms);
    ls.trav[V][TRAV_ISECT_QUEUED_TOP] = grid_for(k_intersect_queued<false, B, S>, B, top, sms);
    ls.trav[V][TRAV_SHADOW] = grid_for(k_shadow<false, B, S>, B, top, sms);
    ls.trav[V][TRAV_SHADOW_QUEUED] = grid_for(k_shadow_queued<false, B, S>, B, 0, sms);
    ls.trav[V][TRAV_SHADOW_QUEUED_TOP] = grid_for(k_shadow_queued<false, B, S>, B, top, sms);
}

LaunchShape launch_shape(int device) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    LaunchShape ls;
    ls.block = BLOCK;
    trav_grids<0>(ls, sms);
    trav_grids<1>(ls, sms);
    trav_grids<2>(ls, sms);
    trav_grids<3>(ls, sms);
    ls.grid_isect = ls.trav[0][TRAV_ISECT];
    ls.grid_isect_queued = ls.trav[0][TRAV_ISECT_QUEUED];
    ls.grid_isect_queued_top = ls.trav[0][TRAV_ISECT_QUEUED_TOP];
    ls.grid_shadow = ls.trav[0][TRAV_SHADOW];
    ls.grid_shadow_queued = ls.trav[0][TRAV_SHADOW_QUEUED];
    ls.grid_shadow_queued_top = ls.trav[0][TRAV_SHADOW_QUEUED_TOP];
    ls.grid_shade = grid_for(k_shade<true, false, true>, BLOCK, 0, sms);
    ls.grid_shade_free = grid_for(k_shade<true, false, false>, BLOCK, 0, sms);
    ls.grid_stream = sms * 8;
    return ls;
}

void launch_wave_begin(const PathPool& pool, const WaveParams& wp, const LaunchShape& ls, cudaStream_t stream) {
    cudaMemsetAsync(pool.counters, 0, CTR_COUNT * sizeof(uint32_t), stream);
    k_raygen<<<ls.grid_stream, BLOCK, 0, stream>>>(pool, wp);
}

void launch_wave_begin_segments(const PathPool& pool, const WaveSegment* segs, uint32_t nseg, uint32_t paths,
                                const uint32_t* hdr, const LaunchShape& ls, cudaStream_t stream) {
    cudaMemsetAsync(pool.counters, 0, CTR_COUNT * sizeof(uint32_t), stream);
    k_raygen_segments<<<ls.grid_stream, BLOCK, 0, stream>>>(pool, segs, nseg, paths, hdr);
}

void launch_accumulate_segments(const PathPool& pool, const WaveSegment* segs, uint32_t nseg, uint32_t items,
                                const uint32_t* hdr, cudaStream_t stream) {
    const uint32_t grid = hdr ? 4096u : (items == 0 ? 1u : min(4096u, (items + 255u) / 256u));
    k_accumulate_segments<<<grid, 256, 0, stream>>>(pool, segs, nseg, items, hdr);
}

template <int V>
void launch_intersect_v(const DeviceScene& scene, const PathPool& pool, uint32_t bounce, uint32_t n0,
                        const LaunchShape& ls, bool count_visits, cudaStream_t stream) {
    constexpr int B = TravVariant<V>::B, S = TravVariant<V>::S;
    const size_t smem = size_t(min(pool.top_nodes, TOP_NODES_MAX)) * 80u;
    if (!scene.has_nonopaque && !pool.per_lane_triangles) {
        const int grid = smem ? ls.trav[V][TRAV_ISECT_QUEUED_TOP] : ls.trav[V][TRAV_ISECT_QUEUED];
        if (count_visits) k_intersect_queued<true, B, S><<<grid, B, smem, stream>>>(scene, pool, bounce, n0);
        else k_intersect_queued<false, B, S><<<grid, B, smem, stream>>>(scene, pool, bounce, n0);
    } else if (count_visits) {
        k_intersect<true, B, S><<<ls.trav[V][TRAV_ISECT], B, smem, stream>>>(scene, pool, bounce, n0);
    } else {
        k_intersect<false, B, S><<<ls.trav[V][TRAV_ISECT], B, smem, stream>>>(scene, pool, bounce, n0);
    }
}

template <int V>
void launch_shadow_v(const DeviceScene& scene, const PathPool& pool, uint32_t bounce, const LaunchShape& ls,
                     bool count_visits, cudaStream_t stream) {
    constexpr int B = TravVariant<V>::B, S = TravVariant<V>::S;
    const size_t smem = size_t(min(pool.top_nodes, TOP_NODES_MAX)) * 80u;
    if (!scene.has_nonopaque && !pool.per_lane_triangles) {
        const int grid = smem ? ls.trav[V][TRAV_SHADOW_QUEUED_TOP] : ls.trav[V][TRAV_SHADOW_QUEUED];
        if (count_visits) k_shadow_queued<true, B, S><<<grid, B, smem, stream>>>(scene, pool, bounce);
        else k_shadow_queued<false, B, S><<<grid, B, smem, stream>>>(scene, pool, bounce);
    } else if (count_visits) {
        k_shadow<true, B, S><<<ls.trav[V][TRAV_SHADOW], B, smem, stream>>>(scene, pool, bounce);
    } else {
        k_shadow<false, B, S><<<ls.trav[V][TRAV_SHADOW], B, smem, stream>>>(scene, pool, bounce);
    }
}

// The pool's traversal variant, with a 16-entry stack replaced by 32 entries
// for a tree whose node groups could need 16 or more.
static uint32_t trav_variant(const DeviceScene& scene, const PathPool& pool) {
    uint32_t v = pool.trav_variant < TRAV_VARIANTS ? pool.trav_variant : 0u;
    if (TRAV_VARIANT_STACK[v] == 16 && TRAVERSAL_STACK_DEPTH - int(scene.stack_room) >= 16) v &= ~1u;
    return v;
}

void launch_intersect(const DeviceScene& scene, const PathPool& pool, uint32_t bounce, uint32_t n0,
                      const LaunchShape& ls, bool count_visits, cudaStream_t stream) {
    switch (trav_variant(scene, pool)) {
    case 1: launch_intersect_v<1>(scene, pool, bounce, n0, ls, count_visits, stream); break;
    case 2: launch_intersect_v<2>(scene, pool, bounce, n0, ls, count_visits, stream); break;
    case 3: launch_intersect_v<3>(scene, pool, bounce, n0, ls, count_visits, stream); break;
    default: launch_intersect_v<0>(scene, pool, bounce, n0, ls, count_visits, stream); break;
    }
}

void launch_shade(const DeviceScene& scene, const PathPool& pool, uint32_t bounce, const WaveParams& wp, uint32_t n0,
                  const LaunchShape& ls, cudaStream_t stream) {
    const bool aov = pool.aov_albedo != nullptr, guided = pool.guide_out != nullptr;
    auto shade = [&](bool layers, uint32_t part) {
        auto args = [&](auto kernel) {
            kernel<<<layers ? ls.grid_shade : ls.grid_shade_free, BLOCK, 0, stream>>>(
                scene, pool, bounce, wp.max_bounces, wp.light_sampling, n0, part);
        };
        if (layers) {
            if (aov && guided) args(k_shade<true, true, true>);
            else if (aov) args(k_shade<true, false, true>);
            else if (guided) args(k_shade<false, true, true>);
            else args(k_shade<false, false, true>);
        } else {
            if (aov && guided) args(k_shade<true, true, false>);
            else if (aov) args(k_shade<true, false, false>);
            else if (guided) args(k_shade<false, true, false>);
            else args(k_shade<false, false, false>);
        }
    };
    if (!scene.has_layers) {
        shade(false, 0);
    } else if (pool.order) {
        // A sorted bounce of a scene with both kinds: the layer-free range
        // (and the misses) without the layered lobes, then the rest.
        shade(false, 1);
        shade(true, 2);
    } else {
        shade(true, 0);
    }
}

void launch_shadow(const DeviceScene& scene, const PathPool& pool, uint32_t bounce, const LaunchShape& ls,
                   bool count_visits, cudaStream_t stream) {
    switch (trav_variant(scene, pool)) {
    case 1: launch_shadow_v<1>(scene, pool, bounce, ls, count_visits, stream); break;
    case 2: launch_shadow_v<2>(scene, pool, bounce, ls, count_visits, stream); break;
    case 3: launch_shadow_v<3>(scene, pool, bounce, ls, count_visits, stream); break;
    default: launch_shadow_v<0>(scene, pool, bounce, ls, count_visits, stream); break;
    }
}

void launch_wave(const DeviceScene& scene, const PathPool& pool, const WaveParams& wp, const LaunchShape& ls,
                 cudaStream_t stream) {
    const uint32_t n0 = wp.pixel_count * wp.samples;
    launch_wave_begin(pool, wp, ls, stream);
    for (uint32_t b = 0; b < wp.max_bounces; ++b) {
        launch_intersect(scene, pool, b, n0, ls, false, stream);
        launch_shade(scene, pool, b, wp, n0, ls, stream);
        launch_shadow(scene, pool, b, ls, false, stream);
    }
}

void launch_accumulate(const PathPool& pool, const FilmTargets& film, uint32_t pixel_base, uint32_t pixel_count,
                       uint32_t tile_width, uint32_t samples, bool reset, cudaStream_t stream) {
    int grid = int((pixel_count + 255) / 256);
    if (grid > 148 * 16) grid = 148 * 16;
    if (pool.aov_albedo && film.albedo)
        k_accumulate<true><<<grid, 256, 0, stream>>>(pool, film, pixel_base, pixel_count, tile_width, samples,
                                                     reset ? 1u : 0u);
    else
        k_accumulate<false><<<grid, 256, 0, stream>>>(pool, film, pixel_base, pixel_count, tile_width, samples,
                                                      reset ? 1u : 0u);
}

void launch_sort_begin(const PathPool& pool, cudaStream_t stream) {
    if (pool.sort_bins) cudaMemsetAsync(pool.sort_bins, 0, SORT_BINS * sizeof(uint32_t), stream);
}

void launch_material_sort(const PathPool& pool, uint32_t bounce, uint32_t n0, const LaunchShape& ls,
                          cudaStream_t stream) {
    if (!pool.order || !pool.sort_keys || !pool.sort_bins) return;  // the caller's pool view carries all three
    k_sort_scan<<<1, 1024, 0, stream>>>(pool.sort_bins);
    k_sort_scatter<<<ls.grid_stream, BLOCK, 0, stream>>>(pool, bounce, n0);
}

void launch_tonemap(const float4* avg, uint32_t* out, uint32_t pixels, float exposure_scale, cudaStream_t stream) {
    int grid = int((pixels + 255) / 256);
    if (grid > 148 * 16) grid = 148 * 16;
    k_tonemap<<<grid, 256, 0, stream>>>(avg, out, pixels, exposure_scale);
}

void launch_resolve1(const float* sum, float* avg, uint32_t pixels, float samples, cudaStream_t stream) {
    int grid = int((pixels + 255) / 256);
    if (grid > 148 * 16) grid = 148 * 16;
    k_resolve1<<<grid, 256, 0, stream>>>(sum, avg, pixels, samples);
}

void launch_resolve(const float4* sum, float4* avg, uint32_t pixels, float samples, cudaStream_t stream) {
    int grid = int((pixels + 255) / 256);
    if (grid > 148 * 16) grid = 148 * 16;
    k_resolve<<<grid, 256, 0, stream>>>(sum, avg, pixels, samples);
}

void launch_copy_rad(const PathPool& pool, float4* out, uint32_t pixel_base, uint32_t pixel_count, uint32_t tile_width,
                     cudaStream_t stream) {
    int grid = int((pixel_count + 255) / 256);
    if (grid > 148 * 16) grid = 148 * 16;
    k_copy_rad<<<grid, 256, 0, stream>>>(pool.rad, out, pixel_base, pixel_count, tile_width);
}

}  // namespace cn
