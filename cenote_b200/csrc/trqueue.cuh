// Warp triangle queue: the closest-hit walk with its triangle tests shared
// by the whole warp.
//
// In the per-lane walk (traverse.cuh, walk_step) every lane tests its own hit
// leaves' triangles one at a time right after the node that found them, so a
// warp spends as many iterations as its busiest lane has triangles while the
// other lanes idle (measured at the bench's wave sizes: 23 % of lanes active
// in the triangle loop on the material chart, 14 % on the terrain). Here a
// lane appends each triangle group (first triangle, 24 pending bits) to a
// per-warp FIFO in shared memory and keeps walking; once the FIFO holds a
// warp's worth of triangles (or no lane has nodes left), a round hands one
// (ray, triangle) pair to every lane: a warp scan of the entries' bit counts
// maps lane j to its entry and bit, the owner's ray comes over shuffles, and
// each owner's candidates reduce to the lexicographic minimum of (t,
// instance, primitive) through shared-memory atomic minima (any-hit queries:
// an OR of occluders). A lane whose walk has ended waits for its queued
// triangles before it takes a new ray.
//
// Results are bitwise those of the per-lane walk: the watertight test of a
// (ray, triangle) pair is the same arithmetic wherever it runs, and both
// commit the lexicographic minimum of (t, instance, primitive) over the
// candidates with t within the ray's bound (the walk's node culling keeps a
// slack above the current hit, so a later commit never drops a winner; a ray
// walking here culls with a bound at least as large as the per-lane walk's,
// which only adds candidates that lose). Only scenes whose triangles are all
// opaque use it: fractional opacity draws its Bernoulli decisions in visit
// order.
#pragma once
#include "shadow.cuh"
#include "traverse.cuh"

namespace cn {

constexpr uint32_t TQ_CAP = 64;  // FIFO entries per warp (a power of two, at least 2 x 32)
constexpr uint32_t TQ_FULL = 0xffffffffu;
// A closest-hit round also runs, partly filled, once this many lanes have
// ended their walks and only wait for queued triangles, so they take new rays
// sooner (chart intersect -4 %; 4 and 16 measured slower; the shadow walk
// measured no gain from it).
constexpr uint32_t TQ_WAITING = 8;

// One warp's queue in shared memory (896 bytes), small enough that a full SM
// of traversal blocks leaves the L1 cache (which holds the walks' stacks and
// the nodes and triangles they revisit) almost all of its capacity.
struct TriQueueSmem {
    uint2 entry[TQ_CAP];     // (first triangle, owner lane << 24 | untested triangle bits)
    // Per owner lane, a round's running minima of the candidates' t key and
    // instance, then its primitive and the winning lane; ~0 between rounds.
    uint32_t key[32], key2[32], winner[32];
};

// The warp's queue positions; every lane holds the same values. Entries
// head .. tail-1 are pending; `tris` counts their untested bits.
struct TriQueue {
    uint32_t head, tail, tris;
};

// The closest hit of a lane's ray so far.
struct Closest {
    float tmax, b1, b2;
    uint32_t inst, prim;
};

__device__ __forceinline__ void closest_begin(Closest& c) {
    c.tmax = 1e30f;
    c.b1 = c.b2 = 0.0f;
    c.inst = LIGHT_NONE;
    c.prim = 0u;
}

// Position of the (k+1)-th lowest set bit of m (m has more than k set bits):
// the largest x with popc(m below x) <= k, by binary search.
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t m, uint32_t k) {
    uint32_t p = 0;
#pragma unroll
    for (uint32_t w = 16; w > 0; w >>= 1)
        if (uint32_t(__popc(m & ((1u << (p + w)) - 1u))) <= k) p += w;
    return p;
}

// Append each lane's triangle group (low 24 bits of grp.y; none when zero).
// All 32 lanes call it together; the caller keeps at most TQ_CAP - 32
// entries pending before the call.
__device__ __forceinline__ void tq_append(TriQueueSmem& sm, TriQueue& q, uint2 grp, uint32_t& last_seq) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t bits = grp.y & 0x00ffffffu;
    const uint32_t ball = __ballot_sync(TQ_FULL, bits != 0u);
    if (bits) {
        const uint32_t seq = q.tail + __popc(ball & ((1u << lane) - 1u));
        sm.entry[seq & (TQ_CAP - 1u)] = make_uint2(grp.x, (lane << 24) | bits);
        last_seq = seq + 1u;
    }
    q.tail += __popc(ball);
    q.tris += __reduce_add_sync(TQ_FULL, __popc(bits));
    __syncwarp();
}

// A round's work for one lane: triangle `tri` of the ray owned by lane
// `owner`, when `act`.
struct TqWork {
    uint32_t tri, owner;
    bool act;
};

// Take the next min(32, pending) triangles of the FIFO, one per lane: a warp
// scan of the entries' bit counts maps lane j to its entry and bit; the entry
// crossing the last slot keeps the bits this round does not reach. Advances
// the queue; all 32 lanes call it together with q.tris > 0.
__device__ __forceinline__ TqWork tq_take(TriQueueSmem& sm, TriQueue& q) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t idx = q.head + lane;
    const bool has = idx < q.tail;
    const uint2 e = has ? sm.entry[idx & (TQ_CAP - 1u)] : make_uint2(0u, 0u);
    const uint32_t bits = e.y & 0x00ffffffu;
    const uint32_t cnt = __popc(bits);
    uint32_t incl = cnt;
#pragma unroll
    for (uint32_t o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(TQ_FULL, incl, o);
        if (lane >= o) incl += v;
    }
    const uint32_t excl = incl - cnt;
    const uint32_t n = min(__shfl_sync(TQ_FULL, incl, 31), 32u);
    // The entry serving slot `lane`: the last one whose prefix is <= lane.
    uint32_t k = 0;
#pragma unroll
    for (uint32_t st = 16; st > 0; st >>= 1)
        if (__shfl_sync(TQ_FULL, excl, k + st) <= lane) k += st;
    const uint32_t kbits = __shfl_sync(TQ_FULL, bits, k);
    const uint32_t kbase = __shfl_sync(TQ_FULL, e.x, k);
    const uint32_t kexcl = __shfl_sync(TQ_FULL, excl, k);
    TqWork wk;
    wk.owner = __shfl_sync(TQ_FULL, e.y >> 24, k);
    wk.act = lane < n;
    wk.tri = wk.act ? kbase + nth_set_bit(kbits, lane - kexcl) : 0u;
    if (has && excl < n && incl > n) {
        const uint32_t cut = nth_set_bit(bits, n - excl - 1u);
        sm.entry[idx & (TQ_CAP - 1u)].y = (e.y & 0xff000000u) | (bits & ~((2u << cut) - 1u));
    }
    q.head += __popc(__ballot_sync(TQ_FULL, has && incl <= n));
    q.tris -= n;
    return wk;
}

// The owner's ray as the watertight test reads it, over shuffles.
__device__ __forceinline__ Ray owner_ray(const Ray& ray, uint32_t owner) {
    Ray ro;
    ro.org = f3(__shfl_sync(TQ_FULL, ray.org.x, owner), __shfl_sync(TQ_FULL, ray.org.y, owner),
                __shfl_sync(TQ_FULL, ray.org.z, owner));
    ro.sx = __shfl_sync(TQ_FULL, ray.sx, owner);
    ro.sy = __shfl_sync(TQ_FULL, ray.sy, owner);
    ro.sz = __shfl_sync(TQ_FULL, ray.sz, owner);
    const uint32_t kp =
        __shfl_sync(TQ_FULL, uint32_t(ray.kx) | (uint32_t(ray.ky) << 2) | (uint32_t(ray.kz) << 4), owner);
    ro.kx = int(kp & 3u);
    ro.ky = int((kp >> 2) & 3u);
    ro.kz = int((kp >> 4) & 3u);
    return ro;
}

// One closest-hit round: each lane's triangle tested against its owner's
// ray; every owner commits the best of its candidates. All 32 lanes call it
// together with q.tris > 0.
template <bool COUNT = false>
__device__ __forceinline__ void tq_round(const DeviceScene& s, TriQueueSmem& sm, TriQueue& q, const Ray& ray,
                                         Closest& c, uint32_t ray_mask, uint32_t* tests) {
    const uint32_t lane = threadIdx.x & 31u;
    const TqWork wk = tq_take(sm, q);
    const uint32_t owner = wk.owner;
    const Ray ro = owner_ray(ray, owner);
    const float tmo = __shfl_sync(TQ_FULL, c.tmax, owner);
    bool cand = false;
    float t = 0.0f, b1 = 0.0f, b2 = 0.0f;
    uint32_t inst = 0u, prim = 0u;
    if (wk.act && wk.tri < s.tri_count) {
        const float4* tp = s.tris + 3u * wk.tri;
        const float4 a = __ldg(tp), b = __ldg(tp + 1), cc = __ldg(tp + 2);
        if (COUNT) ++*tests;
        if ((__float_as_uint(cc.w) & ray_mask) && tri_hit(ro, a, b, cc, tmo, t, b1, b2)) {
            cand = true;
            inst = __float_as_uint(a.w);
            prim = __float_as_uint(b.w);
        }
    }
    // Per owner, the lexicographic minimum of (t, instance, primitive); both
    // zeros of t order as one, as they compare equal in the per-lane walk.
    const uint32_t tkey = cand ? (t == 0.0f ? 0u : __float_as_uint(t)) : 0xffffffffu;
    // Shared-memory minima per owner, one key at a time (the slots start
    // at ~0 and are reset by their owners after the round). Grouping the
    // lanes by owner with a warp match instead measured 30 % slower.
    if (cand) atomicMin(&sm.key[owner], tkey);
    __syncwarp();
    const bool c2 = cand && sm.key[owner] == tkey;
    if (c2) atomicMin(&sm.key2[owner], inst);
    __syncwarp();
    const bool c3 = c2 && sm.key2[owner] == inst;
    if (c3) atomicMin(&sm.winner[owner], prim);
    __syncwarp();
    const bool win = c3 && sm.winner[owner] == prim;
    __syncwarp();
    if (win) sm.winner[owner] = lane;
    const uint32_t hasw = __ballot_sync(TQ_FULL, sm.key[lane] != 0xffffffffu);
    __syncwarp();
    // Each owner takes its winner's candidate over shuffles.
    const bool mine = (hasw >> lane) & 1u;
    const uint32_t from = mine ? sm.winner[lane] : lane;
    const float wt = __shfl_sync(TQ_FULL, t, from), wb1 = __shfl_sync(TQ_FULL, b1, from),
                wb2 = __shfl_sync(TQ_FULL, b2, from);
    const uint32_t wi = __shfl_sync(TQ_FULL, inst, from), wp = __shfl_sync(TQ_FULL, prim, from);
    if (mine && (wt < c.tmax || (wt == c.tmax && (wi < c.inst || (wi == c.inst && wp < c.prim))))) {
        c.tmax = wt;
        c.inst = wi;
        c.prim = wp;
        c.b1 = wb1;
        c.b2 = wb2;
    }
    sm.key[lane] = 0xffffffffu;
    sm.key2[lane] = 0xffffffffu;
    sm.winner[lane] = 0xffffffffu;
    __syncwarp();
}

// The queued closest-hit walk of a persistent warp. `src` supplies and
// retires the rays (all members are called by the whole warp unless noted):
//   uint32_t next(bool live, bool& drained)  an item for each idle lane (~0u: none)
//   void ray(uint32_t item, float3& org, float3& dir)      (per lane)
//   void emit(uint32_t item, uint4 hit, float t)          (per lane)
//   void step(bool finished, uint32_t item, uint32_t instance, float t)  after every step
//   uint32_t want_idle(bool drained)  idle lanes before the warp refills
// Each step a walking lane expands one node and queues the triangles of the
// leaves it hits; rounds run while the FIFO holds a warp's worth of
// triangles, while TQ_WAITING lanes wait on it, or until it is empty once no
// lane has nodes left. A lane whose
// walk has ended completes when its last queued entry has been tested.
// Sets `overflow` when a walk hit its iteration or stack bound.
template <bool COUNT, class Src, int S = TRAVERSAL_STACK>
__device__ __forceinline__ void queued_closest(const DeviceScene& s, TriQueueSmem& sm, Src& src, uint32_t ray_mask,
                                               bool& overflow, uint32_t* visits, uint32_t* tests) {
    TriQueue q{0u, 0u, 0u};
    uint2 stack[S];
    Walk w;
    Ray ray;
    Closest c;
    closest_begin(c);
    uint32_t item = 0u, last_seq = 0u;
    bool live = false, walking = false, drained = false;
    sm.key[threadIdx.x & 31u] = 0xffffffffu;
    sm.key2[threadIdx.x & 31u] = 0xffffffffu;
    sm.winner[threadIdx.x & 31u] = 0xffffffffu;
    __syncwarp();
    for (;;) {
        if (!drained) {
            const uint32_t i = src.next(live, drained);
            if (i != ~0u) {
                float3 o, d;
                src.ray(i, o, d);
                ray = make_ray(o, d);
                closest_begin(c);
                walk_begin(w, ray);
                item = i;
                last_seq = 0u;
                live = true;
                walking = s.node_count != 0;
            }
        }
        if (!__any_sync(TQ_FULL, live)) {
            if (drained) break;
            continue;
        }
        const uint32_t want_idle = src.want_idle(drained);
        for (;;) {
            uint2 grp = make_uint2(0u, 0u);
            if (live && walking) {
                if (++w.iter > walk_bound(s) || !expand_node<COUNT, S>(s, ray, c.tmax, w, stack, visits)) {
                    overflow = true;
                    walking = false;
                } else {
                    grp = w.t;
                    if (!(w.g.y & 0xff000000u)) {
                        if (w.sp == 0) walking = false;
                        else w.g = stack[--w.sp];
                    }
                }
            }
            tq_append(sm, q, grp, last_seq);
            const bool any_walking = __any_sync(TQ_FULL, live && walking);
            const bool many_waiting = uint32_t(__popc(__ballot_sync(TQ_FULL, live && !walking))) >= TQ_WAITING;
            while (q.tris >= 32u || (q.tris > 0u && (!any_walking || many_waiting)))
                tq_round<COUNT>(s, sm, q, ray, c, ray_mask, tests);
            bool finished = false;
            if (live && !walking && q.head >= last_seq) {
                src.emit(item, make_uint4(c.inst, c.prim, __float_as_uint(c.b1), __float_as_uint(c.b2)), c.tmax);
                finished = true;
                live = false;
            }
            src.step(finished, item, c.inst, c.tmax);
            if (uint32_t(__popc(__ballot_sync(TQ_FULL, !live))) >= want_idle) break;
        }
    }
}

// ---- shadow queries (trace_shadow.slang:29-72) ------------------------------------

// A shadow query as the queued walk keeps it: its bound (the target
// triangle's distance, or tmax without one), the target's leaf (~0 when the
// target was not hit or there is none) and (instance, primitive) identity.
struct AnyQuery {
    float tm;
    uint32_t leaf, light, lprim;
    bool occluded;
};

// One any-hit round: each lane's triangle tested against its owner's query;
// an opaque hit nearer than the owner's target (equal distance: the smaller
// (instance, primitive) key) occludes it, as in shadow_step. All 32 lanes
// call it together with q.tris > 0.
template <bool COUNT = false>
__device__ __forceinline__ void tq_round_any(const DeviceScene& s, TriQueueSmem& sm, TriQueue& q, const Ray& ray,
                                             AnyQuery& a, uint32_t* tests) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t dead = __ballot_sync(TQ_FULL, a.occluded);
    const TqWork wk = tq_take(sm, q);
    const uint32_t owner = wk.owner;
    const Ray ro = owner_ray(ray, owner);
    const float tmo = __shfl_sync(TQ_FULL, a.tm, owner);
    const uint32_t leaf = __shfl_sync(TQ_FULL, a.leaf, owner), light = __shfl_sync(TQ_FULL, a.light, owner),
                   lprim = __shfl_sync(TQ_FULL, a.lprim, owner);
    bool occl = false;
    if (wk.act && !((dead >> owner) & 1u) && wk.tri != leaf && wk.tri < s.tri_count) {
        const float4* tp = s.tris + 3u * wk.tri;
        const float4 v0 = __ldg(tp), v1 = __ldg(tp + 1), v2 = __ldg(tp + 2);
        if (COUNT) ++*tests;
        float t, b1, b2;
        if (tri_hit(ro, v0, v1, v2, tmo, t, b1, b2)) {
            const uint32_t inst = __float_as_uint(v0.w), prim = __float_as_uint(v1.w);
            occl = !(leaf != 0xffffffffu && t == tmo && !(inst < light || (inst == light && prim < lprim)));
        }
    }
    if ((__reduce_or_sync(TQ_FULL, occl ? (1u << owner) : 0u) >> lane) & 1u) a.occluded = true;
    __syncwarp();
}

// The queued shadow walk of a persistent warp over scenes whose triangles
// are all opaque. `src` supplies and retires the queries (the whole warp
// calls each member unless noted):
//   uint32_t next(bool live, bool& drained)  an item for each idle lane (~0u: none)
//   bool begin(uint32_t item, Ray& ray, AnyQuery& a)   (per lane) false: the
//       query has no target leaf to bound it; then `closest(item)` answers it
//       with the per-lane closest-hit walk
//   template <int S> void closest(uint32_t item, uint2* stack)  (per lane; the
//       stack holds S entries)
//   void emit(uint32_t item, bool visible)              (per lane; a query
//       whose walk hit a bound counts as occluded)
//   uint32_t want_idle(bool drained)
// An occluded query stops walking at once; its entries still queued are
// skipped, and it completes when they have left the queue.
template <bool COUNT, class Src, int S = TRAVERSAL_STACK>
__device__ __forceinline__ void queued_any(const DeviceScene& s, TriQueueSmem& sm, Src& src, bool& overflow,
                                           uint32_t* visits, uint32_t* tests) {
    TriQueue q{0u, 0u, 0u};
    uint2 stack[S];
    Walk w;
    Ray ray;
    AnyQuery a{0.0f, 0xffffffffu, LIGHT_NONE, 0u, false};
    uint32_t item = 0u, last_seq = 0u;
    bool live = false, walking = false, drained = false, ovf = false;
    for (;;) {
        if (!drained) {
            const uint32_t i = src.next(live, drained);
            if (i != ~0u) {
                item = i;
                last_seq = 0u;
                live = true;
                ovf = false;
                walking = src.begin(i, ray, a) && s.node_count != 0;
                if (!walking && !a.occluded && s.node_count != 0) {
                    src.template closest<S>(i, stack);  // no target leaf: the per-lane closest-hit query
                    live = false;
                }
                walk_begin(w, ray);
            }
        }
        if (!__any_sync(TQ_FULL, live)) {
            if (drained) break;
            continue;
        }
        const uint32_t want_idle = src.want_idle(drained);
        for (;;) {
            uint2 grp = make_uint2(0u, 0u);
            if (live && walking && !a.occluded) {
                if (++w.iter > walk_bound(s) || !expand_node<COUNT, S>(s, ray, a.tm, w, stack, visits)) {
                    overflow = true;
                    ovf = true;  // dropped, as the per-lane walk drops it
                    walking = false;
                } else {
                    grp = w.t;
                    if (!(w.g.y & 0xff000000u)) {
                        if (w.sp == 0) walking = false;
                        else w.g = stack[--w.sp];
                    }
                }
            }
            tq_append(sm, q, grp, last_seq);
            const bool any_walking = __any_sync(TQ_FULL, live && walking && !a.occluded);
            while (q.tris >= 32u || (q.tris > 0u && !any_walking)) tq_round_any<COUNT>(s, sm, q, ray, a, tests);
            if (live && (!walking || a.occluded) && q.head >= last_seq) {
                src.emit(item, !a.occluded && !ovf);
                live = false;
            }
            if (uint32_t(__popc(__ballot_sync(TQ_FULL, !live))) >= want_idle) break;
        }
    }
}

}  // namespace cn
