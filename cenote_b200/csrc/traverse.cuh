// Ray traversal of the compressed 8-wide BVH and the watertight triangle test.
//
// One thread per ray. A node is five 16-byte read-only loads; its eight
// child boxes are decoded from bytes against the node's quantisation frame
// and tested in one pass, producing a 32-bit hit mask: bits 24-31 carry the
// hit inner children at position 24 + (slot XOR octant) so that taking the
// highest bit visits children near to far, bits 0-23 carry the triangles of
// the hit leaf children (Ylitie, Karras & Laine, HPG 2017, node/triangle
// groups). The stack holds node groups (base index, pending bits | imask).
//
// Triangle test: Woop, Benthin & Wald, "Watertight Ray/Triangle
// Intersection", JCGT 2013, with the double-precision fallback on zero edge
// functions. It is written with explicitly rounded intrinsics so the compiler
// cannot contract it into FMAs: the CPU check evaluates the same operations
// and commits bit-identical hits. Equal-t candidates resolve to the smaller
// (instance, primitive) key, so the committed hit never depends on traversal
// order. Every loop is bounded; hitting a bound raises an overflow flag.
#pragma once
#include "records.h"
#include "vecmath.cuh"

namespace cn {


constexpr int TRAVERSAL_STACK = TRAVERSAL_STACK_DEPTH;

struct Ray {
    float3 org, dir, idir;
    int kx, ky, kz;
    float sx, sy, sz;
    uint32_t oct_inv;  // bit 2: dir.x >= 0, bit 1: dir.y >= 0, bit 0: dir.z >= 0
};

__device__ __forceinline__ float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

__device__ __forceinline__ Ray make_ray(float3 org, float3 dir) {
    Ray r;
    r.org = org;
    r.dir = dir;
    r.idir = f3(__fdiv_rn(1.0f, dir.x), __fdiv_rn(1.0f, dir.y), __fdiv_rn(1.0f, dir.z));
    float ax = fabsf(dir.x), ay = fabsf(dir.y), az = fabsf(dir.z);
    int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    float dz = comp(dir, kz);
    if (dz < 0.0f) {
        int t = kx;
        kx = ky;
        ky = t;
    }
    r.kx = kx;
    r.ky = ky;
    r.kz = kz;
    // The shear constants (Woop et al. 2013) from the reciprocal already
    // taken: any per-ray constants keep the test watertight, as long as every
    // triangle of the ray uses the same ones.
    r.sz = comp(r.idir, kz);
    r.sx = __fmul_rn(comp(dir, kx), r.sz);
    r.sy = __fmul_rn(comp(dir, ky), r.sz);
    r.oct_inv = (dir.x >= 0.0f ? 4u : 0u) | (dir.y >= 0.0f ? 2u : 0u) | (dir.z >= 0.0f ? 1u : 0u);
    return r;
}

// t in [0, tmax]; (b1, b2) = weights on (v1, v2).
__device__ __forceinline__ bool tri_hit(const Ray& r, float4 a, float4 b, float4 c, float tmax, float& t, float& b1,
                                        float& b2) {
    float3 A = f3(__fsub_rn(a.x, r.org.x), __fsub_rn(a.y, r.org.y), __fsub_rn(a.z, r.org.z));
    float3 B = f3(__fsub_rn(b.x, r.org.x), __fsub_rn(b.y, r.org.y), __fsub_rn(b.z, r.org.z));
    float3 C = f3(__fsub_rn(c.x, r.org.x), __fsub_rn(c.y, r.org.y), __fsub_rn(c.z, r.org.z));
    float Akz = comp(A, r.kz), Bkz = comp(B, r.kz), Ckz = comp(C, r.kz);
    float Ax = __fsub_rn(comp(A, r.kx), __fmul_rn(r.sx, Akz)), Ay = __fsub_rn(comp(A, r.ky), __fmul_rn(r.sy, Akz));
    float Bx = __fsub_rn(comp(B, r.kx), __fmul_rn(r.sx, Bkz)), By = __fsub_rn(comp(B, r.ky), __fmul_rn(r.sy, Bkz));
    float Cx = __fsub_rn(comp(C, r.kx), __fmul_rn(r.sx, Ckz)), Cy = __fsub_rn(comp(C, r.ky), __fmul_rn(r.sy, Ckz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = __double2float_rn(__dsub_rn(__dmul_rn(double(Cx), double(By)), __dmul_rn(double(Cy), double(Bx))));
        V = __double2float_rn(__dsub_rn(__dmul_rn(double(Ax), double(Cy)), __dmul_rn(double(Ay), double(Cx))));
        W = __double2float_rn(__dsub_rn(__dmul_rn(double(Bx), double(Ay)), __dmul_rn(double(By), double(Ax))));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.0f) return false;
    float Az = __fmul_rn(r.sz, Akz), Bz = __fmul_rn(r.sz, Bkz), Cz = __fmul_rn(r.sz, Ckz);
    float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
    float rcp = __fdiv_rn(1.0f, det);
    float tt = __fmul_rn(T, rcp);
    if (!(tt >= 0.0f && tt <= tmax)) return false;
    t = tt;
    b1 = __fmul_rn(V, rcp);
    b2 = __fmul_rn(W, rcp);
    return true;
}

__device__ __forceinline__ uint32_t byte_of(uint32_t lo4, uint32_t hi4, int i) {
    return ((i < 4 ? lo4 : hi4) >> (8 * (i & 3))) & 0xffu;
}

// Intersect the eight children of node `ni`. Returns the hit mask; fills the
// node's child/triangle base indices and inner mask.
__device__ __forceinline__ uint4 ld_shared4(uint32_t addr) {
    uint4 v;
#ifdef __CUDA_ARCH__
    asm("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(addr));
#else
    v = make_uint4(0u, 0u, 0u, 0u);
#endif
    return v;
}

// Copy the first `limit` nodes (at most the scene's) into `smem` for the
// whole block and record them in `s`; every thread of the block must call it.
__device__ __forceinline__ void stage_top_levels(DeviceScene& s, uint4* smem, uint32_t limit) {
#ifdef __CUDA_ARCH__
    const uint32_t n = min(s.node_count, limit);
    const uint4* src = reinterpret_cast<const uint4*>(s.nodes);
    for (uint32_t k = threadIdx.x; k < 5u * n; k += blockDim.x) smem[k] = __ldg(src + k);
    __syncthreads();
    s.top_count = n;
    s.top_smem = uint32_t(__cvta_generic_to_shared(smem));
#endif
}

__device__ __forceinline__ uint32_t intersect_node(const DeviceScene& s, uint32_t ni, const Ray& r, float tmax,
                                                   uint32_t& base_child, uint32_t& base_tri, uint32_t& imask) {
    uint4 n0, n1, n2, n3, n4;
    if (ni < s.top_count) {
        const uint32_t a = s.top_smem + 80u * ni;
        n0 = ld_shared4(a);
        n1 = ld_shared4(a + 16u);
        n2 = ld_shared4(a + 32u);
        n3 = ld_shared4(a + 48u);
        n4 = ld_shared4(a + 64u);
    } else {
        const uint4* q = reinterpret_cast<const uint4*>(s.nodes + ni);
        n0 = __ldg(q);
        n1 = __ldg(q + 1);
        n2 = __ldg(q + 2);
        n3 = __ldg(q + 3);
        n4 = __ldg(q + 4);
    }
    float3 p = f3(__uint_as_float(n0.x), __uint_as_float(n0.y), __uint_as_float(n0.z));
    float sx = __uint_as_float((n0.w & 0xffu) << 23);
    float sy = __uint_as_float(((n0.w >> 8) & 0xffu) << 23);
    float sz = __uint_as_float(((n0.w >> 16) & 0xffu) << 23);
    imask = n0.w >> 24;
    base_child = n1.x;
    base_tri = n1.y;
    float3 aid = f3(sx * r.idir.x, sy * r.idir.y, sz * r.idir.z);
    float3 aor = f3((p.x - r.org.x) * r.idir.x, (p.y - r.org.y) * r.idir.y, (p.z - r.org.z) * r.idir.z);
    // Near/far plane words per axis, swapped for negative directions.
    uint32_t nx0 = n2.x, nx1 = n2.y, fx0 = n3.z, fx1 = n3.w;
    uint32_t ny0 = n2.z, ny1 = n2.w, fy0 = n4.x, fy1 = n4.y;
    uint32_t nz0 = n3.x, nz1 = n3.y, fz0 = n4.z, fz1 = n4.w;
    if (r.idir.x < 0.0f) { uint32_t t0 = nx0, t1 = nx1; nx0 = fx0; nx1 = fx1; fx0 = t0; fx1 = t1; }
    if (r.idir.y < 0.0f) { uint32_t t0 = ny0, t1 = ny1; ny0 = fy0; ny1 = fy1; fy0 = t0; fy1 = t1; }
    if (r.idir.z < 0.0f) { uint32_t t0 = nz0, t1 = nz1; nz0 = fz0; nz1 = fz1; fz0 = t0; fz1 = t1; }
    const float tlimit = tmax * 1.00002f;  // cull only nodes clearly beyond the current hit
    // An inner child's meta byte is 0b001_11sss (bit 24 + slot); XOR its slot
    // with the ray's octant for all eight children at once: bit 3 of a byte
    // is set where its bits 3 and 4 both are (inner children only: leaf
    // offsets stop at 23), moved to bit 0 and multiplied by the octant (at
    // most 7, so no carry crosses a byte).
    const uint32_t ml = n1.z ^ ((((n1.z >> 1) & n1.z & 0x08080808u) >> 3) * r.oct_inv);
    const uint32_t mh = n1.w ^ ((((n1.w >> 1) & n1.w & 0x08080808u) >> 3) * r.oct_inv);
    uint32_t mask = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        uint32_t meta = byte_of(ml, mh, i);  // 0 for an empty slot: contributes no bits
        float tnx = fmaf(float(byte_of(nx0, nx1, i)), aid.x, aor.x);
        float tny = fmaf(float(byte_of(ny0, ny1, i)), aid.y, aor.y);
        float tnz = fmaf(float(byte_of(nz0, nz1, i)), aid.z, aor.z);
        float tfx = fmaf(float(byte_of(fx0, fx1, i)), aid.x, aor.x);
        float tfy = fmaf(float(byte_of(fy0, fy1, i)), aid.y, aor.y);
        float tfz = fmaf(float(byte_of(fz0, fz1, i)), aid.z, aor.z);
        float t0 = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, 0.0f));
        float t1 = fminf(fminf(tfx, tfy), fminf(tfz, tlimit)) * 1.0000004f;
        if (t0 <= t1) {
            mask |= (meta >> 5) << (meta & 0x1fu);
        }
    }
    return mask;
}

// Walk the BVH, handing each candidate triangle to `visit(tri_index, v0, v1,
// v2, tmax&)`, which may shrink tmax and returns true to stop the walk.
// Returns false if a bound was exceeded (the caller flags an overflow).
//
// Node groups and triangle groups share the stack (a group with bits 24-31
// set is a node group; otherwise its low 24 bits are pending triangles).
// When fewer than POSTPONE lanes of the warp have triangles to test, the
// triangle group is pushed and the lane keeps walking nodes, so warps test
// triangles together instead of idling through each other's leaves
// (Ylitie et al. 2017, postponement).
#ifndef CN_POSTPONE
#define CN_POSTPONE 2  // 2 vs 4 vs 8: level / -1 % / -8 % on the terrain, level / level / -5 % on the chart
#endif
constexpr uint32_t POSTPONE = CN_POSTPONE;

// The walk as a resumable state machine, so a persistent kernel can retire a
// finished ray and start a new one in its lane while the warp's other lanes
// are mid-walk (dynamic ray fetching, Aila & Laine, HPG 2009). The stack
// lives with the caller.
struct Walk {
    uint2 g, t;      // the node group being expanded, the triangle group being tested
    int sp;
    uint32_t iter;
    bool resumed;    // the triangle group came off the stack: never postpone it twice
};

enum : int { WALK_CONTINUE = 0, WALK_DONE = 1, WALK_OVERFLOW = -1 };

__device__ __forceinline__ void walk_begin(Walk& w, const Ray& r) {
    w.g = make_uint2(0u, (1u << (24u + r.oct_inv)) | 1u);  // the root: inner slot 0 of a virtual parent
    w.t = make_uint2(0u, 0u);
    w.sp = 0;
    w.iter = 0;
    w.resumed = false;
}

__device__ __forceinline__ uint32_t walk_bound(const DeviceScene& s) { return 4u * (s.node_count + s.tri_count) + 64u; }

// Take the nearest pending inner child of the node group w.g (which must
// have one), push what remains of the group and intersect the child: w.g
// becomes its inner children, w.t its hit leaves' triangles. Returns false
// when the stack is full.
template <bool COUNT = false, int S = TRAVERSAL_STACK>
__device__ __forceinline__ bool expand_node(const DeviceScene& s, const Ray& r, float tmax, Walk& w, uint2* stack,
                                            uint32_t* visits) {
    uint32_t pos = 31u - __clz(w.g.y & 0xff000000u);
    w.g.y &= ~(1u << pos);
    uint32_t slot = (pos - 24u) ^ r.oct_inv;
    uint32_t ni = w.g.x + __popc(w.g.y & 0xffu & ((1u << slot) - 1u));
    if (w.g.y & 0xff000000u) {
        if (w.sp >= S) return false;
        stack[w.sp++] = w.g;
    }
    uint32_t bc, bt, im;
    uint32_t hits = intersect_node(s, ni, r, tmax, bc, bt, im);
    if (COUNT) ++*visits;
    w.g = make_uint2(bc, (hits & 0xff000000u) | im);
    w.t = make_uint2(bt, hits & 0x00ffffffu);
    return true;
}

// One step: expand one node (or resume one postponed triangle group), then
// test its triangles unless too few lanes of the warp would test alongside.
// `visit` returning true stops the walk (WALK_DONE). `S`: the stack's
// entries; a triangle group is postponed only while the node groups that
// may follow (the tree's stack need) still fit behind it.
template <bool COUNT = false, int S = TRAVERSAL_STACK, class Visit>
__device__ __forceinline__ int walk_step(const DeviceScene& s, const Ray& r, float& tmax, Walk& w, uint2* stack,
                                         Visit&& visit, uint32_t* visits = nullptr, uint32_t* tests = nullptr) {
    if (++w.iter > walk_bound(s)) return WALK_OVERFLOW;
    if (w.g.y & 0xff000000u) {
        if (!expand_node<COUNT, S>(s, r, tmax, w, stack, visits)) return WALK_OVERFLOW;
        w.resumed = false;
    } else {
        w.t = w.g;  // a postponed triangle group came off the stack
        w.g = make_uint2(0u, 0u);
        w.resumed = true;
    }
    while (w.t.y & 0x00ffffffu) {
        if (!w.resumed && w.sp + (TRAVERSAL_STACK_DEPTH - int(s.stack_room)) < S &&
            uint32_t(__popc(__activemask())) < POSTPONE) {
            stack[w.sp++] = w.t;
            break;
        }
        uint32_t k = __ffs(w.t.y) - 1u;
        w.t.y &= w.t.y - 1u;
        uint32_t ti = w.t.x + k;
        const float4* tp = s.tris + 3u * ti;
        float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
        if (COUNT) ++*tests;
        if (visit(ti, a, b, c, tmax)) return WALK_DONE;
    }
    if (!(w.g.y & 0xff000000u)) {
        if (w.sp == 0) return WALK_DONE;
        w.g = stack[--w.sp];
    }
    return WALK_CONTINUE;
}

// The whole walk for one ray, handing each candidate triangle to
// `visit(tri_index, v0, v1, v2, tmax&)`, which may shrink tmax and returns
// true to stop. Returns false if a bound was exceeded (the caller flags an
// overflow).
template <bool COUNT = false, class Visit>
__device__ __forceinline__ bool traverse(const DeviceScene& s, const Ray& r, float& tmax, Visit&& visit,
                                         uint32_t* visits = nullptr, uint32_t* tests = nullptr) {
    if (s.node_count == 0) return true;
    uint2 stack[TRAVERSAL_STACK];
    Walk w;
    walk_begin(w, r);
    for (;;) {
        int st = walk_step<COUNT>(s, r, tmax, w, stack, visit, visits, tests);
        if (st == WALK_DONE) return true;
        if (st == WALK_OVERFLOW) return false;
    }
}

}  // namespace cn
