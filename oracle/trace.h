// Test infrastructure (CPU oracle): a plain binary BVH over world-space
// triangles with the watertight ray-triangle test of Woop, Benthin & Wald,
// "Watertight Ray/Triangle Intersection" (JCGT 2013). The reference traces on
// RT cores (crates/cenote/src/gpu/accel.rs), whose traversal has no source;
// this is the CPU side of the traversal parity check. Closest-hit ties at
// equal t resolve to the smaller (instance, primitive) key so the committed
// hit does not depend on traversal order.
#pragma once
#include <cstdint>
#include <vector>
#include <algorithm>
#include <cmath>
#include "vec.h"

namespace oracle {

struct Tri {
    V3f v0, v1, v2;
    uint32_t instance, primitive;
    uint32_t mask;    // ray-mask bits this triangle's instance carries
    uint32_t opaque;  // 0: fractional-opacity instance (candidates surface)
};

struct RayPre {
    V3f org, dir;
    int kx, ky, kz;
    float sx, sy, sz;
};

inline RayPre ray_pre(V3f org, V3f dir) {
    RayPre r;
    r.org = org;
    r.dir = dir;
    float ax = std::fabs(dir.x), ay = std::fabs(dir.y), az = std::fabs(dir.z);
    r.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    r.kx = r.kz + 1 == 3 ? 0 : r.kz + 1;
    r.ky = r.kx + 1 == 3 ? 0 : r.kx + 1;
    if (dir[r.kz] < 0.0f) std::swap(r.kx, r.ky);
    r.sz = 1.0f / dir[r.kz];
    r.sx = dir[r.kx] * r.sz;
    r.sy = dir[r.ky] * r.sz;
    return r;
}

// Returns true with t in [0, tmax] and barycentrics (b1, b2) = weights on
// (v1, v2), the convention of crates/cenote/shaders/scene.slang:140-149.
inline bool intersect_tri(const RayPre& r, const Tri& t, float tmax, float* tout, float* b1, float* b2) {
    V3f A = t.v0 - r.org, B = t.v1 - r.org, C = t.v2 - r.org;
    float Ax = A[r.kx] - r.sx * A[r.kz], Ay = A[r.ky] - r.sy * A[r.kz];
    float Bx = B[r.kx] - r.sx * B[r.kz], By = B[r.ky] - r.sy * B[r.kz];
    float Cx = C[r.kx] - r.sx * C[r.kz], Cy = C[r.ky] - r.sy * C[r.kz];
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = float(double(Cx) * double(By) - double(Cy) * double(Bx));
        V = float(double(Ax) * double(Cy) - double(Ay) * double(Cx));
        W = float(double(Bx) * double(Ay) - double(By) * double(Ax));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = U + V + W;
    if (det == 0.0f) return false;
    float Az = r.sz * A[r.kz], Bz = r.sz * B[r.kz], Cz = r.sz * C[r.kz];
    float T = U * Az + V * Bz + W * Cz;
    float rcp = 1.0f / det;
    float tt = T * rcp;
    if (!(tt >= 0.0f && tt <= tmax)) return false;
    *tout = tt;
    *b1 = V * rcp;
    *b2 = W * rcp;
    return true;
}

struct BvhNode {
    V3f lo, hi;
    uint32_t left_or_first;  // interior: left child index; leaf: first triangle
    uint32_t count;          // 0: interior (right = left + 1)
};

struct Bvh {
    std::vector<BvhNode> nodes;
    std::vector<Tri> tris;  // reordered into leaf order

    static void bounds(const Tri& t, V3f* lo, V3f* hi) {
        *lo = vmin(vmin(t.v0, t.v1), t.v2);
        *hi = vmax(vmax(t.v0, t.v1), t.v2);
    }

    void build(std::vector<Tri> in) {
        tris = std::move(in);
        nodes.clear();
        if (tris.empty()) return;
        nodes.reserve(2 * tris.size());
        nodes.push_back({});
        std::vector<V3f> cen(tris.size());
        for (size_t i = 0; i < tris.size(); ++i) cen[i] = (tris[i].v0 + tris[i].v1 + tris[i].v2) * (1.0f / 3.0f);
        std::vector<uint32_t> idx(tris.size());
        for (size_t i = 0; i < idx.size(); ++i) idx[i] = uint32_t(i);
        struct Job { uint32_t node, first, count; };
        std::vector<Job> stack{{0, 0, uint32_t(tris.size())}};
        while (!stack.empty()) {
            Job j = stack.back();
            stack.pop_back();
            V3f lo(1e30f), hi(-1e30f), clo(1e30f), chi(-1e30f);
            for (uint32_t i = j.first; i < j.first + j.count; ++i) {
                V3f a, b;
                bounds(tris[idx[i]], &a, &b);
                lo = vmin(lo, a);
                hi = vmax(hi, b);
                clo = vmin(clo, cen[idx[i]]);
                chi = vmax(chi, cen[idx[i]]);
            }
            BvhNode& n = nodes[j.node];
            n.lo = lo;
            n.hi = hi;
            if (j.count <= 4) {
                n.left_or_first = j.first;
                n.count = j.count;
                continue;
            }
            V3f ext = chi - clo;
            int axis = ext.x > ext.y ? (ext.x > ext.z ? 0 : 2) : (ext.y > ext.z ? 1 : 2);
            uint32_t mid = j.first + j.count / 2;
            if (ext[axis] > 0.0f) {
                // Binned SAH over 16 bins on the widest centroid axis.
                const int NB = 16;
                struct Bin { V3f lo{1e30f}, hi{-1e30f}; uint32_t n = 0; } bins[NB];
                float scale = float(NB) / ext[axis];
                auto bin_of = [&](uint32_t i) {
                    int b = int((cen[i][axis] - clo[axis]) * scale);
                    return std::min(std::max(b, 0), NB - 1);
                };
                for (uint32_t i = j.first; i < j.first + j.count; ++i) {
                    int b = bin_of(idx[i]);
                    V3f a, c;
                    bounds(tris[idx[i]], &a, &c);
                    bins[b].lo = vmin(bins[b].lo, a);
                    bins[b].hi = vmax(bins[b].hi, c);
                    bins[b].n++;
                }
                auto area = [](V3f a, V3f b) {
                    V3f d = vmax(b - a, V3f(0.0f));
                    return d.x * d.y + d.y * d.z + d.z * d.x;
                };
                float best = 1e30f;
                int best_split = -1;
                for (int s = 1; s < NB; ++s) {
                    V3f l0(1e30f), l1(-1e30f), r0(1e30f), r1(-1e30f);
                    uint32_t nl = 0, nr = 0;
                    for (int b = 0; b < s; ++b) { l0 = vmin(l0, bins[b].lo); l1 = vmax(l1, bins[b].hi); nl += bins[b].n; }
                    for (int b = s; b < NB; ++b) { r0 = vmin(r0, bins[b].lo); r1 = vmax(r1, bins[b].hi); nr += bins[b].n; }
                    if (!nl || !nr) continue;
                    float cost = area(l0, l1) * float(nl) + area(r0, r1) * float(nr);
                    if (cost < best) { best = cost; best_split = s; }
                }
                if (best_split > 0) {
                    auto it = std::partition(idx.begin() + j.first, idx.begin() + j.first + j.count,
                                             [&](uint32_t i) { return bin_of(i) < best_split; });
                    mid = uint32_t(it - idx.begin());
                } else {
                    std::nth_element(idx.begin() + j.first, idx.begin() + mid, idx.begin() + j.first + j.count,
                                     [&](uint32_t a, uint32_t b) { return cen[a][axis] < cen[b][axis]; });
                }
            }
            if (mid == j.first || mid == j.first + j.count) mid = j.first + j.count / 2;
            uint32_t left = uint32_t(nodes.size());
            nodes.push_back({});
            nodes.push_back({});
            nodes[j.node].left_or_first = left;
            nodes[j.node].count = 0;
            stack.push_back({left, j.first, mid - j.first});
            stack.push_back({left + 1, mid, j.first + j.count - mid});
        }
        std::vector<Tri> ordered(tris.size());
        for (size_t i = 0; i < idx.size(); ++i) ordered[i] = tris[idx[i]];
        tris.swap(ordered);
    }

    static bool slab(const BvhNode& n, const RayPre& r, V3f inv, float tmax, float* tnear) {
        // Conservative against rounding: a node is culled only when its entry
        // lies clearly beyond the current hit (and the far planes get two ulps).
        float t0 = 0.0f, t1 = tmax * 1.00002f;
        for (int a = 0; a < 3; ++a) {
            float ta = (n.lo[a] - r.org[a]) * inv[a];
            float tb = (n.hi[a] - r.org[a]) * inv[a];
            if (ta > tb) std::swap(ta, tb);
            tb *= 1.0f + 2.0f * 1.1920929e-07f;  // robust slab (Ize 2013)
            t0 = ta > t0 ? ta : t0;
            t1 = tb < t1 ? tb : t1;
        }
        *tnear = t0;
        return t0 <= t1;
    }

    // Visit every triangle whose leaf box the ray reaches within the current
    // tmax, calling f(tri index) -> updated tmax. Order is near-first but the
    // callers' results do not depend on it (ties break by key).
    template <class F>
    void walk(const RayPre& r, float tmax, F&& f) const {
        if (nodes.empty()) return;
        V3f inv(1.0f / r.dir.x, 1.0f / r.dir.y, 1.0f / r.dir.z);
        uint32_t stack[256];
        int sp = 0;
        stack[sp++] = 0;
        while (sp) {
            const BvhNode& n = nodes[stack[--sp]];
            float tn;
            if (!slab(n, r, inv, tmax, &tn)) continue;
            if (n.count) {
                for (uint32_t i = n.left_or_first; i < n.left_or_first + n.count; ++i) tmax = f(i, tmax);
                continue;
            }
            float ta, tb;
            bool ha = slab(nodes[n.left_or_first], r, inv, tmax, &ta);
            bool hb = slab(nodes[n.left_or_first + 1], r, inv, tmax, &tb);
            if (ha && hb) {
                if (ta <= tb) { stack[sp++] = n.left_or_first + 1; stack[sp++] = n.left_or_first; }
                else { stack[sp++] = n.left_or_first; stack[sp++] = n.left_or_first + 1; }
            } else if (ha) stack[sp++] = n.left_or_first;
            else if (hb) stack[sp++] = n.left_or_first + 1;
        }
    }
};

inline uint64_t hit_key(uint32_t inst, uint32_t prim) { return (uint64_t(inst) << 32) | prim; }

}  // namespace oracle
