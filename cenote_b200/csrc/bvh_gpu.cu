// GPU construction of the compressed 8-wide BVH: a binary tree by PLOC
// (Meister & Bittner, "Parallel Locally-Ordered Clustering for Bounding Volume
// Hierarchy Construction", IEEE TVCG 2018) over Morton-ordered triangles,
// collapsed level by level into the node format of records.h.
//
// The collapse makes the same choices as the host build (bvh_build.cpp): the
// cost-optimal dynamic programme over the binary tree (at most eight
// children, leaf children of at most three triangles), octant-scored child
// slots, 8-bit boxes quantised in double precision. Node indices are assigned by prefix sums
// per level, so the layout is deterministic and breadth first (the top levels
// are the first nodes, which the traversal kernels may stage in shared
// memory). Closest hits do not depend on the tree: equal distances resolve by
// the (instance, primitive) key.
#include "bvh_gpu.h"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cfloat>
#include <vector>

namespace cn {
namespace {

constexpr uint32_t NONE = 0xffffffffu;
constexpr int PLOC_RADIUS = 16;
constexpr int BLOCK = 256;

// Binary nodes 0..n-1 are the leaves in Morton order (leaf j holds triangle
// tri_of[j]); merged nodes follow. lo.w / hi.w carry the children (NONE in
// lo.w marks a leaf, whose hi.w is then its triangle).
struct Tree {
    float4* lo;
    float4* hi;
    uint32_t* tris;  // triangles under the node
};

__device__ __forceinline__ uint32_t f2ord(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ float half_area(float3 lo, float3 hi) {
    float dx = fmaxf(hi.x - lo.x, 0.0f), dy = fmaxf(hi.y - lo.y, 0.0f), dz = fmaxf(hi.z - lo.z, 0.0f);
    return dx * dy + dy * dz + dz * dx;
}

// Per-triangle boxes and the centroid bounds (ordered-int atomics into cb[6]).
__global__ void k_leaf_bounds(const float4* __restrict__ in, uint32_t n, float4* lo, float4* hi, uint32_t* cb) {
    uint32_t mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 a = in[3 * size_t(i)], b = in[3 * size_t(i) + 1], c = in[3 * size_t(i) + 2];
        float3 l = make_float3(fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z));
        float3 h = make_float3(fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z));
        lo[i] = make_float4(l.x, l.y, l.z, __uint_as_float(NONE));
        hi[i] = make_float4(h.x, h.y, h.z, __uint_as_float(i));
        const float cen[3] = {0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z)};
        for (int k = 0; k < 3; ++k) {
            mn[k] = min(mn[k], f2ord(cen[k]));
            mx[k] = max(mx[k], f2ord(cen[k]));
        }
    }
    for (int k = 0; k < 3; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
            mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
    }
    if ((threadIdx.x & 31u) == 0) {
        for (int k = 0; k < 3; ++k) {
            atomicMin(cb + k, mn[k]);
            atomicMax(cb + 3 + k, mx[k]);
        }
    }
}

__device__ __forceinline__ uint64_t spread21(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

// 63-bit Morton code of each centroid in the centroid bounds.
__global__ void k_morton(const float4* __restrict__ lo, const float4* __restrict__ hi, uint32_t n, const uint32_t* cb,
                         unsigned long long* keys, uint32_t* vals) {
    float bmin[3], scale[3];
    for (int k = 0; k < 3; ++k) {
        bmin[k] = ord2f(cb[k]);
        float ext = ord2f(cb[3 + k]) - bmin[k];
        scale[k] = ext > 0.0f ? 2097151.0f / ext : 0.0f;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 l = lo[i], h = hi[i];
        const float cen[3] = {0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z)};
        uint64_t q[3];
        for (int k = 0; k < 3; ++k)
            q[k] = uint64_t(fminf(fmaxf((cen[k] - bmin[k]) * scale[k], 0.0f), 2097151.0f));
        keys[i] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
        vals[i] = i;
    }
}

// The leaves in Morton order: leaf j takes triangle tri_of[j]'s box.
__global__ void k_place_leaves(const uint32_t* __restrict__ tri_of, uint32_t n, const float4* __restrict__ lo0,
                               const float4* __restrict__ hi0, Tree t, uint32_t* clusters) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint32_t tri = tri_of[j];
        float4 l = lo0[tri], h = hi0[tri];
        t.lo[j] = make_float4(l.x, l.y, l.z, __uint_as_float(NONE));
        t.hi[j] = make_float4(h.x, h.y, h.z, __uint_as_float(tri));
        t.tris[j] = 1;
        clusters[j] = j;
    }
}

// A symmetric hash of a cluster pair: exact ties in the distance (duplicate
// triangles, regular grids) go to the pair with the smaller hash, so tied
// clusters pair up like a random matching instead of all choosing the same
// lowest index (which merges one pair per run and round, and builds a chain).
__device__ __forceinline__ uint32_t pair_hash(uint32_t i, uint32_t j) {
    uint32_t x = (min(i, j) * 0x9E3779B1u) ^ max(i, j);
    x ^= x >> 16;
    x *= 0x85EBCA6Bu;
    x ^= x >> 13;
    x *= 0xC2B2AE35u;
    x ^= x >> 16;
    return x;
}

// PLOC step 1: each cluster's nearest neighbour within PLOC_RADIUS in the
// ordered list (surface area of the union; exact ties by pair_hash).
__global__ void __launch_bounds__(BLOCK) k_nearest(Tree t, const uint32_t* __restrict__ clusters, uint32_t m,
                                                   uint32_t* nn) {
    __shared__ float3 slo[BLOCK + 2 * PLOC_RADIUS], shi[BLOCK + 2 * PLOC_RADIUS];
    const int base = int(blockIdx.x) * BLOCK - PLOC_RADIUS;
    for (int k = threadIdx.x; k < BLOCK + 2 * PLOC_RADIUS; k += BLOCK) {
        const int j = base + k;
        if (j >= 0 && j < int(m)) {
            const uint32_t c = clusters[j];
            float4 l = t.lo[c], h = t.hi[c];
            slo[k] = make_float3(l.x, l.y, l.z);
            shi[k] = make_float3(h.x, h.y, h.z);
        }
    }
    __syncthreads();
    const int i = int(blockIdx.x) * BLOCK + int(threadIdx.x);
    if (i >= int(m)) return;
    const int si = int(threadIdx.x) + PLOC_RADIUS;
    const float3 li = slo[si], hi = shi[si];
    float best = FLT_MAX;
    uint32_t best_h = 0;
    int bj = -1;
    const int j0 = max(0, i - PLOC_RADIUS), j1 = min(int(m) - 1, i + PLOC_RADIUS);
    for (int j = j0; j <= j1; ++j) {
        if (j == i) continue;
        const int sj = j - base;
        const float3 lj = slo[sj], hj = shi[sj];
        const float a = half_area(make_float3(fminf(li.x, lj.x), fminf(li.y, lj.y), fminf(li.z, lj.z)),
                                  make_float3(fmaxf(hi.x, hj.x), fmaxf(hi.y, hj.y), fmaxf(hi.z, hj.z)));
        const uint32_t h = pair_hash(uint32_t(i), uint32_t(j));
        if (a < best || (a == best && h < best_h)) {
            best = a;
            best_h = h;
            bj = j;
        }
    }
    nn[i] = uint32_t(bj);
}

// PLOC step 2: flags for the scan: low word = this cluster creates a node
// (mutual pair, lower index), high word = it survives into the next list.
__global__ void k_merge_flags(const uint32_t* __restrict__ nn, uint32_t m, unsigned long long* flags) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const uint32_t j = nn[i];
        const bool mutual = j < m && nn[j] == i;
        const bool make = mutual && i < j;
        const bool keep = !mutual || i < j;
        flags[i] = (uint64_t(keep) << 32) | uint64_t(make);
    }
}

// PLOC step 3: create the merged nodes and write the next cluster list.
__global__ void k_merge(Tree t, const uint32_t* __restrict__ clusters, const uint32_t* __restrict__ nn, uint32_t m,
                        const unsigned long long* __restrict__ flags, const unsigned long long* __restrict__ offs,
                        uint32_t node_base, uint32_t* next) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const uint64_t f = flags[i], o = offs[i];
        if (!(f >> 32)) continue;
        uint32_t out = clusters[i];
        if (f & 1ull) {
            const uint32_t a = clusters[i], b = clusters[nn[i]];
            out = node_base + uint32_t(o & 0xffffffffull);
            float4 la = t.lo[a], ha = t.hi[a], lb = t.lo[b], hb = t.hi[b];
            t.lo[out] = make_float4(fminf(la.x, lb.x), fminf(la.y, lb.y), fminf(la.z, lb.z), __uint_as_float(a));
            t.hi[out] = make_float4(fmaxf(ha.x, hb.x), fmaxf(ha.y, hb.y), fmaxf(ha.z, hb.z), __uint_as_float(b));
            t.tris[out] = t.tris[a] + t.tris[b];
        }
        next[uint32_t(o >> 32)] = out;
    }
}

// ---- collapse ------------------------------------------------------------------------
//
// Cost-optimal collapse (Ylitie, Karras & Laine 2017, §3.1), the host
// build's dynamic programme: bottom-up, cost[b][i] is the cheapest SAH cost of
// covering b's subtree with at most i child slots of the parent (i = 1..7);
// a slot is a leaf of up to three triangles or an 8-wide node whose own
// children spread over its 8 slots. c_node = 1 per node visit, c_prim = 0.3
// per triangle test, each weighted by the node's surface area relative to the
// root's. how[b][1]: 0 leaf / 1 node; how[b][i > 1]: 0 = as i - 1, k = the
// left child gets k slots; split8[b]: the left child's share when b is an
// 8-wide node. PLOC numbers a merged node above both its children, so the
// nodes one merge round made form an index range whose children are all
// lower: one launch per round, in order, is a bottom-up pass.
struct Collapse {
    float* cost;     // 8 per binary node (1..7 used)
    uint8_t* how;    // 8 per binary node
    uint8_t* split8;
};

constexpr float C_NODE = 1.0f, C_PRIM = 0.3f;

__global__ void k_collapse_cost(Tree t, Collapse c, uint32_t first, uint32_t end, double inv_root) {
    for (uint32_t b = first + blockIdx.x * blockDim.x + threadIdx.x; b < end; b += gridDim.x * blockDim.x) {
        const float4 lo = t.lo[b], hi = t.hi[b];
        double d[3] = {fmax(double(hi.x) - double(lo.x), 0.0), fmax(double(hi.y) - double(lo.y), 0.0),
                       fmax(double(hi.z) - double(lo.z), 0.0)};
        const float area = float((d[0] * d[1] + d[1] * d[2] + d[2] * d[0]) * inv_root);
        const uint32_t tris = t.tris[b];
        const float leaf = tris <= 3u ? area * C_PRIM * float(tris) : __int_as_float(0x7f800000);
        float* cb = c.cost + 8 * size_t(b);
        uint8_t* hb = c.how + 8 * size_t(b);
        const uint32_t l = __float_as_uint(lo.w);
        if (l == NONE) {
            for (int i = 0; i < 8; ++i) {
                cb[i] = leaf;
                hb[i] = 0;
            }
            c.split8[b] = 0;
            continue;
        }
        const uint32_t r = __float_as_uint(hi.w);
        float cl[8], cr[8];
        for (int i = 1; i < 8; ++i) {
            cl[i] = c.cost[8 * size_t(l) + i];
            cr[i] = c.cost[8 * size_t(r) + i];
        }
        float dist[9];
        uint8_t dsplit[9];
        for (int j = 2; j <= 8; ++j) {
            dist[j] = __int_as_float(0x7f800000);
            dsplit[j] = 0;
            for (int k = 1; k < j; ++k) {
                const float v = cl[k] + cr[j - k];
                if (v < dist[j]) {
                    dist[j] = v;
                    dsplit[j] = uint8_t(k);
                }
            }
        }
        c.split8[b] = dsplit[8] ? dsplit[8] : 4;
        const float node = dist[8] + area * C_NODE;
        cb[0] = 0.0f;
        hb[0] = 0;
        cb[1] = fminf(leaf, node);
        hb[1] = leaf <= node ? 0 : 1;
        for (int i = 2; i < 8; ++i) {
            if (dist[i] < cb[i - 1]) {
                cb[i] = dist[i];
                hb[i] = dsplit[i];
            } else {
                cb[i] = cb[i - 1];
                hb[i] = 0;
            }
        }
    }
}

// A binary node the collapse turns into a leaf child: a true leaf, or a
// subtree of at most three triangles whose leaf cost won.
__device__ __forceinline__ bool leafish(const Tree& t, const Collapse& c, uint32_t b) {
    return __float_as_uint(t.lo[b].w) == NONE || c.how[8 * size_t(b) + 1] == 0;
}

// The up-to-eight binary nodes a wide node over `b` takes as children, as the
// programme chose them.
__device__ int gather_kids(const Tree& t, const Collapse& c, uint32_t b, uint32_t kids[8]) {
    if (leafish(t, c, b)) {
        kids[0] = b;
        return 1;
    }
    uint32_t st_node[16], st_slots[16];
    int sp = 0, n = 0;
    const uint32_t k = c.split8[b];
    st_node[sp] = __float_as_uint(t.hi[b].w);
    st_slots[sp++] = 8u - k;
    st_node[sp] = __float_as_uint(t.lo[b].w);
    st_slots[sp++] = k;
    while (sp > 0 && n < 8) {
        const uint32_t x = st_node[--sp];
        uint32_t i = st_slots[sp];
        while (i > 1 && c.how[8 * size_t(x) + i] == 0) --i;
        if (i <= 1 || __float_as_uint(t.lo[x].w) == NONE) {
            kids[n++] = x;
            continue;
        }
        const uint32_t kk = c.how[8 * size_t(x) + i];
        if (sp + 2 > 16) {  // cannot happen (at most 8 slots split): keep the node whole
            kids[n++] = x;
            continue;
        }
        st_node[sp] = __float_as_uint(t.hi[x].w);
        st_slots[sp++] = i - kk;
        st_node[sp] = __float_as_uint(t.lo[x].w);
        st_slots[sp++] = kk;
    }
    return n;
}

struct Item {
    uint32_t binary, wide;
};

// Pass 1: children of every wide node of the level, and its counts (high
// word: inner children, low word: triangles) for the scan.
__global__ void k_collapse_plan(Tree t, Collapse c, const Item* __restrict__ items, uint32_t count, uint32_t* plan,
                                unsigned long long* counts) {
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < count; w += gridDim.x * blockDim.x) {
        uint32_t kids[8];
        const int n = gather_kids(t, c, items[w].binary, kids);
        uint32_t inner = 0, tris = 0;
        for (int i = 0; i < 8; ++i) {
            plan[8 * size_t(w) + i] = i < n ? kids[i] : NONE;
            if (i < n) {
                if (leafish(t, c, kids[i])) tris += t.tris[kids[i]];
                else inner++;
            }
        }
        counts[w] = (uint64_t(inner) << 32) | tris;
    }
}

// Pass 2: encode each wide node, emit its leaf triangles and the next
// level's items.
__global__ void k_collapse_emit(Tree t, Collapse cp, const Item* __restrict__ items, uint32_t count,
                                const uint32_t* __restrict__ plan,
                                const unsigned long long* __restrict__ offs, uint32_t child_base, uint32_t tri_base,
                                const float4* __restrict__ in, WideNode* nodes, float4* tris_out, Item* next) {
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < count; w += gridDim.x * blockDim.x) {
        uint32_t kids[8];
        int n = 0;
        for (int i = 0; i < 8; ++i)
            if (plan[8 * size_t(w) + i] != NONE) kids[n++] = plan[8 * size_t(w) + i];
        const uint64_t o = offs[w];
        const uint32_t first_child = child_base + uint32_t(o >> 32);
        const uint32_t first_tri = tri_base + uint32_t(o & 0xffffffffull);
        const uint32_t next_item = uint32_t(o >> 32);
        float klo[8][3], khi[8][3];
        float nlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, nhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int i = 0; i < n; ++i) {
            float4 l = t.lo[kids[i]], h = t.hi[kids[i]];
            klo[i][0] = l.x; klo[i][1] = l.y; klo[i][2] = l.z;
            khi[i][0] = h.x; khi[i][1] = h.y; khi[i][2] = h.z;
            for (int a = 0; a < 3; ++a) {
                nlo[a] = fminf(nlo[a], klo[i][a]);
                nhi[a] = fmaxf(nhi[a], khi[i][a]);
            }
        }
        // Octant slots: centre offsets scored against each slot's direction
        // (bit 2: +x, bit 1: +y, bit 0: +z); greedy best pair first.
        float nc[3];
        for (int a = 0; a < 3; ++a) nc[a] = 0.5f * (nlo[a] + nhi[a]);
        float score[8][8];
        for (int i = 0; i < n; ++i)
            for (int s = 0; s < 8; ++s) {
                float d = 0.0f;
                for (int a = 0; a < 3; ++a) {
                    float off = 0.5f * (klo[i][a] + khi[i][a]) - nc[a];
                    d += ((s >> (2 - a)) & 1) ? off : -off;
                }
                score[i][s] = d;
            }
        int kid_in_slot[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
        uint32_t kid_done = 0, slot_used = 0;
        for (int round = 0; round < n; ++round) {
            float best = -FLT_MAX;
            int bi = -1, bs = -1;
            for (int i = 0; i < n; ++i) {
                if (kid_done >> i & 1u) continue;
                for (int s = 0; s < 8; ++s) {
                    if (slot_used >> s & 1u) continue;
                    if (bi < 0 || score[i][s] > best) {
                        best = score[i][s];
                        bi = i;
                        bs = s;
                    }
                }
            }
            kid_done |= 1u << bi;
            slot_used |= 1u << bs;
            kid_in_slot[bs] = bi;
        }
        // The quantisation frame (the host build's rule, in double).
        WideNode wn;
        uint8_t* raw = reinterpret_cast<uint8_t*>(&wn);
        for (int k = 0; k < int(sizeof(WideNode)); ++k) raw[k] = 0;
        int exps[3];
        for (int a = 0; a < 3; ++a) {
            wn.p[a] = nlo[a];
            double ext = double(nhi[a]) - double(nlo[a]);
            int e = ext > 0.0 ? int(ceil(log2(ext / 254.0))) : -126;
            exps[a] = max(-126, min(127, e));
        }
        for (int guard = 0; guard < 512; ++guard) {
            bool ok = true;
            for (int i = 0; i < n && ok; ++i)
                for (int a = 0; a < 3; ++a) {
                    double sc = ldexp(1.0, exps[a]);
                    double h = ceil((double(khi[i][a]) - double(wn.p[a])) / sc + 1e-4);
                    if (h > 255.0 && exps[a] < 127) {
                        exps[a]++;
                        ok = false;
                        break;
                    }
                }
            if (ok) break;
        }
        for (int a = 0; a < 3; ++a) wn.e[a] = uint8_t(exps[a] + 127);
        wn.base_child = first_child;
        wn.base_tri = first_tri;
        uint32_t next_child = 0, tri_off = 0;
        for (int s = 0; s < 8; ++s) {
            const int i = kid_in_slot[s];
            if (i < 0) continue;
            uint8_t ql[3], qh[3];
            for (int a = 0; a < 3; ++a) {
                double sc = ldexp(1.0, exps[a]);
                double l = floor((double(klo[i][a]) - double(wn.p[a])) / sc - 1e-4);
                double h = ceil((double(khi[i][a]) - double(wn.p[a])) / sc + 1e-4);
                ql[a] = uint8_t(fmax(0.0, fmin(255.0, l)));
                qh[a] = uint8_t(fmax(0.0, fmin(255.0, h)));
            }
            wn.qlo_x[s] = ql[0]; wn.qhi_x[s] = qh[0];
            wn.qlo_y[s] = ql[1]; wn.qhi_y[s] = qh[1];
            wn.qlo_z[s] = ql[2]; wn.qhi_z[s] = qh[2];
            const uint32_t b = kids[i];
            if (leafish(t, cp, b)) {
                // Its 1..3 triangles, left before right.
                uint32_t stack[8], sp = 0, cnt = 0;
                stack[sp++] = b;
                while (sp > 0) {
                    const uint32_t x = stack[--sp];
                    const uint32_t l = __float_as_uint(t.lo[x].w);
                    if (l == NONE) {
                        const uint32_t tri = __float_as_uint(t.hi[x].w);
                        const size_t dst = 3 * size_t(first_tri + tri_off + cnt);
                        tris_out[dst] = in[3 * size_t(tri)];
                        tris_out[dst + 1] = in[3 * size_t(tri) + 1];
                        tris_out[dst + 2] = in[3 * size_t(tri) + 2];
                        ++cnt;
                    } else if (sp + 2 <= 8) {
                        stack[sp++] = __float_as_uint(t.hi[x].w);
                        stack[sp++] = l;
                    }
                }
                wn.meta[s] = uint8_t((((1u << cnt) - 1u) << 5) | tri_off);
                tri_off += cnt;
            } else {
                wn.imask |= uint8_t(1u << s);
                wn.meta[s] = uint8_t((1u << 5) | (24u + uint32_t(s)));
                next[next_item + next_child] = {b, first_child + next_child};
                ++next_child;
            }
        }
        nodes[items[w].wide] = wn;
    }
}

// Each emissive triangle's leaf index, for the shadow query's target test.
__global__ void k_light_leaves(const float4* __restrict__ tris, uint32_t n, const GeomRecord* __restrict__ geometry,
                               uint32_t* light_leaf) {
    for (uint32_t leaf = blockIdx.x * blockDim.x + threadIdx.x; leaf < n; leaf += gridDim.x * blockDim.x) {
        const uint32_t inst = __float_as_uint(tris[3 * size_t(leaf)].w);
        const uint32_t prim = __float_as_uint(tris[3 * size_t(leaf) + 1].w);
        const uint32_t first = geometry[inst].light;
        if (first != LIGHT_NONE) light_leaf[first + prim] = leaf;
    }
}

int grid_for(uint32_t n) {
    uint32_t g = (n + BLOCK - 1) / BLOCK;
    return int(g < 1 ? 1 : (g > 148u * 32u ? 148u * 32u : g));
}

struct Scratch {
    void* p = nullptr;
    ~Scratch() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t bytes) {
        if (p) cudaFree(p);
        p = nullptr;
        return cudaMalloc(&p, bytes ? bytes : 16);
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

#define BVH_TRY(x)                         \
    do {                                   \
        cudaError_t e_ = (x);              \
        if (e_ != cudaSuccess) return e_;  \
    } while (0)

cudaError_t sync_read(void* host, const void* dev, size_t bytes, cudaStream_t s) {
    BVH_TRY(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s));
    return cudaStreamSynchronize(s);
}

}  // namespace

cudaError_t build_wide_bvh_gpu(const float4* in, uint32_t n, GpuBvh* out, cudaStream_t s) {
    out->node_count = 0;
    out->depth = 0;
    out->nodes = nullptr;
    out->tris = nullptr;
    if (n == 0) return cudaSuccess;
    const size_t total = 2 * size_t(n) - 1;
    Scratch lo0, hi0, cb, keys, keys2, vals, vals2, sort_tmp, tlo, thi, ttris, cl0, cl1, nn, flags, offs, scan_tmp;
    BVH_TRY(lo0.alloc(n * 16ull));
    BVH_TRY(hi0.alloc(n * 16ull));
    BVH_TRY(cb.alloc(32));
    const uint32_t cb_init[8] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u, 0u, 0u};
    BVH_TRY(cudaMemcpyAsync(cb.p, cb_init, 32, cudaMemcpyHostToDevice, s));
    k_leaf_bounds<<<grid_for(n), BLOCK, 0, s>>>(in, n, lo0.as<float4>(), hi0.as<float4>(), cb.as<uint32_t>());
    BVH_TRY(keys.alloc(n * 8ull));
    BVH_TRY(keys2.alloc(n * 8ull));
    BVH_TRY(vals.alloc(n * 4ull));
    BVH_TRY(vals2.alloc(n * 4ull));
    k_morton<<<grid_for(n), BLOCK, 0, s>>>(lo0.as<float4>(), hi0.as<float4>(), n, cb.as<uint32_t>(),
                                           keys.as<unsigned long long>(), vals.as<uint32_t>());
    size_t sort_bytes = 0;
    BVH_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, keys.as<unsigned long long>(),
                                            keys2.as<unsigned long long>(), vals.as<uint32_t>(), vals2.as<uint32_t>(),
                                            int(n), 0, 63, s));
    BVH_TRY(sort_tmp.alloc(sort_bytes));
    BVH_TRY(cub::DeviceRadixSort::SortPairs(sort_tmp.p, sort_bytes, keys.as<unsigned long long>(),
                                            keys2.as<unsigned long long>(), vals.as<uint32_t>(), vals2.as<uint32_t>(),
                                            int(n), 0, 63, s));
    keys.alloc(0);
    keys2.alloc(0);
    sort_tmp.alloc(0);

    BVH_TRY(tlo.alloc(total * 16));
    BVH_TRY(thi.alloc(total * 16));
    BVH_TRY(ttris.alloc(total * 4));
    Tree t{tlo.as<float4>(), thi.as<float4>(), ttris.as<uint32_t>()};
    BVH_TRY(cl0.alloc(n * 4ull));
    BVH_TRY(cl1.alloc(n * 4ull));
    BVH_TRY(nn.alloc(n * 4ull));
    BVH_TRY(flags.alloc(n * 8ull));
    BVH_TRY(offs.alloc(n * 8ull));
    k_place_leaves<<<grid_for(n), BLOCK, 0, s>>>(vals2.as<uint32_t>(), n, lo0.as<float4>(), hi0.as<float4>(), t,
                                                 cl0.as<uint32_t>());
    size_t scan_bytes = 0;
    BVH_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, flags.as<unsigned long long>(),
                                          offs.as<unsigned long long>(), int(n), s));
    BVH_TRY(scan_tmp.alloc(scan_bytes));

    // PLOC: merge mutual nearest neighbours until one cluster is left. Every
    // round merges at least the globally closest pair, so at most n - 1 rounds.
    uint32_t m = n, node_next = n;
    std::vector<uint32_t> round_end;  // node_next after each merge round
    uint32_t* cur = cl0.as<uint32_t>();
    uint32_t* nxt = cl1.as<uint32_t>();
    for (uint32_t round = 0; m > 1; ++round) {
        if (round >= n) return cudaErrorUnknown;
        k_nearest<<<(m + BLOCK - 1) / BLOCK, BLOCK, 0, s>>>(t, cur, m, nn.as<uint32_t>());
        k_merge_flags<<<grid_for(m), BLOCK, 0, s>>>(nn.as<uint32_t>(), m, flags.as<unsigned long long>());
        BVH_TRY(cub::DeviceScan::ExclusiveSum(scan_tmp.p, scan_bytes, flags.as<unsigned long long>(),
                                              offs.as<unsigned long long>(), int(m), s));
        k_merge<<<grid_for(m), BLOCK, 0, s>>>(t, cur, nn.as<uint32_t>(), m, flags.as<unsigned long long>(),
                                              offs.as<unsigned long long>(), node_next, nxt);
        unsigned long long last[2];
        BVH_TRY(sync_read(&last[0], offs.as<unsigned long long>() + (m - 1), 8, s));
        BVH_TRY(sync_read(&last[1], flags.as<unsigned long long>() + (m - 1), 8, s));
        const unsigned long long tot = last[0] + last[1];
        const uint32_t made = uint32_t(tot & 0xffffffffull), kept = uint32_t(tot >> 32);
        if (made == 0 || kept >= m || node_next + made > total) return cudaErrorUnknown;
        node_next += made;
        round_end.push_back(node_next);
        m = kept;
        uint32_t* tmp = cur;
        cur = nxt;
        nxt = tmp;
    }
    uint32_t root = 0;
    BVH_TRY(sync_read(&root, cur, 4, s));
    nn.alloc(0);
    flags.alloc(0);
    offs.alloc(0);
    scan_tmp.alloc(0);

    // The collapse's costs, bottom-up: the leaves, then each merge round's
    // nodes in the order the rounds made them.
    Scratch ccost, chow, csplit;
    BVH_TRY(ccost.alloc(total * 32));
    BVH_TRY(chow.alloc(total * 8));
    BVH_TRY(csplit.alloc(total));
    Collapse cp{ccost.as<float>(), chow.as<uint8_t>(), csplit.as<uint8_t>()};
    float4 root_box[2];
    BVH_TRY(sync_read(&root_box[0], t.lo + root, 16, s));
    BVH_TRY(sync_read(&root_box[1], t.hi + root, 16, s));
    {
        const double dx = std::max(double(root_box[1].x) - double(root_box[0].x), 0.0);
        const double dy = std::max(double(root_box[1].y) - double(root_box[0].y), 0.0);
        const double dz = std::max(double(root_box[1].z) - double(root_box[0].z), 0.0);
        const double inv_root = 1.0 / std::max(dx * dy + dy * dz + dz * dx, 1e-300);
        uint32_t first = 0, end = n;
        k_collapse_cost<<<grid_for(end - first), BLOCK, 0, s>>>(t, cp, first, end, inv_root);
        for (uint32_t e : round_end) {
            first = end;
            end = e;
            if (end > first) k_collapse_cost<<<grid_for(end - first), BLOCK, 0, s>>>(t, cp, first, end, inv_root);
        }
        BVH_TRY(cudaGetLastError());
    }

    // Collapse, one level of wide nodes at a time. Every wide node holds at
    // least two binary nodes' worth of the tree, so there are fewer than n.
    Scratch nodes, tris, items0, items1, plan, counts, coffs, ctmp;
    BVH_TRY(nodes.alloc(size_t(n) * sizeof(WideNode)));
    BVH_TRY(tris.alloc(size_t(n) * 48));
    BVH_TRY(items0.alloc(size_t(n) * sizeof(Item)));
    BVH_TRY(items1.alloc(size_t(n) * sizeof(Item)));
    BVH_TRY(plan.alloc(size_t(n) * 32));
    BVH_TRY(counts.alloc(size_t(n) * 8));
    BVH_TRY(coffs.alloc(size_t(n) * 8));
    size_t cscan_bytes = 0;
    BVH_TRY(cub::DeviceScan::ExclusiveSum(nullptr, cscan_bytes, counts.as<unsigned long long>(),
                                          coffs.as<unsigned long long>(), int(n), s));
    BVH_TRY(ctmp.alloc(cscan_bytes));
    const Item first{root, 0u};
    BVH_TRY(cudaMemcpyAsync(items0.p, &first, sizeof first, cudaMemcpyHostToDevice, s));
    Item* level = items0.as<Item>();
    Item* next_level = items1.as<Item>();
    uint32_t count = 1, node_total = 1, tri_total = 0, depth = 0;
    while (count > 0) {
        if (depth > n) return cudaErrorUnknown;
        ++depth;
        k_collapse_plan<<<grid_for(count), BLOCK, 0, s>>>(t, cp, level, count, plan.as<uint32_t>(),
                                                          counts.as<unsigned long long>());
        BVH_TRY(cub::DeviceScan::ExclusiveSum(ctmp.p, cscan_bytes, counts.as<unsigned long long>(),
                                              coffs.as<unsigned long long>(), int(count), s));
        unsigned long long last[2];
        BVH_TRY(sync_read(&last[0], coffs.as<unsigned long long>() + (count - 1), 8, s));
        BVH_TRY(sync_read(&last[1], counts.as<unsigned long long>() + (count - 1), 8, s));
        const unsigned long long tot = last[0] + last[1];
        const uint32_t inner = uint32_t(tot >> 32), ntri = uint32_t(tot & 0xffffffffull);
        if (node_total + inner > n || tri_total + ntri > n) return cudaErrorUnknown;
        k_collapse_emit<<<grid_for(count), BLOCK, 0, s>>>(t, cp, level, count, plan.as<uint32_t>(),
                                                          coffs.as<unsigned long long>(), node_total, tri_total, in,
                                                          nodes.as<WideNode>(), tris.as<float4>(), next_level);
        BVH_TRY(cudaGetLastError());
        node_total += inner;
        tri_total += ntri;
        count = inner;
        Item* tmp = level;
        level = next_level;
        next_level = tmp;
    }
    if (tri_total != n) return cudaErrorUnknown;
    BVH_TRY(cudaStreamSynchronize(s));
    out->nodes = nodes.p;
    out->tris = tris.p;
    nodes.p = nullptr;
    tris.p = nullptr;
    out->node_count = node_total;
    out->depth = depth;
    return cudaSuccess;
}

void launch_light_leaves(const float4* tris, uint32_t n, const GeomRecord* geometry, uint32_t* light_leaf,
                         cudaStream_t s) {
    if (n) k_light_leaves<<<grid_for(n), BLOCK, 0, s>>>(tris, n, geometry, light_leaf);
}

}  // namespace cn
