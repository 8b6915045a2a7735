// GPU construction of the compressed 8-wide BVH: a binary tree by binned SAH
// (top down, breadth first, the host build's split rule) or by PLOC (Meister &
// Bittner, "Parallel Locally-Ordered Clustering for Bounding Volume Hierarchy
// Construction", IEEE TVCG 2018) over Morton-ordered triangles, collapsed
// level by level into the node format of records.h.
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

// Per-triangle boxes, the centroid bounds and the scene box (ordered-int
// atomics into cb[0..5] and cb[6..11]).
__global__ void k_leaf_bounds(const float4* __restrict__ in, uint32_t n, float4* lo, float4* hi, uint32_t* cb) {
    uint32_t mn[6], mx[6];
    for (int k = 0; k < 6; ++k) {
        mn[k] = 0xffffffffu;
        mx[k] = 0u;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 a = in[3 * size_t(i)], b = in[3 * size_t(i) + 1], c = in[3 * size_t(i) + 2];
        float3 l = make_float3(fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z));
        float3 h = make_float3(fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z));
        lo[i] = make_float4(l.x, l.y, l.z, __uint_as_float(NONE));
        hi[i] = make_float4(h.x, h.y, h.z, __uint_as_float(i));
        const float cen[3] = {0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z)};
        const float bl[3] = {l.x, l.y, l.z}, bh[3] = {h.x, h.y, h.z};
        for (int k = 0; k < 3; ++k) {
            mn[k] = min(mn[k], f2ord(cen[k]));
            mx[k] = max(mx[k], f2ord(cen[k]));
            mn[3 + k] = min(mn[3 + k], f2ord(bl[k]));
            mx[3 + k] = max(mx[3 + k], f2ord(bh[k]));
        }
    }
    for (int k = 0; k < 6; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
            mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
    }
    if ((threadIdx.x & 31u) == 0) {
        for (int k = 0; k < 3; ++k) {
            atomicMin(cb + k, mn[k]);
            atomicMax(cb + 3 + k, mx[k]);
            atomicMin(cb + 6 + k, mn[3 + k]);
            atomicMax(cb + 9 + k, mx[3 + k]);
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

// ---- binned SAH, top down and breadth first ------------------------------------------
//
// The host build's rule (bvh_build.cpp) on the device: every task (a range of
// the triangle order under one binary node) bins its triangles' centroids
// into 32 bins per axis and splits where A_left·N_left + A_right·N_right is
// least (ties to the lower axis, then the lower bin); equal centroids, or a
// task past 48 levels, split by position at the middle, which bounds the
// depth. A task of at most 8,192 triangles bins and partitions in one warp
// (bins in shared memory); larger tasks bin in chunks of 8,192 over many
// CTAs and partition through a device-wide scan. Each level's internal nodes
// take a contiguous index range after the n leaves (leaf j = position j of
// the final order), so the collapse runs bottom-up level by level. Every
// step is deterministic (integer atomics on order-preserving float codes).
constexpr int NBIN = 32;
constexpr uint32_t WARP_TASK_MAX = 8192;
constexpr uint32_t CHUNK = 8192;
constexpr uint32_t SAH_LEVEL_MAX = 48;
constexpr int BIN_WORDS = 13;  // box lo, box hi, centroid lo, centroid hi (ordered codes), count
constexpr int BINS_WORDS = 3 * NBIN * BIN_WORDS;
constexpr int SAH_WARPS = 8;

struct SahTask {
    uint32_t first, count, node, pad;
    float4 lo, hi;    // the node's box
    float4 clo, chi;  // its centroids' bounds
};

struct SahSplit {
    uint32_t axis;  // 0..2: binned split on that axis; 3: by position at the middle
    uint32_t bin;   // the right side's first bin
    uint32_t nl;    // triangles on the left
    uint32_t pad;
    float4 lo[2], hi[2], clo[2], chi[2];  // left, right
};

struct SahChunk {
    uint32_t task, slot, begin, end;
};

__device__ __forceinline__ float3 centroid_of(float4 l, float4 h) {
    return make_float3(0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z));
}

__device__ __forceinline__ float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
__device__ __forceinline__ float comp4(float4 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// The host's binning: int((c - lo) · (32 / extent)), clamped.
__device__ __forceinline__ int bin_of(float c, float lo, float scale) {
    return min(NBIN - 1, max(0, int((c - lo) * scale)));
}

__device__ __forceinline__ void bins_init(uint32_t* bins, uint32_t lane, uint32_t lanes) {
    for (uint32_t w = lane; w < uint32_t(BINS_WORDS); w += lanes) {
        const uint32_t f = w % BIN_WORDS;
        bins[w] = (f < 3 || (f >= 6 && f < 9)) ? 0xffffffffu : 0u;
    }
}

__device__ __forceinline__ void bins_add(uint32_t* bins, const float scale[3], const float clo[3], float4 l, float4 h) {
    const float3 c = centroid_of(l, h);
    const uint32_t code[12] = {f2ord(l.x), f2ord(l.y), f2ord(l.z), f2ord(h.x), f2ord(h.y), f2ord(h.z),
                               f2ord(c.x), f2ord(c.y), f2ord(c.z), f2ord(c.x), f2ord(c.y), f2ord(c.z)};
    for (int a = 0; a < 3; ++a) {
        uint32_t* w = bins + (a * NBIN + bin_of(comp(c, a), clo[a], scale[a])) * BIN_WORDS;
        for (int f = 0; f < 3; ++f) atomicMin(w + f, code[f]);
        for (int f = 3; f < 6; ++f) atomicMax(w + f, code[f]);
        for (int f = 6; f < 9; ++f) atomicMin(w + f, code[f]);
        for (int f = 9; f < 12; ++f) atomicMax(w + f, code[f]);
        atomicAdd(w + 12, 1u);
    }
}

__device__ __forceinline__ void task_scale(const SahTask& t, float scale[3], float clo[3]) {
    for (int a = 0; a < 3; ++a) {
        clo[a] = comp4(t.clo, a);
        const float ext = comp4(t.chi, a) - clo[a];
        scale[a] = ext > 0.0f ? float(NBIN) / ext : 0.0f;
    }
}

// Large tasks: each CTA bins one chunk in shared memory and merges it into
// the task's global bins.
__global__ void __launch_bounds__(BLOCK) k_sah_bin_chunks(const SahChunk* __restrict__ chunks, const SahTask* __restrict__ tasks,
                                                        const uint32_t* __restrict__ idx, const float4* __restrict__ lo0,
                                                        const float4* __restrict__ hi0, uint32_t* gbins) {
    __shared__ uint32_t bins[BINS_WORDS];
    const SahChunk ch = chunks[blockIdx.x];
    const SahTask t = tasks[ch.task];
    float scale[3], clo[3];
    task_scale(t, scale, clo);
    bins_init(bins, threadIdx.x, blockDim.x);
    __syncthreads();
    for (uint32_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        const uint32_t p = idx[i];
        bins_add(bins, scale, clo, lo0[p], hi0[p]);
    }
    __syncthreads();
    uint32_t* g = gbins + size_t(ch.slot) * BINS_WORDS;
    for (uint32_t w = threadIdx.x; w < uint32_t(BINS_WORDS); w += blockDim.x) {
        const uint32_t f = w % BIN_WORDS, b = w / BIN_WORDS;
        if (bins[b * BIN_WORDS + 12] == 0u) continue;
        if (f == 12) atomicAdd(g + w, bins[w]);
        else if (f < 3 || (f >= 6 && f < 9)) atomicMin(g + w, bins[w]);
        else atomicMax(g + w, bins[w]);
    }
}

__global__ void k_sah_bins_init(uint32_t* gbins, uint32_t sets) {
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < sets * uint32_t(BINS_WORDS); w += gridDim.x * blockDim.x) {
        const uint32_t f = w % BIN_WORDS;
        gbins[w] = (f < 3 || (f >= 6 && f < 9)) ? 0xffffffffu : 0u;
    }
}

struct Box6 {
    float3 lo, hi;
};

__device__ __forceinline__ Box6 box_empty() {
    const float inf = __int_as_float(0x7f800000);
    return {make_float3(inf, inf, inf), make_float3(-inf, -inf, -inf)};
}
__device__ __forceinline__ Box6 box_union(Box6 a, Box6 b) {
    return {make_float3(fminf(a.lo.x, b.lo.x), fminf(a.lo.y, b.lo.y), fminf(a.lo.z, b.lo.z)),
            make_float3(fmaxf(a.hi.x, b.hi.x), fmaxf(a.hi.y, b.hi.y), fmaxf(a.hi.z, b.hi.z))};
}
__device__ __forceinline__ Box6 box_shfl(Box6 b, int src, bool up, int delta) {
    Box6 o;
    if (up) {
        o.lo = make_float3(__shfl_up_sync(0xffffffffu, b.lo.x, delta), __shfl_up_sync(0xffffffffu, b.lo.y, delta),
                           __shfl_up_sync(0xffffffffu, b.lo.z, delta));
        o.hi = make_float3(__shfl_up_sync(0xffffffffu, b.hi.x, delta), __shfl_up_sync(0xffffffffu, b.hi.y, delta),
                           __shfl_up_sync(0xffffffffu, b.hi.z, delta));
    } else {
        o.lo = make_float3(__shfl_down_sync(0xffffffffu, b.lo.x, delta), __shfl_down_sync(0xffffffffu, b.lo.y, delta),
                           __shfl_down_sync(0xffffffffu, b.lo.z, delta));
        o.hi = make_float3(__shfl_down_sync(0xffffffffu, b.hi.x, delta), __shfl_down_sync(0xffffffffu, b.hi.y, delta),
                           __shfl_down_sync(0xffffffffu, b.hi.z, delta));
    }
    (void)src;
    return o;
}
__device__ __forceinline__ Box6 box_reduce(Box6 b) {
    for (int o = 16; o > 0; o >>= 1) {
        Box6 x;
        x.lo = make_float3(__shfl_xor_sync(0xffffffffu, b.lo.x, o), __shfl_xor_sync(0xffffffffu, b.lo.y, o),
                           __shfl_xor_sync(0xffffffffu, b.lo.z, o));
        x.hi = make_float3(__shfl_xor_sync(0xffffffffu, b.hi.x, o), __shfl_xor_sync(0xffffffffu, b.hi.y, o),
                           __shfl_xor_sync(0xffffffffu, b.hi.z, o));
        b = box_union(b, x);
    }
    return b;
}
__device__ __forceinline__ float box_area(Box6 b) {
    const float dx = fmaxf(b.hi.x - b.lo.x, 0.0f), dy = fmaxf(b.hi.y - b.lo.y, 0.0f), dz = fmaxf(b.hi.z - b.lo.z, 0.0f);
    return dx * dy + dy * dz + dz * dx;
}

// Bin (axis, b): its triangles' box and centroid bounds (empty when count is 0).
__device__ __forceinline__ uint32_t bin_read(const uint32_t* bins, int axis, int b, Box6* box, Box6* cbox) {
    const uint32_t* w = bins + (axis * NBIN + b) * BIN_WORDS;
    const uint32_t n = w[12];
    if (n == 0u) {
        *box = box_empty();
        *cbox = box_empty();
        return 0u;
    }
    box->lo = make_float3(ord2f(w[0]), ord2f(w[1]), ord2f(w[2]));
    box->hi = make_float3(ord2f(w[3]), ord2f(w[4]), ord2f(w[5]));
    cbox->lo = make_float3(ord2f(w[6]), ord2f(w[7]), ord2f(w[8]));
    cbox->hi = make_float3(ord2f(w[9]), ord2f(w[10]), ord2f(w[11]));
    return n;
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// One warp per task: bin (or take the chunk passes' bins), choose the split,
// and record the children's counts, boxes and centroid bounds.
__global__ void __launch_bounds__(SAH_WARPS * 32) k_sah_decide(const SahTask* __restrict__ tasks, uint32_t count,
                                                                const uint32_t* __restrict__ slots,
                                                                const uint32_t* __restrict__ gbins,
                                                                const uint32_t* __restrict__ idx,
                                                                const float4* __restrict__ lo0,
                                                                const float4* __restrict__ hi0, uint32_t by_position,
                                                                SahSplit* splits, uint32_t* internal) {
    extern __shared__ uint32_t sah_smem[];
    const uint32_t wib = threadIdx.x / 32u, lane = lane_id();
    const uint32_t w = blockIdx.x * SAH_WARPS + wib;
    if (w >= count) return;
    uint32_t* bins = sah_smem + wib * BINS_WORDS;
    const SahTask t = tasks[w];
    float scale[3], clo[3];
    task_scale(t, scale, clo);
    const uint32_t slot = slots ? slots[w] : NONE;
    if (slot != NONE) {
        for (uint32_t k = lane; k < uint32_t(BINS_WORDS); k += 32u) bins[k] = gbins[size_t(slot) * BINS_WORDS + k];
    } else {
        bins_init(bins, lane, 32u);
        __syncwarp();
        for (uint32_t i = t.first + lane; i < t.first + t.count; i += 32u) {
            const uint32_t p = idx[i];
            bins_add(bins, scale, clo, lo0[p], hi0[p]);
        }
    }
    __syncwarp();
    const float inf = __int_as_float(0x7f800000);
    float best = inf;
    uint32_t best_axis = 3u, best_bin = 0u;
    if (!by_position) {
        for (int a = 0; a < 3; ++a) {
            if (!(scale[a] > 0.0f)) continue;
            Box6 b, cb;
            uint32_t n = bin_read(bins, a, int(lane), &b, &cb);
            Box6 pre = b, suf = b;
            uint32_t npre = n, nsuf = n;
            for (int d = 1; d < 32; d <<= 1) {
                const Box6 u = box_shfl(pre, 0, true, d);
                const uint32_t nu = __shfl_up_sync(0xffffffffu, npre, d);
                const Box6 v = box_shfl(suf, 0, false, d);
                const uint32_t nv = __shfl_down_sync(0xffffffffu, nsuf, d);
                if (lane >= uint32_t(d)) {
                    pre = box_union(pre, u);
                    npre += nu;
                }
                if (lane + uint32_t(d) < 32u) {
                    suf = box_union(suf, v);
                    nsuf += nv;
                }
            }
            const Box6 left = box_shfl(pre, 0, true, 1);  // bins [0, lane)
            const uint32_t nl = __shfl_up_sync(0xffffffffu, npre, 1);
            if (lane >= 1u && nl > 0u && nsuf > 0u) {
                const float c = box_area(left) * float(nl) + box_area(suf) * float(nsuf);
                if (c < best) {
                    best = c;
                    best_axis = uint32_t(a);
                    best_bin = lane;
                }
            }
        }
        for (int o = 16; o > 0; o >>= 1) {  // least (cost, axis, bin)
            const float oc = __shfl_xor_sync(0xffffffffu, best, o);
            const uint32_t oa = __shfl_xor_sync(0xffffffffu, best_axis, o);
            const uint32_t ob = __shfl_xor_sync(0xffffffffu, best_bin, o);
            if (oc < best || (oc == best && (oa < best_axis || (oa == best_axis && ob < best_bin)))) {
                best = oc;
                best_axis = oa;
                best_bin = ob;
            }
        }
    }
    Box6 side_box[2] = {box_empty(), box_empty()}, side_cbox[2] = {box_empty(), box_empty()};
    uint32_t nl;
    if (best_axis < 3u) {
        Box6 b, cb;
        const uint32_t n = bin_read(bins, int(best_axis), int(lane), &b, &cb);
        const int s = lane < best_bin ? 0 : 1;
        side_box[s] = b;
        side_cbox[s] = cb;
        uint32_t nleft = lane < best_bin ? n : 0u;
        for (int o = 16; o > 0; o >>= 1) nleft += __shfl_xor_sync(0xffffffffu, nleft, o);
        nl = nleft;
    } else {
        nl = t.count / 2u;
        for (uint32_t i = t.first + lane; i < t.first + t.count; i += 32u) {
            const uint32_t p = idx[i];
            const float4 l = lo0[p], h = hi0[p];
            const float3 c = centroid_of(l, h);
            const int s = (i - t.first) < nl ? 0 : 1;
            side_box[s] = box_union(side_box[s], Box6{make_float3(l.x, l.y, l.z), make_float3(h.x, h.y, h.z)});
            side_cbox[s] = box_union(side_cbox[s], Box6{c, c});
        }
    }
    for (int s = 0; s < 2; ++s) {
        side_box[s] = box_reduce(side_box[s]);
        side_cbox[s] = box_reduce(side_cbox[s]);
    }
    if (lane == 0u) {
        SahSplit sp;
        sp.axis = best_axis;
        sp.bin = best_bin;
        sp.nl = nl;
        sp.pad = 0u;
        for (int s = 0; s < 2; ++s) {
            sp.lo[s] = make_float4(side_box[s].lo.x, side_box[s].lo.y, side_box[s].lo.z, 0.0f);
            sp.hi[s] = make_float4(side_box[s].hi.x, side_box[s].hi.y, side_box[s].hi.z, 0.0f);
            sp.clo[s] = make_float4(side_cbox[s].lo.x, side_cbox[s].lo.y, side_cbox[s].lo.z, 0.0f);
            sp.chi[s] = make_float4(side_cbox[s].hi.x, side_cbox[s].hi.y, side_cbox[s].hi.z, 0.0f);
        }
        splits[w] = sp;
        internal[w] = (nl > 1u ? 1u : 0u) + (t.count - nl > 1u ? 1u : 0u);
    }
}

__device__ __forceinline__ bool goes_left(const SahTask& t, const SahSplit& sp, uint32_t i, float4 l, float4 h) {
    if (sp.axis >= 3u) return (i - t.first) < sp.nl;
    const int a = int(sp.axis);
    const float lo = comp4(t.clo, a), ext = comp4(t.chi, a) - lo;
    const float scale = ext > 0.0f ? float(NBIN) / ext : 0.0f;
    return uint32_t(bin_of(comp(centroid_of(l, h), a), lo, scale)) < sp.bin;
}

// Small tasks: one warp partitions its range stably (left side first).
__global__ void __launch_bounds__(SAH_WARPS * 32) k_sah_partition(const SahTask* __restrict__ tasks, uint32_t count,
                                                                   const uint32_t* __restrict__ slots,
                                                                   const SahSplit* __restrict__ splits,
                                                                   const uint32_t* __restrict__ idx,
                                                                   const float4* __restrict__ lo0,
                                                                   const float4* __restrict__ hi0, uint32_t* idx_next) {
    const uint32_t lane = lane_id();
    const uint32_t w = blockIdx.x * SAH_WARPS + threadIdx.x / 32u;
    if (w >= count || (slots && slots[w] != NONE)) return;
    const SahTask t = tasks[w];
    const SahSplit sp = splits[w];
    uint32_t base_l = t.first, base_r = t.first + sp.nl;
    const uint32_t below = (1u << lane) - 1u;
    for (uint32_t i0 = t.first; i0 < t.first + t.count; i0 += 32u) {
        const uint32_t i = i0 + lane;
        const bool valid = i < t.first + t.count;
        uint32_t p = 0u;
        bool left = false;
        if (valid) {
            p = idx[i];
            left = goes_left(t, sp, i, lo0[p], hi0[p]);
        }
        const uint32_t ml = __ballot_sync(0xffffffffu, valid && left), mr = __ballot_sync(0xffffffffu, valid && !left);
        const uint32_t dest = left ? base_l + __popc(ml & below) : base_r + __popc(mr & below);
        // The sides repeat the decision's binning exactly; the bound only
        // keeps a broken split inside the task (the collapse's triangle
        // count then rejects the tree).
        if (valid && dest < t.first + t.count) idx_next[dest] = p;
        base_l += __popc(ml);
        base_r += __popc(mr);
    }
}

// Large tasks: side flags per chunk, a device-wide exclusive scan, then a
// scatter by each position's rank within its task.
__global__ void __launch_bounds__(BLOCK) k_sah_flags(const SahChunk* __restrict__ chunks, const SahTask* __restrict__ tasks,
                                                   const SahSplit* __restrict__ splits, const uint32_t* __restrict__ idx,
                                                   const float4* __restrict__ lo0, const float4* __restrict__ hi0,
                                                   uint32_t* flags) {
    const SahChunk ch = chunks[blockIdx.x];
    const SahTask t = tasks[ch.task];
    const SahSplit sp = splits[ch.task];
    for (uint32_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        const uint32_t p = idx[i];
        flags[i] = goes_left(t, sp, i, lo0[p], hi0[p]) ? 1u : 0u;
    }
}

__global__ void __launch_bounds__(BLOCK) k_sah_scatter(const SahChunk* __restrict__ chunks, const SahTask* __restrict__ tasks,
                                                     const SahSplit* __restrict__ splits, const uint32_t* __restrict__ idx,
                                                     const uint32_t* __restrict__ flags, const uint32_t* __restrict__ rank,
                                                     uint32_t* idx_next) {
    const SahChunk ch = chunks[blockIdx.x];
    const SahTask t = tasks[ch.task];
    const uint32_t nl = splits[ch.task].nl, r0 = rank[t.first];
    for (uint32_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        const uint32_t r = rank[i] - r0;
        const uint32_t dest = flags[i] ? t.first + r : t.first + nl + (i - t.first - r);
        if (dest < t.first + t.count) idx_next[dest] = idx[i];
    }
}

// Write every task's binary node, its leaf children and its internal
// children's tasks (numbered from node_base in task order).
__global__ void k_sah_emit(const SahTask* __restrict__ tasks, uint32_t count, const SahSplit* __restrict__ splits,
                           const uint32_t* __restrict__ offs, uint32_t node_base, const uint32_t* __restrict__ idx_next,
                           const float4* __restrict__ lo0, const float4* __restrict__ hi0, Tree tr, SahTask* next,
                           uint32_t* max_count) {
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < count; w += gridDim.x * blockDim.x) {
        const SahTask t = tasks[w];
        const SahSplit sp = splits[w];
        const uint32_t n[2] = {sp.nl, t.count - sp.nl}, first[2] = {t.first, t.first + sp.nl};
        uint32_t o = offs[w], id[2], big = 0u;
        for (int s = 0; s < 2; ++s) {
            if (n[s] > 1u) {
                id[s] = node_base + o;
                SahTask c;
                c.first = first[s];
                c.count = n[s];
                c.node = id[s];
                c.pad = 0u;
                c.lo = sp.lo[s];
                c.hi = sp.hi[s];
                c.clo = sp.clo[s];
                c.chi = sp.chi[s];
                next[o++] = c;
                big = max(big, n[s]);
            } else {
                id[s] = first[s];
                const uint32_t tri = idx_next[first[s]];
                const float4 l = lo0[tri], h = hi0[tri];
                tr.lo[id[s]] = make_float4(l.x, l.y, l.z, __uint_as_float(NONE));
                tr.hi[id[s]] = make_float4(h.x, h.y, h.z, __uint_as_float(tri));
                tr.tris[id[s]] = 1u;
            }
        }
        tr.lo[t.node] = make_float4(t.lo.x, t.lo.y, t.lo.z, __uint_as_float(id[0]));
        tr.hi[t.node] = make_float4(t.hi.x, t.hi.y, t.hi.z, __uint_as_float(id[1]));
        tr.tris[t.node] = t.count;
        if (big) atomicMax(max_count, big);
    }
}

// The root task from the scene bounds (cb: centroid lo/hi, then box lo/hi,
// as ordered codes), and the identity order.
__global__ void k_sah_root(const uint32_t* __restrict__ cb, uint32_t n, SahTask* task, uint32_t* idx) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) idx[i] = i;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        SahTask t;
        t.first = 0u;
        t.count = n;
        t.node = n;
        t.pad = 0u;
        t.clo = make_float4(ord2f(cb[0]), ord2f(cb[1]), ord2f(cb[2]), 0.0f);
        t.chi = make_float4(ord2f(cb[3]), ord2f(cb[4]), ord2f(cb[5]), 0.0f);
        t.lo = make_float4(ord2f(cb[6]), ord2f(cb[7]), ord2f(cb[8]), 0.0f);
        t.hi = make_float4(ord2f(cb[9]), ord2f(cb[10]), ord2f(cb[11]), 0.0f);
        *task = t;
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

#ifndef CN_COLLAPSE_C_PRIM
#define CN_COLLAPSE_C_PRIM 0.3f
#endif
constexpr float C_NODE = 1.0f, C_PRIM = CN_COLLAPSE_C_PRIM;

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

namespace {

// PLOC binary tree over the Morton order (leaf j holds the j-th triangle of
// that order); `order` receives the node ranges a bottom-up pass takes.
cudaError_t binary_ploc(uint32_t n, const float4* lo0, const float4* hi0, const uint32_t* cb, Tree t, uint32_t* root,
                        std::vector<std::pair<uint32_t, uint32_t>>* order, cudaStream_t s) {
    const size_t total = 2 * size_t(n) - 1;
    Scratch keys, keys2, vals, vals2, sort_tmp, cl0, cl1, nn, flags, offs, scan_tmp;
    BVH_TRY(keys.alloc(n * 8ull));
    BVH_TRY(keys2.alloc(n * 8ull));
    BVH_TRY(vals.alloc(n * 4ull));
    BVH_TRY(vals2.alloc(n * 4ull));
    k_morton<<<grid_for(n), BLOCK, 0, s>>>(lo0, hi0, n, cb,
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

    BVH_TRY(cl0.alloc(n * 4ull));
    BVH_TRY(cl1.alloc(n * 4ull));
    BVH_TRY(nn.alloc(n * 4ull));
    BVH_TRY(flags.alloc(n * 8ull));
    BVH_TRY(offs.alloc(n * 8ull));
    k_place_leaves<<<grid_for(n), BLOCK, 0, s>>>(vals2.as<uint32_t>(), n, lo0, hi0, t,
                                                 cl0.as<uint32_t>());
    size_t scan_bytes = 0;
    BVH_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, flags.as<unsigned long long>(),
                                          offs.as<unsigned long long>(), int(n), s));
    BVH_TRY(scan_tmp.alloc(scan_bytes));

    // PLOC: merge mutual nearest neighbours until one cluster is left. Every
    // round merges at least the globally closest pair, so at most n - 1 rounds.
    uint32_t m = n, node_next = n;
    order->assign(1, {0u, n});  // the leaves, then each merge round's nodes
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
        order->push_back({node_next, node_next + made});
        node_next += made;
        m = kept;
        uint32_t* tmp = cur;
        cur = nxt;
        nxt = tmp;
    }
    BVH_TRY(sync_read(root, cur, 4, s));
    nn.alloc(0);
    flags.alloc(0);
    offs.alloc(0);
    scan_tmp.alloc(0);

    return cudaSuccess;
}

// Binned SAH binary tree, top down one level at a time (leaf j holds the
// triangle at position j of the final order).
cudaError_t binary_sah(uint32_t n, const float4* lo0, const float4* hi0, const uint32_t* cb, Tree t, uint32_t* root,
                       std::vector<std::pair<uint32_t, uint32_t>>* order, cudaStream_t s) {
    Scratch idx0, idx1, tasks0, tasks1, splits, internal, offs, scan_tmp, maxc, flags, rank, rank_tmp, gbins, chunks,
        slots;
    BVH_TRY(idx0.alloc(n * 4ull));
    BVH_TRY(idx1.alloc(n * 4ull));
    if (n == 1) {
        BVH_TRY(cudaMemsetAsync(idx0.p, 0, 4, s));
        k_place_leaves<<<1, 32, 0, s>>>(idx0.as<uint32_t>(), 1u, lo0, hi0, t, idx1.as<uint32_t>());
        *root = 0u;
        order->assign(1, {0u, 1u});
        return cudaGetLastError();
    }
    const size_t max_tasks = n / 2 + 1;  // every task holds at least two triangles
    BVH_TRY(tasks0.alloc(max_tasks * sizeof(SahTask)));
    BVH_TRY(tasks1.alloc(max_tasks * sizeof(SahTask)));
    BVH_TRY(splits.alloc(max_tasks * sizeof(SahSplit)));
    BVH_TRY(internal.alloc(max_tasks * 4));
    BVH_TRY(offs.alloc(max_tasks * 4));
    BVH_TRY(maxc.alloc(4));
    BVH_TRY(flags.alloc(n * 4ull));
    BVH_TRY(rank.alloc(n * 4ull));
    size_t scan_bytes = 0, rank_bytes = 0;
    BVH_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, internal.as<uint32_t>(), offs.as<uint32_t>(),
                                          int(max_tasks), s));
    BVH_TRY(scan_tmp.alloc(scan_bytes));
    BVH_TRY(cub::DeviceScan::ExclusiveSum(nullptr, rank_bytes, flags.as<uint32_t>(), rank.as<uint32_t>(), int(n), s));
    BVH_TRY(rank_tmp.alloc(rank_bytes));
    const uint32_t max_large = n / WARP_TASK_MAX + 1;
    BVH_TRY(gbins.alloc(size_t(max_large) * BINS_WORDS * 4));
    BVH_TRY(chunks.alloc((size_t(n) / CHUNK + 2 * max_large) * sizeof(SahChunk)));
    BVH_TRY(slots.alloc(max_tasks * 4));
    k_sah_root<<<grid_for(n), BLOCK, 0, s>>>(cb, n, tasks0.as<SahTask>(), idx0.as<uint32_t>());
    BVH_TRY(cudaGetLastError());
    *root = n;
    std::vector<std::pair<uint32_t, uint32_t>> levels;
    SahTask* cur = tasks0.as<SahTask>();
    SahTask* nxt = tasks1.as<SahTask>();
    uint32_t* idx = idx0.as<uint32_t>();
    uint32_t* idx_next = idx1.as<uint32_t>();
    uint32_t count = 1, base = n, largest = n;
    std::vector<SahTask> host_tasks;
    std::vector<SahChunk> host_chunks;
    std::vector<uint32_t> host_slots;
    const size_t smem = size_t(SAH_WARPS) * BINS_WORDS * 4;
    for (uint32_t level = 0; count > 0; ++level) {
        if (level > n) return cudaErrorUnknown;
        levels.push_back({base, base + count});
        // Tasks above the one-warp size bin in chunks over many CTAs.
        const bool large = largest > WARP_TASK_MAX;
        uint32_t nchunks = 0;
        if (large) {
            host_tasks.resize(count);
            BVH_TRY(sync_read(host_tasks.data(), cur, count * sizeof(SahTask), s));
            host_chunks.clear();
            host_slots.assign(count, NONE);
            uint32_t nslots = 0;
            for (uint32_t k = 0; k < count; ++k) {
                if (host_tasks[k].count <= WARP_TASK_MAX) continue;
                host_slots[k] = nslots;
                for (uint32_t b0 = host_tasks[k].first; b0 < host_tasks[k].first + host_tasks[k].count; b0 += CHUNK)
                    host_chunks.push_back({k, nslots, b0, std::min(b0 + CHUNK, host_tasks[k].first + host_tasks[k].count)});
                ++nslots;
            }
            nchunks = uint32_t(host_chunks.size());
            BVH_TRY(cudaMemcpyAsync(chunks.p, host_chunks.data(), nchunks * sizeof(SahChunk), cudaMemcpyHostToDevice, s));
            BVH_TRY(cudaMemcpyAsync(slots.p, host_slots.data(), count * 4ull, cudaMemcpyHostToDevice, s));
            k_sah_bins_init<<<grid_for(nslots * uint32_t(BINS_WORDS)), BLOCK, 0, s>>>(gbins.as<uint32_t>(), nslots);
            k_sah_bin_chunks<<<nchunks, BLOCK, 0, s>>>(chunks.as<SahChunk>(), cur, idx, lo0, hi0, gbins.as<uint32_t>());
        }
        const uint32_t* slot_ptr = large ? slots.as<uint32_t>() : nullptr;
        const uint32_t warps_grid = (count + SAH_WARPS - 1) / SAH_WARPS;
        k_sah_decide<<<warps_grid, SAH_WARPS * 32, smem, s>>>(cur, count, slot_ptr, gbins.as<uint32_t>(), idx, lo0, hi0,
                                                              level >= SAH_LEVEL_MAX ? 1u : 0u, splits.as<SahSplit>(),
                                                              internal.as<uint32_t>());
        BVH_TRY(cub::DeviceScan::ExclusiveSum(scan_tmp.p, scan_bytes, internal.as<uint32_t>(), offs.as<uint32_t>(),
                                              int(count), s));
        if (large) {
            k_sah_flags<<<nchunks, BLOCK, 0, s>>>(chunks.as<SahChunk>(), cur, splits.as<SahSplit>(), idx, lo0, hi0,
                                                  flags.as<uint32_t>());
            BVH_TRY(cub::DeviceScan::ExclusiveSum(rank_tmp.p, rank_bytes, flags.as<uint32_t>(), rank.as<uint32_t>(),
                                                  int(n), s));
            k_sah_scatter<<<nchunks, BLOCK, 0, s>>>(chunks.as<SahChunk>(), cur, splits.as<SahSplit>(), idx,
                                                    flags.as<uint32_t>(), rank.as<uint32_t>(), idx_next);
        }
        k_sah_partition<<<warps_grid, SAH_WARPS * 32, 0, s>>>(cur, count, slot_ptr, splits.as<SahSplit>(), idx, lo0,
                                                              hi0, idx_next);
        BVH_TRY(cudaMemsetAsync(maxc.p, 0, 4, s));
        const uint32_t next_base = base + count;
        k_sah_emit<<<grid_for(count), BLOCK, 0, s>>>(cur, count, splits.as<SahSplit>(), offs.as<uint32_t>(), next_base,
                                                     idx_next, lo0, hi0, t, nxt, maxc.as<uint32_t>());
        BVH_TRY(cudaGetLastError());
        uint32_t last[3];
        BVH_TRY(cudaMemcpyAsync(&last[0], offs.as<uint32_t>() + (count - 1), 4, cudaMemcpyDeviceToHost, s));
        BVH_TRY(cudaMemcpyAsync(&last[1], internal.as<uint32_t>() + (count - 1), 4, cudaMemcpyDeviceToHost, s));
        BVH_TRY(cudaMemcpyAsync(&last[2], maxc.p, 4, cudaMemcpyDeviceToHost, s));
        BVH_TRY(cudaStreamSynchronize(s));
        const uint32_t made = last[0] + last[1];
        if (next_base + made > 2 * n - 1 || made > max_tasks) return cudaErrorUnknown;
        // Positions outside this level's tasks are final (leaves), so only
        // the tasks' ranges need carrying from one order to the next.
        std::swap(idx, idx_next);
        std::swap(cur, nxt);
        base = next_base;
        count = made;
        largest = last[2];
    }
    order->assign(1, {0u, n});
    for (size_t k = levels.size(); k-- > 0;) order->push_back(levels[k]);
    return cudaSuccess;
}

}  // namespace

cudaError_t build_wide_bvh_gpu(const float4* in, uint32_t n, GpuBvh* out, cudaStream_t s, bool sah) {
    out->node_count = 0;
    out->depth = 0;
    out->nodes = nullptr;
    out->tris = nullptr;
    if (n == 0) return cudaSuccess;
    const size_t total = 2 * size_t(n) - 1;
    Scratch lo0, hi0, cb, tlo, thi, ttris;
    BVH_TRY(lo0.alloc(n * 16ull));
    BVH_TRY(hi0.alloc(n * 16ull));
    BVH_TRY(cb.alloc(48));
    const uint32_t cb_init[12] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u,
                                  0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    BVH_TRY(cudaMemcpyAsync(cb.p, cb_init, 48, cudaMemcpyHostToDevice, s));
    k_leaf_bounds<<<grid_for(n), BLOCK, 0, s>>>(in, n, lo0.as<float4>(), hi0.as<float4>(), cb.as<uint32_t>());
    BVH_TRY(tlo.alloc(total * 16));
    BVH_TRY(thi.alloc(total * 16));
    BVH_TRY(ttris.alloc(total * 4));
    Tree t{tlo.as<float4>(), thi.as<float4>(), ttris.as<uint32_t>()};
    uint32_t root = 0;
    std::vector<std::pair<uint32_t, uint32_t>> order;  // node ranges, children's before their parents'
    if (sah)
        BVH_TRY(binary_sah(n, lo0.as<float4>(), hi0.as<float4>(), cb.as<uint32_t>(), t, &root, &order, s));
    else
        BVH_TRY(binary_ploc(n, lo0.as<float4>(), hi0.as<float4>(), cb.as<uint32_t>(), t, &root, &order, s));

    // The collapse's costs, bottom-up over the builder's node ranges.
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
        for (const auto& r : order)
            if (r.second > r.first)
                k_collapse_cost<<<grid_for(r.second - r.first), BLOCK, 0, s>>>(t, cp, r.first, r.second, inv_root);
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
