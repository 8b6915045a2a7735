// Host harness: build the compressed wide BVH with the library's own builder,
// check its structure, and trace rays with the device traversal code
// (traverse.cuh through cuda_host_shim.h).
//
//   traverse_host <tris.bin> <rays.bin> <hits.bin>
// tris.bin: uint32 n, then n × (9 float corners, uint32 instance, primitive, flags)
// rays.bin: uint32 m, then m × (3 float origin, 3 float direction)
// hits.bin: m × (uint32 instance, primitive, b1 bits, b2 bits, float t)
// Exit status 0 = structure valid and every ray traced within bounds; stdout
// reports the tree's size and the wide nodes and triangles tested per ray.
#include "cuda_host_shim.h"
#include "traverse.cuh"
#include "bvh_build.h"

#include <cstdio>
#include <vector>

using namespace cn;

static int fail(const char* what, long a = 0, long b = 0) {
    std::fprintf(stderr, "structure check failed: %s (%ld, %ld)\n", what, a, b);
    return 2;
}

int main(int argc, char** argv) {
    if (argc != 4) return 1;
    FILE* f = std::fopen(argv[1], "rb");
    uint32_t n = 0;
    if (std::fread(&n, 4, 1, f) != 1) return 1;
    std::vector<BuildTri> tris(n);
    for (auto& t : tris) {
        float v[9];
        uint32_t ids[3];
        if (std::fread(v, 4, 9, f) != 9 || std::fread(ids, 4, 3, f) != 3) return 1;
        std::memcpy(t.v, v, sizeof v);
        t.instance = ids[0];
        t.primitive = ids[1];
        t.flags = ids[2];
    }
    std::fclose(f);
    WideBvh bvh = build_wide_bvh(tris, 4);
    const uint32_t nn = uint32_t(bvh.nodes.size()), nt = uint32_t(bvh.tris.size() / 12);
    if (nt != n) return fail("triangle count", nt, n);
    // Structure: every child index in range, every triangle referenced once,
    // every decoded child box contains its subtree.
    std::vector<int> seen(nt, 0), node_seen(nn, 0);
    for (uint32_t i = 0; i < nn; ++i) {
        const WideNode& w = bvh.nodes[i];
        uint32_t inner = 0;
        for (int s = 0; s < 8; ++s) {
            uint8_t m = w.meta[s];
            if (!m) continue;
            bool is_inner = (m & 0x18) == 0x18;
            if (is_inner != bool((w.imask >> s) & 1)) return fail("imask/meta disagree", i, s);
            if (is_inner) {
                if ((m & 0x1f) != 24 + s || (m >> 5) != 1) return fail("inner meta", i, m);
                uint32_t ci = w.base_child + inner++;
                if (ci >= nn) return fail("child index", i, ci);
                node_seen[ci]++;
            } else {
                uint32_t cnt = __builtin_popcount(m >> 5), off = m & 0x1f;
                if (cnt < 1 || cnt > 3 || ((m >> 5) != (1u << cnt) - 1)) return fail("leaf count", i, m);
                for (uint32_t k = 0; k < cnt; ++k) {
                    uint32_t ti = w.base_tri + off + k;
                    if (ti >= nt) return fail("triangle index", i, ti);
                    seen[ti]++;
                }
            }
        }
    }
    for (uint32_t t = 0; t < nt; ++t)
        if (seen[t] != 1) return fail("triangle referenced != once", t, seen[t]);
    for (uint32_t i = 1; i < nn; ++i)
        if (node_seen[i] != 1) return fail("node referenced != once", i, node_seen[i]);

    f = std::fopen(argv[2], "rb");
    uint32_t m = 0;
    if (std::fread(&m, 4, 1, f) != 1) return 1;
    std::vector<float> rays(size_t(m) * 6);
    if (std::fread(rays.data(), 4, rays.size(), f) != rays.size()) return 1;
    std::fclose(f);
    DeviceScene s{};
    s.nodes = bvh.nodes.data();
    s.tris = reinterpret_cast<const float4*>(bvh.tris.data());
    s.node_count = nn;
    s.tri_count = nt;
    if (bvh.stack_need >= uint32_t(TRAVERSAL_STACK_DEPTH)) return fail("stack need", bvh.stack_need, bvh.depth);
    s.stack_room = uint32_t(TRAVERSAL_STACK_DEPTH) - bvh.stack_need;
    FILE* o = std::fopen(argv[3], "wb");
    int bad = 0;
    uint32_t visits = 0, tests = 0;  // wide nodes expanded, triangles tested
    for (uint32_t i = 0; i < m; ++i) {
        Ray ray = make_ray(make_float3(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]),
                           make_float3(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]));
        float tmax = 1e30f;
        uint32_t bi = LIGHT_NONE, bp = 0, b1s = 0, b2s = 0;
        bool ok = traverse<true>(s, ray, tmax, [&](uint32_t, float4 a, float4 b, float4 c, float& tm) {
            float t, b1, b2;
            if (!tri_hit(ray, a, b, c, tm, t, b1, b2)) return false;
            uint32_t inst = __float_as_uint(a.w), prim = __float_as_uint(b.w);
            if (!(t < tm || (t == tm && (inst < bi || (inst == bi && prim < bp))))) return false;
            tm = t;
            bi = inst;
            bp = prim;
            b1s = __float_as_uint(b1);
            b2s = __float_as_uint(b2);
            return false;
        }, &visits, &tests);
        if (!ok) bad++;
        float tt = bi == LIGHT_NONE ? -1.0f : tmax;
        uint32_t rec[5] = {bi, bp, b1s, b2s, __float_as_uint(tt)};
        std::fwrite(rec, 4, 5, o);
    }
    std::fclose(o);
    std::fprintf(stdout, "nodes %u tris %u depth %u stack %u bad %d visits/ray %.4f tests/ray %.4f\n", nn, nt,
                 bvh.depth, bvh.stack_need, bad,
                 m ? double(visits) / m : 0.0, m ? double(tests) / m : 0.0);
    return bad ? 3 : 0;
}
