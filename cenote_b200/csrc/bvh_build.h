// Host construction of the compressed 8-wide BVH the traversal kernels walk.
#pragma once
#include <cstdint>
#include <vector>
#include "records.h"

namespace cn {

struct BuildTri {
    float v[3][3];       // world-space corners
    uint32_t instance;
    uint32_t primitive;
    uint32_t flags;      // ray-mask bits | TRI_OPAQUE
};

struct WideBvh {
    std::vector<WideNode> nodes;
    std::vector<float> tris;  // 12 floats per triangle (three float4), leaf order
    uint32_t depth = 0;
    uint32_t stack_need = 0;  // node groups a walk may hold on its stack at once
};

// SAH binary build (32 bins per axis above 65,536 triangles, an exact sweep
// over sorted centroids below; object-median splits past 48 levels, so the
// tree stays at most 48 + log2(n) levels deep; single-triangle leaves), then
// a cost-optimal collapse (a dynamic programme over the binary tree) into
// 8-wide nodes with up to three triangles per leaf child, octant-ordered
// child slots and 8-bit quantised boxes. `depth` is the wide tree's;
// `stack_need` bounds the node groups its walks push.
// Parallelism is fixed, not set by `threads` (kept for the ABI): the two
// subtrees of a range above 65,536 triangles in the top four levels build
// on separate threads (std::async), at most 16 at once.
WideBvh build_wide_bvh(const std::vector<BuildTri>& tris, unsigned threads);

}  // namespace cn
