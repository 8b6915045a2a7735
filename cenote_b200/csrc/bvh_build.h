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
};

// SAH binary build (32 bins per axis above 65,536 triangles, an exact sweep
// over sorted centroids below; single-triangle leaves), then a
// cost-optimal collapse (a dynamic programme over the binary tree) into
// 8-wide nodes with up to three triangles per leaf child, octant-ordered
// child slots and 8-bit quantised boxes.
// `threads` > 1 builds independent subtrees in parallel.
WideBvh build_wide_bvh(const std::vector<BuildTri>& tris, unsigned threads);

}  // namespace cn
