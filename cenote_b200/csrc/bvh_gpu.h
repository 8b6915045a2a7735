// GPU construction of the compressed 8-wide BVH (bvh_gpu.cu): a binned SAH or
// PLOC binary build, collapsed on the device into the node format the
// traversal kernels walk.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "records.h"

namespace cn {

struct GpuBvh {
    void* nodes;          // WideNode[node_count] (cudaMalloc'd; the caller frees)
    void* tris;           // float4[3 * triangles], leaf order (cudaMalloc'd; the caller frees)
    uint32_t node_count;
    uint32_t depth;       // wide levels
};

// `in`: n triangles as three float4 each (corners, identity in the w lanes:
// instance, primitive, flags), device memory. `sah`: the binned SAH binary
// tree (32 bins per axis at every level), else PLOC. Synchronises `s`.
cudaError_t build_wide_bvh_gpu(const float4* in, uint32_t n, GpuBvh* out, cudaStream_t s, bool sah);

// Each emissive triangle's leaf index: light_leaf[geometry[inst].light + prim] = leaf.
void launch_light_leaves(const float4* tris, uint32_t n, const GeomRecord* geometry, uint32_t* light_leaf,
                         cudaStream_t s);

}  // namespace cn
