// Byte layouts shared by the host library and the sm_100a kernels.
//
// Material (144 B) and LightRecord (80 B) keep the reference's records field
// for field (crates/cenote/src/material.rs:28-116, crates/cenote/src/lights.rs:79-115)
// because the C ABI hands them across unchanged. Everything else is this
// library's own B200 layout: the scene is flattened into one world-space
// triangle set under one compressed 8-wide BVH (HBM is plentiful, and a
// single level spares every ray the per-instance transforms of a two-level
// walk), path state is SoA with 16-byte fields, and queues are index arrays.
#pragma once
#include <cstdint>
#include "../../include/cenote_c.h"

#include <cuda_runtime.h>

namespace cn {

// Buckets of the environment CDFs' cutpoint tables (a power of two, so u·ENV_CUTS is exact).
#ifndef CN_ENV_CUTS
#define CN_ENV_CUTS 256
#endif
constexpr uint32_t ENV_CUTS = CN_ENV_CUTS;

using Material = cenote_material;
static_assert(sizeof(Material) == 144, "material record is 144 bytes");

constexpr uint32_t LIGHT_NONE = 0xffffffffu;
constexpr uint32_t MEDIUM_NONE = 0xffffffu;  // pathstate.slang:188
constexpr uint32_t TEXTURE_NONE = 0xffffffffu;
constexpr uint32_t KIND_TRIANGLE = 0, KIND_DISTANT = 1, KIND_POINT = 2;
constexpr uint32_t RAY_MASK_CAMERA = 0x01u, RAY_MASK_ALL = 0xffu;
constexpr uint32_t TRANSPARENT_CAP = 8;   // intersect.slang:199
constexpr uint32_t ROULETTE_START = 3;    // shade_surface.slang:53

struct LightRecord {
    float anchor[3];
    float pdf;
    float edge1[3];
    float alias_threshold;
    float edge2[3];
    uint32_t alias_index;
    float emission[3];
    uint32_t instance;
    uint32_t kind;
    uint32_t primitive;
    uint32_t pad0[2];
};
static_assert(sizeof(LightRecord) == 80, "light record is 80 bytes");

// Everything shading needs to re-evaluate a hit on one instance: its
// object-space attributes, both transforms, and its first light record.
struct GeomRecord {
    const float* positions;
    const float* normals;
    const float* uvs;
    const uint32_t* indices;
    float o2w[3][4];
    float w2o[3][4];
    uint32_t light;
    uint32_t pad[3];
};

// Compressed wide BVH node (Ylitie, Karras & Laine, HPG 2017): 80 bytes =
// five 16-byte vector loads. Child boxes are 8-bit offsets from `p` in units
// of 2^(e-127) per axis. meta[i]: 0 = empty slot; inner child = 0b001 << 5 |
// (24 + i); leaf = unary triangle count (0b001/0b011/0b111) << 5 | offset of
// its first triangle from base_tri. Inner children are stored contiguously
// from base_child in slot order; imask bit i marks slot i as inner.
struct alignas(16) WideNode {
    float p[3];
    uint8_t e[3];
    uint8_t imask;
    uint32_t base_child;
    uint32_t base_tri;
    uint8_t meta[8];
    uint8_t qlo_x[8], qlo_y[8], qlo_z[8];
    uint8_t qhi_x[8], qhi_y[8], qhi_z[8];
};
static_assert(sizeof(WideNode) == 80, "wide node is 80 bytes");

// One leaf-ordered triangle: three float4 with the identity folded into the
// w lanes — v0.w = instance, v1.w = primitive, v2.w = flags (bits 0-7 ray
// mask, bit 8 opaque) — so a hit needs no second fetch.
constexpr uint32_t TRI_OPAQUE = 0x100u;

// Entries of a walk's traversal stack (node groups and postponed triangle
// groups). Scene creation rejects a wide BVH whose node groups alone could
// fill it.
constexpr int TRAVERSAL_STACK_DEPTH = 32;

// What every kernel reads about the scene; passed by value (kernel params
// live in the constant bank, uniform across the grid).
struct DeviceScene {
    const WideNode* nodes;
    const float4* tris;        // 3 per triangle, leaf order
    const GeomRecord* geometry;
    const Material* materials;
    const LightRecord* lights;
    const float* bsdf_tables;
    const float* env_marginal;
    const float* env_conditional;
    // Cutpoints of the CDFs (marginal first, then each row's conditional):
    // ENV_CUTS + 1 per CDF, entry b the index its search returns for b / ENV_CUTS.
    const uint32_t* env_cut;
    const float* env_pdfs;
    unsigned long long env_tex;  // cudaTextureObject_t
    uint32_t env_w, env_h;
    float select_prob;
    uint32_t light_count;
    uint32_t node_count, tri_count;
    uint32_t has_nonopaque;
    uint32_t has_layers;  // a material with coat, fuzz, transmission or thin walls

    const uint32_t* light_leaf;  // per light record: its triangle's leaf index, ~0 for delta lights
    const uint8_t* instance_layers;  // per instance: 1 if its material has coat, fuzz, transmission or thin walls
    const unsigned long long* textures;  // cudaTextureObject_t per bindless slot
    uint32_t texture_count;
    // TRAVERSAL_STACK_DEPTH minus the wide tree's depth: a walk postpones a
    // triangle group onto the stack only below this height, so the node
    // groups (one per level) that may follow always fit.
    uint32_t stack_room;
    float bbox_min[3];    // world bounds of every triangle, for the guide's position encoding
    float bbox_inv;       // 1 / the bounds' largest extent
    // Set inside a traversal kernel (0 elsewhere): nodes 0..top_count-1 (the
    // BVH's top levels: the builder lays nodes out breadth first) are staged
    // in the block's shared memory at shared-window address top_smem.
    uint32_t top_count;
    uint32_t top_smem;
};

// One queued shadow ray: 64 bytes, four 16-byte lanes.
struct alignas(16) ShadowRay {
    float org[3];
    float tmax;
    float dir[3];
    uint32_t path;
    float contrib[3];
    uint32_t light;
    uint32_t primitive;
    uint32_t leaf;     // the target triangle's leaf index, ~0 when unknown or none
    uint32_t pad[2];
};

}  // namespace cn
