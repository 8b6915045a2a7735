// Host-side view of the wavefront engine: path pool layout and the launch
// entry points of wavefront.cu.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "records.h"

namespace cn {

// Per-wave device counters, one uint32 each, zeroed at wave start.
constexpr uint32_t MAX_BOUNCES = 255;
constexpr uint32_t CTR_RAYS = 0;        // [b]: paths entering bounce b (b = 0 is the camera wave)
constexpr uint32_t CTR_SHADOWS = 256;   // [b]: shadow rays pushed at bounce b
constexpr uint32_t CTR_FETCH_ISECT = 512;
constexpr uint32_t CTR_FETCH_SHADE = 768;
constexpr uint32_t CTR_FETCH_SHADOW = 1024;
constexpr uint32_t CTR_OVERFLOW = 1280;
constexpr uint32_t CTR_VISITS = 1284;   // 64-bit: wide nodes visited (instrumented launches only)
constexpr uint32_t CTR_TESTS = 1286;    // 64-bit: triangles tested (instrumented launches only)
constexpr uint32_t CTR_HITS = 1288;     // 64-bit: closest hits on a surface (instrumented waves only)
constexpr uint32_t CTR_FETCH_SHADE_LAYERS = 1296;  // [b]: the layered part of a split shading launch
constexpr uint32_t CTR_COUNT = 1552;

// Structure-of-arrays path state: one 16-byte lane per logical field, so
// every stage reads and writes with coalesced 128-bit accesses.
struct PathPool {
    float4* org;       // xyz origin
    float4* dir;       // xyz direction, w = cosine to the camera's forward axis
    float4* thr;       // xyz throughput, w = pdf of the scatter that made the ray (0: camera ray)
    uint4* hit;        // (instance | 0xffffffff on a miss, primitive, b1 bits, b2 bits)
    uint2* ps;         // (pixel, sample index)
    uint32_t* state;   // lobe << 24 | medium
    float4* rad;       // the path's radiance, alpha = finished
    // Denoiser guides (pathstate.slang:82-106), all null on a wave that
    // traces none. Path-owned accumulators zeroed by raygen: albedo and
    // normal (xyz, w = 0) and camera-plane depth of the first hit (+inf on
    // a miss); `aov_guide` is the feature throughput still open, written by
    // scatters and read from bounce 1 on (a camera ray's is 1).
    float4* aov_albedo;
    float4* aov_normal;
    float* aov_depth;
    float4* aov_guide;
    // The learned guide (all null without one): 40 raw mixture outputs per
    // path for the current bounce, the path's open training record (~0u: none),
    // and the wave's record buffer with its counter.
    float* guide_out;
    uint32_t* guide_rec;
    struct GuideRecordSink* sink;
    // Material sort (null when off): the shading order of the bounce's paths,
    // each queue entry's key, and SORT_BINS key counts turned into offsets.
    uint32_t* order;
    uint32_t* sort_keys;
    uint32_t* sort_bins;
    uint32_t* queue[2];   // ray queues, ping-pong by bounce parity
    ShadowRay* shadows;
    uint32_t* counters;
    uint32_t capacity;
    // Idle lanes before a traversal warp refills with new rays (1..32; 0 =
    // the built-in default): a per-scene tuning knob.
    uint32_t refill_idle;
    // BVH nodes each traversal block stages in shared memory (0..TOP_NODES_MAX).
    uint32_t top_nodes;
    // 1: traversal lanes test their own triangles even in an all-opaque scene
    // (0: the warp triangle queue, trqueue.cuh).
    uint32_t per_lane_triangles;
    // The traversal launch variant (block size, stack entries; TRAV_VARIANT_*).
    uint32_t trav_variant;
    uint32_t sort_location;  // 1: layer-free hits sort by their location's Morton cell, not by instance
};

constexpr uint32_t TOP_NODES_MAX = 320;  // 25.6 KB per 128-thread block: 8 blocks still fit an SM

// Where guided vertices record themselves for training.
struct GuideRecordSink {
    void* records;        // guide::Record[capacity]
    uint32_t* count;
    uint32_t capacity;
    float rate;           // probability that a guided vertex records
    float fraction;       // the guide's share of the one-sample MIS
    uint32_t pad;
};

struct WaveParams {
    uint32_t width, height;
    uint32_t pixel_base, pixel_count;  // the pixel range of this wave
    uint32_t samples;                  // samples of each pixel traced in this wave
    uint32_t sample_base;              // sample index of the first
    uint32_t max_bounces;
    uint32_t light_sampling;
    float3 cam_pos, cam_right, cam_up, cam_fwd;  // basis pre-scaled to the focal plane when the lens is open
    float aperture;
    // When set, added to every sample index: a replayed CUDA graph reads its
    // progress from device memory instead of baked launch parameters.
    const uint32_t* sample_offset;
    // Non-zero (the image width, a multiple of 8, with the height a multiple
    // of 4 and the wave covering the whole image): camera paths take their
    // pixels in 8 x 4 tiles, 32 consecutive paths to a tile (wave_pixel).
    uint32_t tile_width;
};

// The pixel of a wave's local path index j (within one sample): j itself,
// or with tiling the row-major order of 8 x 4 tiles of a tile_width-wide
// image, each tile's 32 pixels row-major inside it, so a warp's camera rays
// leave a square of the image instead of a 32-pixel strip.
__host__ __device__ inline uint32_t wave_pixel(uint32_t j, uint32_t tile_width) {
    if (tile_width == 0u) return j;
    const uint32_t t = j >> 5, k = j & 31u, tiles_x = tile_width >> 3;
    return ((t / tiles_x) * 4u + (k >> 3)) * tile_width + (t % tiles_x) * 8u + (k & 7u);
}

// One job's share of a multi-job wave (the serving loop): samples
// sample_base .. sample_base + samples - 1 of pixels pixel_base ..
// pixel_base + pixel_count - 1 of a width x height image, traced as the
// wave's paths start .. start + samples * pixel_count - 1 (sample-major) and
// added into `film` as accumulate items pixel_start .. pixel_start +
// pixel_count - 1. Segments are ordered by start (and pixel_start).
struct WaveSegment {
    uint32_t start, pixel_start;
    uint32_t width, height;
    uint32_t pixel_base, pixel_count;
    uint32_t samples, sample_base;
    float3 cam_pos, cam_right, cam_up, cam_fwd;  // basis pre-scaled to the focal plane when the lens is open
    float aperture;
    uint32_t reset;  // the segment's first sample starts the film (the job's first samples)
    float4* film;    // the job's beauty sums
};

// Keys of the material sort: 0 for a miss; a hit's instance (its material
// slot) folded into 1 .. SORT_LAYERS - 1 when its material has no coat,
// fuzz, transmission or thin walls, else into SORT_LAYERS .. SORT_BINS - 1,
// so a sorted bounce shades its layer-free paths and its layered ones as two
// ranges.
constexpr uint32_t SORT_BINS = 2048;
constexpr uint32_t SORT_LAYERS = 1024;

// Traversal launch variants (PathPool::trav_variant): 0 = 128 threads per
// block and 32 stack entries per lane (the default), 1 = 128 / 16,
// 2 = 256 / 32, 3 = 256 / 16.
constexpr uint32_t TRAV_VARIANTS = 4;
constexpr int TRAV_VARIANT_BLOCK[TRAV_VARIANTS] = {128, 128, 256, 256};
constexpr int TRAV_VARIANT_STACK[TRAV_VARIANTS] = {32, 16, 32, 16};
enum : int { TRAV_ISECT, TRAV_ISECT_QUEUED, TRAV_ISECT_QUEUED_TOP, TRAV_SHADOW, TRAV_SHADOW_QUEUED,
             TRAV_SHADOW_QUEUED_TOP, TRAV_KINDS };

struct LaunchShape {
    int grid_isect, grid_isect_queued, grid_isect_queued_top, grid_shade, grid_shade_free, grid_shadow, grid_shadow_queued,
        grid_shadow_queued_top, grid_stream;
    int block;
    int trav[TRAV_VARIANTS][TRAV_KINDS];  // persistent grids of each traversal variant
};

LaunchShape launch_shape(int device);

// One wave: raygen, then max_bounces × (intersect, shade, shadow). Path
// radiance lands in pool.rad[path] with path = s · pixel_count + local pixel.
// The stages are also exposed one by one so a caller can time them.
void launch_wave(const DeviceScene& scene, const PathPool& pool, const WaveParams& wp, const LaunchShape& ls,
                 cudaStream_t stream);
void launch_wave_begin(const PathPool& pool, const WaveParams& wp, const LaunchShape& ls, cudaStream_t stream);
// `count_visits` selects the instrumented traversal that tallies wide-node
// visits and triangle tests into the counters (for the roofline's traffic).
void launch_intersect(const DeviceScene& scene, const PathPool& pool, uint32_t bounce, uint32_t n0,
                      const LaunchShape& ls, bool count_visits, cudaStream_t stream);
void launch_shade(const DeviceScene& scene, const PathPool& pool, uint32_t bounce, const WaveParams& wp, uint32_t n0,
                  const LaunchShape& ls, cudaStream_t stream);
void launch_shadow(const DeviceScene& scene, const PathPool& pool, uint32_t bounce, const LaunchShape& ls,
                   bool count_visits, cudaStream_t stream);

// The film's running sums. The guide sums may be null (no guides traced).
struct FilmTargets {
    float4* sum;
    float4* albedo;
    float4* normal;
    float* depth;
};

// Film: sum[pixel] += guarded rad[s · count + local], s ascending (the
// film's guard, crates/cenote/shaders/accumulate.slang:38-67: a non-finite
// channel drops that buffer's sample, depth drops only NaN); reset
// overwrites with the first sample instead. The guides accumulate when both
// the pool and the film carry them.
// With tile_width set (a tiled whole-image wave) local index p is pixel
// wave_pixel(p, tile_width).
void launch_accumulate(const PathPool& pool, const FilmTargets& film, uint32_t pixel_base, uint32_t pixel_count,
                       uint32_t tile_width, uint32_t samples, bool reset, cudaStream_t stream);
void launch_resolve(const float4* sum, float4* avg, uint32_t pixels, float samples, cudaStream_t stream);
void launch_resolve1(const float* sum, float* avg, uint32_t pixels, float samples, cudaStream_t stream);
// The display transform (tonemap.slang): linear ACEScg averages -> sRGB RGBA8.
// Counting sort of bounce `bounce`'s queue by material key into pool.order.
// launch_sort_begin clears the key counts before the bounce's intersect,
// which (given a pool view with sort_keys set) writes and counts every ray's
// key; launch_material_sort then turns the counts into offsets and scatters
// the paths; the shading kernel reads them in that order.
void launch_sort_begin(const PathPool& pool, cudaStream_t stream);
void launch_material_sort(const PathPool& pool, uint32_t bounce, uint32_t n0, const LaunchShape& ls,
                          cudaStream_t stream);
void launch_tonemap(const float4* avg, uint32_t* out, uint32_t pixels, float exposure_scale, cudaStream_t stream);
// tally[0] += extension rays, [1] += shadow rays, [2] |= overflow,
// [3] += node visits, [4] += triangle tests, [5] += surface hits.
void launch_tally(const PathPool& pool, unsigned long long* tally, uint32_t n0, uint32_t max_bounces,
                  cudaStream_t stream);
// Instrumented waves: count bounce `bounce`'s rays that hit a surface into
// CTR_HITS (misses are shaded by the same kernel but read no records).
void launch_count_hits(const PathPool& pool, uint32_t bounce, uint32_t n0, cudaStream_t stream);
// A multi-job wave: counters cleared and the camera paths of every segment
// (`segs` in device memory), then, after the bounces, each segment's
// samples added into its job's film. With `hdr` (device memory: segments,
// paths, accumulate items) the counts are read on the device and the
// bounce launches take n0 = 0, so one captured graph serves every wave.
void launch_wave_begin_segments(const PathPool& pool, const WaveSegment* segs, uint32_t nseg, uint32_t paths,
                                const uint32_t* hdr, const LaunchShape& ls, cudaStream_t stream);
void launch_accumulate_segments(const PathPool& pool, const WaveSegment* segs, uint32_t nseg, uint32_t items,
                                const uint32_t* hdr, cudaStream_t stream);
void launch_copy_rad(const PathPool& pool, float4* out, uint32_t pixel_base, uint32_t pixel_count, uint32_t tile_width,
                     cudaStream_t stream);
// *counter += n on the device (a graph's progress counter).
void launch_advance(uint32_t* counter, uint32_t n, cudaStream_t stream);

}  // namespace cn
