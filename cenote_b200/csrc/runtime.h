// The library's runtime objects shared by the C ABI (capi.cpp) and the
// serving loop (server.cpp): the opaque handle types, device buffers, the
// status/error helpers, and the wave planner and enqueuer that drive the
// kernels of wavefront.cu.
#pragma once
#include <atomic>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/cenote_c.h"
#include "guide.h"
#include "records.h"
#include "wavefront.h"

namespace cn {

// Record `msg` as this thread's last error and return `code`.
int32_t fail(int32_t code, const std::string& msg);
// The calling thread's last error message (cenote_last_error).
const char* last_error();

#define CN_CUDA(call)                                                                       \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return ::cn::fail(e_ == cudaErrorMemoryAllocation ? CENOTE_E_ALLOCATION : CENOTE_E_DEVICE, \
                              std::string(#call ": ") + cudaGetErrorString(e_));            \
    } while (0)

#define CN_CHECK(cond, code, msg) \
    do {                          \
        if (!(cond)) return ::cn::fail((code), (msg)); \
    } while (0)

// Bounded wait: record `ev` on `s` and poll it until it completes or
// `timeout_ms` passes (CENOTE_E_TIMEOUT).
int32_t wait_stream(cudaStream_t s, cudaEvent_t ev, double timeout_ms);
int32_t wait_event(cudaEvent_t ev, double timeout_ms);

struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    cudaError_t alloc(size_t n) {
        release();
        if (n == 0) n = 16;
        bytes = n;
        return cudaMalloc(&ptr, n);
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(ptr);
    }
};

}  // namespace cn

using cn::DeviceBuffer;
using cn::DeviceScene;
using cn::LightRecord;
using cn::ShadowRay;
using cn::LaunchShape;
using cn::PathPool;
using cn::FilmTargets;
using cn::GuideRecordSink;
namespace guide = cn::guide;

struct cenote_context {
    // Handles made from this context hold a reference; the context is freed
    // when cenote_context_destroy has been called and the last one is gone,
    // so destroy order never leaves a dangling pointer.
    std::atomic<int> refs{1};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t sync_ev = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    LaunchShape shape{};
    cn::DeviceBuffer tables;
    std::mutex mu;
    // L2 persistence (this context's own set-aside; nothing outlives it).
    size_t l2_persist_max = 0, l2_window_max = 0, l2_set_aside = 0;
    uint32_t bvh_builder = CENOTE_BVH_AUTO;  // for scenes created from now on
};

struct cenote_scene {
    cenote_context* ctx = nullptr;
    DeviceScene ds{};
    std::vector<std::unique_ptr<DeviceBuffer>> buffers;
    cudaArray_t env_array = nullptr;
    cudaTextureObject_t env_tex = 0;
    cenote_camera camera{};
    std::vector<LightRecord> lights;
    uint32_t env_w = 1, env_h = 1;
    double env_power = 0.0;
    float select_prob = 0.0f;
    float prep_ms[3] = {0, 0, 0};
    uint32_t bvh_builder = CENOTE_BVH_HOST_SAH;  // the builder this scene's BVH came from
    uint64_t device_bytes = 0;
    DeviceBuffer* env_marginal = nullptr;
    DeviceBuffer* env_conditional = nullptr;
    DeviceBuffer* env_cut = nullptr;
    DeviceBuffer* env_pdfs = nullptr;
    std::vector<cudaArray_t> tex_arrays;            // the bindless table's storage
    std::vector<cudaTextureObject_t> tex_objects;

    // Take ownership of memory cudaMalloc'd elsewhere (the GPU BVH build).
    DeviceBuffer* adopt(void* p, size_t bytes) {
        buffers.push_back(std::make_unique<DeviceBuffer>());
        buffers.back()->ptr = p;
        buffers.back()->bytes = bytes;
        device_bytes += bytes;
        return buffers.back().get();
    }
        DeviceBuffer* add(size_t bytes, cudaError_t* err) {
        buffers.push_back(std::make_unique<DeviceBuffer>());
        *err = buffers.back()->alloc(bytes);
        device_bytes += bytes;
        return buffers.back().get();
    }
    ~cenote_scene() {
        for (cudaTextureObject_t t : tex_objects) cudaDestroyTextureObject(t);
        for (cudaArray_t a : tex_arrays) cudaFreeArray(a);
        if (env_tex) cudaDestroyTextureObject(env_tex);
        if (env_array) cudaFreeArray(env_array);
    }
};

struct cenote_renderer {
    cenote_context* ctx = nullptr;
    uint32_t max_bounces = 8;
    uint32_t light_sampling = 0;
    uint32_t capacity_req = 0;
    uint32_t samples_per_wave = 0;
    uint32_t profiling = 0;
    std::vector<cudaEvent_t> events;
    PathPool pool{};
    DeviceBuffer org, dir, thr, hit, ps, state, rad, q0, q1, shadows, counters, tally, scratch;
    // Material sort before shading: CENOTE_SORT_NONE, _ALL or _SECONDARY
    // (every bounce by default: 1.1x on the material chart, 1.6x on the
    // textured 2 M-triangle terrain, measured on a B200).
    uint32_t material_sort = 1;
    uint32_t refill_idle = 0;  // 0: the kernels' default
    uint32_t top_nodes = 0;    // BVH nodes staged in shared memory by the traversal kernels
    uint32_t l2_window = 0;    // mark the BVH nodes persisting in L2 during this renderer's waves
    uint32_t per_lane_triangles = 0;  // 1: no warp triangle queue in the traversal kernels
    uint32_t trav_variant = 0;        // traversal block size and stack depth (TRAV_VARIANT_*)
    uint32_t sort_by_location = 0;    // 1: the material sort keys layer-free hits by location
    float tuned_ms_per_sample = 0.0f;
    DeviceBuffer sort_order, sort_keys, sort_bins;
    DeviceBuffer aov_albedo, aov_normal, aov_depth, aov_guide;
    size_t pool_cap = 0, aov_cap = 0;
    // The learned guide (cenote_renderer_set_guide): per-path mixture outputs
    // and open records, the wave's training records and its sink.
    cenote_guide* guide = nullptr;
    float guide_fraction = 0.5f, guide_lr = 1e-2f;
    uint32_t guide_steps = 0;
    DeviceBuffer g_out, g_rec, g_records, g_count, g_sink;
    size_t g_cap = 0;
    static constexpr uint32_t GUIDE_RECORDS = 1u << 20;
    static constexpr uint32_t GUIDE_BATCH = 65536;
    cenote_stats stats{};
    unsigned long long tally_prev[6] = {0, 0, 0, 0, 0, 0};

    ~cenote_renderer() {
        for (cudaEvent_t e : events) cudaEventDestroy(e);
    }
    cudaEvent_t event(size_t i) {
        while (events.size() <= i) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
            events.push_back(e);
        }
        return events[i];
    }

    cudaError_t ensure(size_t cap) {
        if (cap <= pool_cap) return cudaSuccess;
        cudaError_t e;
        if ((e = org.alloc(cap * 16)) || (e = dir.alloc(cap * 16)) || (e = thr.alloc(cap * 16)) ||
            (e = hit.alloc(cap * 16)) || (e = ps.alloc(cap * 8)) || (e = state.alloc(cap * 4)) ||
            (e = rad.alloc(cap * 16)) || (e = q0.alloc(cap * 4)) || (e = q1.alloc(cap * 4)) ||
            (e = shadows.alloc(cap * sizeof(ShadowRay))) || (e = sort_order.alloc(cap * 4)) ||
            (e = sort_keys.alloc(cap * 4)) || (e = sort_bins.alloc(cn::SORT_BINS * 4)))
            return e;
        pool.org = org.as<float4>();
        pool.dir = dir.as<float4>();
        pool.thr = thr.as<float4>();
        pool.hit = hit.as<uint4>();
        pool.ps = ps.as<uint2>();
        pool.state = state.as<uint32_t>();
        pool.rad = rad.as<float4>();
        pool.queue[0] = q0.as<uint32_t>();
        pool.queue[1] = q1.as<uint32_t>();
        pool.shadows = shadows.as<ShadowRay>();
        // Null here: the wave loop passes a view with all three set to the
        // bounces it sorts.
        pool.order = nullptr;
        pool.sort_keys = nullptr;
        pool.sort_bins = nullptr;
        pool.capacity = uint32_t(cap);
        pool_cap = cap;
        return cudaSuccess;
    }

    // The learned guide's lanes, sized with the pool; detached without a guide.
    cudaError_t set_learned_guide(bool on) {
        if (on && g_cap < pool_cap) {
            cudaError_t e;
            if ((e = g_out.alloc(pool_cap * guide::OUT_ACT * 4)) || (e = g_rec.alloc(pool_cap * 4))) return e;
            g_cap = pool_cap;
        }
        if (on && !g_records.ptr) {
            cudaError_t e;
            if ((e = g_records.alloc(size_t(GUIDE_RECORDS) * sizeof(guide::Record))) || (e = g_count.alloc(16)) ||
                (e = g_sink.alloc(sizeof(GuideRecordSink))))
                return e;
        }
        pool.guide_out = on ? g_out.as<float>() : nullptr;
        pool.guide_rec = on ? g_rec.as<uint32_t>() : nullptr;
        pool.sink = on ? g_sink.as<GuideRecordSink>() : nullptr;
        return cudaSuccess;
    }

    // The guide lanes: allocated on the first wave that traces guides,
    // detached (null) for waves that do not.
    // The pool as the bounces that sort see it.
    PathPool sorted_view() const {
        PathPool p = pool;
        p.order = sort_order.as<uint32_t>();
        p.sort_keys = sort_keys.as<uint32_t>();
        p.sort_bins = sort_bins.as<uint32_t>();
        return p;
    }

        cudaError_t set_guides(bool on) {
        if (on && aov_cap < pool_cap) {
            cudaError_t e;
            if ((e = aov_albedo.alloc(pool_cap * 16)) || (e = aov_normal.alloc(pool_cap * 16)) ||
                (e = aov_depth.alloc(pool_cap * 4)) || (e = aov_guide.alloc(pool_cap * 16)))
                return e;
            aov_cap = pool_cap;
        }
        pool.aov_albedo = on ? aov_albedo.as<float4>() : nullptr;
        pool.aov_normal = on ? aov_normal.as<float4>() : nullptr;
        pool.aov_depth = on ? aov_depth.as<float>() : nullptr;
        pool.aov_guide = on ? aov_guide.as<float4>() : nullptr;
        return cudaSuccess;
    }
};

struct cenote_guide {
    cenote_context* ctx = nullptr;
    DeviceBuffer params, grad, m, v, w1, w2, w3, w4, b4, err, loss;
    DeviceBuffer feats, out, save, dz4, dirs, weights;
    size_t cap = 0;
    uint32_t step = 0;
    int sms = 148;

    guide::Buffers view() {
        return {params.as<float>(), grad.as<float>(), m.as<float>(), v.as<float>(), w1.as<__nv_bfloat16>(),
                w2.as<__nv_bfloat16>(), w3.as<__nv_bfloat16>(), w4.as<__nv_bfloat16>(), b4.as<float>(),
                err.as<int>()};
    }
    guide::TrainScratch scratch(uint32_t rows) {
        return {out.as<float>(), save.as<__nv_bfloat16>(), dz4.as<__nv_bfloat16>(), loss.as<float>(), rows};
    }
    cudaError_t ensure(size_t n) {
        if (n <= cap) return cudaSuccess;
        cudaError_t e;
        if ((e = feats.alloc(n * guide::IN * 4)) || (e = out.alloc(n * guide::OUT * 4)) ||
            (e = save.alloc(n * guide::ACT * 2)) || (e = dz4.alloc(n * guide::OUT_PAD * 2)) ||
            (e = dirs.alloc(n * 12)) || (e = weights.alloc(n * 4)))
            return e;
        cap = n;
        return cudaSuccess;
    }
};

struct cenote_film {
    cenote_context* ctx = nullptr;
    uint32_t width = 0, height = 0;
    uint32_t samples = 0;
    DeviceBuffer sum, avg;
    DeviceBuffer albedo, normal, depth;  // guide sums (film.rs:95-112)
    FilmTargets targets() {
        return {sum.as<float4>(), albedo.as<float4>(), normal.as<float4>(), depth.as<float>()};
    }
};

namespace cn {
inline void free_context(cenote_context* ctx) {
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->tables.release();
    if (ctx->sync_ev) cudaEventDestroy(ctx->sync_ev);
    if (ctx->t0) cudaEventDestroy(ctx->t0);
    if (ctx->t1) cudaEventDestroy(ctx->t1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}
inline void retain(cenote_context* ctx) { ctx->refs.fetch_add(1); }
inline void release(cenote_context* ctx) {
    if (ctx->refs.fetch_sub(1) == 1) free_context(ctx);
}
}  // namespace cn


namespace cn {

// How a call splits into waves: `range` pixels per wave, `spw` samples each.
struct WavePlan {
    uint32_t range, spw;
    uint64_t need;  // paths the pool must hold
};

struct WaveCounts {
    uint32_t launches = 0, waves = 0;
    size_t events = 0;
};

WavePlan plan_waves(const cenote_renderer* r, uint64_t pixels, uint32_t count, bool oneshot);

// Enqueue `count` samples from `sample0` for every pixel on `stream`, with no
// host synchronisation (so a stream capture can record it): each wave's
// samples go into the film in ascending order or, for a one-shot render,
// into `oneshot` as raw RGBA. The pool must already hold `plan.need` paths
// and the guide lanes must match `film`. `sample_offset` (device, may be
// null) is added to every sample index. Timing marks are recorded only when
// `timing` is set (never inside a capture).
cudaError_t enqueue_waves(cenote_renderer* r, const cenote_scene* sc, uint32_t width, uint32_t height,
                          uint32_t sample0, uint32_t count, uint32_t max_bounces, const WavePlan& plan,
                          const FilmTargets* film, bool film_reset, float4* oneshot, const uint32_t* sample_offset,
                          cudaStream_t stream, bool timing, bool counting, WaveCounts* wc);

// The bounces of one wave whose n0 camera paths are in the pool.
void enqueue_bounces(cenote_renderer* r, const cenote_scene* sc, const WaveParams& wp, uint32_t n0, bool guided,
                     cudaStream_t stream, bool timing, bool counting, WaveCounts* wc);

// One multi-job wave (the serving loop): segments in device memory, their
// camera paths, the bounces, and each segment's samples into its job's film.
cudaError_t enqueue_segments(cenote_renderer* r, const cenote_scene* sc, const WaveSegment* segs, uint32_t nseg,
                             uint32_t paths, uint32_t items, const uint32_t* hdr, uint32_t max_bounces,
                             cudaStream_t stream, WaveCounts* wc);

}  // namespace cn
