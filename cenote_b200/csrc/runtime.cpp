// Runtime helpers shared by the C ABI and the serving loop: errors, bounded
// waits, and the wave planner/enqueuer over the kernels of wavefront.cu.
#include <algorithm>
#include <chrono>
#include <thread>

#include "runtime.h"

// 1: a wave that covers a whole image whose sides are multiples of 8 and 4
// hands its camera paths out in 8 x 4 pixel tiles (WaveParams::tile_width);
// 0: row-major pixels. Films are the same either way (a path's samples are
// keyed by its pixel and sample, not by its slot).
#ifndef CN_TILE_PIXELS
#define CN_TILE_PIXELS 1
#endif

namespace cn {

void camera_basis(const cenote_camera& cam, float aspect, WaveParams& wp);

namespace {

thread_local std::string g_error;

}  // namespace

const char* last_error() { return g_error.c_str(); }


int32_t fail(int32_t code, const std::string& msg) {
    g_error = msg;
    return code;
}

// Bounded wait: record an event on `s` and poll it until it completes or
// `timeout_ms` passes.
int32_t wait_stream(cudaStream_t s, cudaEvent_t ev, double timeout_ms) {
    cudaError_t e = cudaEventRecord(ev, s);
    if (e != cudaSuccess) return fail(CENOTE_E_DEVICE, std::string("cudaEventRecord: ") + cudaGetErrorString(e));
    return wait_event(ev, timeout_ms);
}

// Bounded wait on an event already recorded.
int32_t wait_event(cudaEvent_t ev, double timeout_ms) {
    cudaError_t e;
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        e = cudaEventQuery(ev);
        if (e == cudaSuccess) return CENOTE_OK;
        if (e != cudaErrorNotReady) return fail(CENOTE_E_DEVICE, std::string("device error: ") + cudaGetErrorString(e));
        double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (ms > timeout_ms) return fail(CENOTE_E_TIMEOUT, "device work did not finish within the wait bound");
        std::this_thread::sleep_for(std::chrono::microseconds(ms < 5.0 ? 20 : 200));
    }
}

// How a call splits into waves: `range` pixels per wave, `spw` samples each.
WavePlan plan_waves(const cenote_renderer* r, uint64_t pixels, uint32_t count, bool oneshot) {
    WavePlan p{uint32_t(pixels), 1, 0};
    if (r->capacity_req && r->capacity_req < pixels) {
        p.range = r->capacity_req;
        p.spw = 1;
    } else if (r->samples_per_wave) {
        p.spw = r->samples_per_wave;
    } else {
        // Enough paths per wave to keep 148 SMs busy through the tail bounces
        // and amortise each bounce's launches (16 M paths, ~4 GB of path
        // state; on the chart 4 M-path waves left intersect 20 % slower).
        uint64_t want = (uint64_t(1) << 24) / pixels;
        p.spw = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(want, 64)));
    }
    if (oneshot) p.spw = 1;
    p.spw = std::max(1u, std::min(p.spw, count));
    p.need = uint64_t(p.range) * p.spw;
    if (r->capacity_req) p.need = std::max<uint64_t>(p.need, std::min<uint64_t>(r->capacity_req, p.need));
    return p;
}

// The bounces of one wave of n0 camera paths already in the pool: per
// bounce intersect, (the guide's inference,) the material sort, shade and
// shadow. Timing marks bracket intersect, shade and shadow when `timing`.
void enqueue_bounces(cenote_renderer* r, const cenote_scene* sc, const WaveParams& wp, uint32_t n0, bool guided,
                     cudaStream_t stream, bool timing, bool counting, WaveCounts* wc) {
    cenote_context* ctx = r->ctx;
    auto mark = [&]() {
        if (timing) cudaEventRecord(r->event(wc->events++), stream);
    };
    for (uint32_t b = 0; b < wp.max_bounces; ++b) {
        const bool sort = r->material_sort == CENOTE_SORT_ALL || (r->material_sort == CENOTE_SORT_SECONDARY && b > 0);
        const PathPool view = sort ? r->sorted_view() : r->pool;
        if (sort) launch_sort_begin(view, stream);
        launch_intersect(sc->ds, view, b, n0, ctx->shape, counting, stream);
        if (counting) {
            launch_count_hits(view, b, n0, stream);
            wc->launches++;
        }
        mark();
        if (guided) guide::launch_infer_paths(r->guide->view(), sc->ds, r->pool, b, n0, r->guide->sms, stream);
        if (sort) {
            launch_material_sort(view, b, n0, ctx->shape, stream);
            wc->launches += sc->ds.has_layers ? 3 : 2;  // a split shading launch adds one
        }
        launch_shade(sc->ds, view, b, wp, n0, ctx->shape, stream);
        mark();
        launch_shadow(sc->ds, r->pool, b, ctx->shape, counting, stream);
        mark();
    }
}

// One multi-job wave on `stream` (the serving loop): the segments' camera
// paths (`segs`, device memory, `nseg` of them, `paths` paths and `items`
// accumulate items in all; with `hdr` those three counts are read from it on
// the device instead, so a captured graph replays any wave), the bounces,
// and each segment's samples added into its job's film. No guides, no
// learned guide, no host waits. The pool must hold the wave's paths.
cudaError_t enqueue_segments(cenote_renderer* r, const cenote_scene* sc, const WaveSegment* segs, uint32_t nseg,
                             uint32_t paths, uint32_t items, const uint32_t* hdr, uint32_t max_bounces,
                             cudaStream_t stream, WaveCounts* wc) {
    r->pool.refill_idle = r->refill_idle;
    r->pool.top_nodes = r->top_nodes;
    r->pool.per_lane_triangles = r->per_lane_triangles;
    r->pool.trav_variant = r->trav_variant;
    r->pool.sort_location = r->sort_by_location;
    WaveParams wp{};
    wp.max_bounces = max_bounces;
    wp.light_sampling = r->light_sampling;
    const uint32_t n0 = hdr ? 0u : paths;  // 0: the kernels read the count raygen leaves
    launch_wave_begin_segments(r->pool, segs, nseg, paths, hdr, r->ctx->shape, stream);
    enqueue_bounces(r, sc, wp, n0, false, stream, false, false, wc);
    launch_tally(r->pool, r->tally.as<unsigned long long>(), n0, max_bounces, stream);
    launch_accumulate_segments(r->pool, segs, nseg, items, hdr, stream);
    wc->launches += 3 + 3 * max_bounces;
    wc->waves++;
    return cudaGetLastError();
}

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
                          cudaStream_t stream, bool timing, bool counting, WaveCounts* wc) {
    cenote_context* ctx = r->ctx;
    const uint64_t pixels = uint64_t(width) * height;
    r->pool.refill_idle = r->refill_idle;
    r->pool.top_nodes = r->top_nodes;
    r->pool.per_lane_triangles = r->per_lane_triangles;
    r->pool.trav_variant = r->trav_variant;
    r->pool.sort_location = r->sort_by_location;
    WaveParams wp{};
    wp.width = width;
    wp.height = height;
    wp.max_bounces = max_bounces;
    wp.light_sampling = r->light_sampling;
    wp.sample_offset = sample_offset;
    camera_basis(sc->camera, float(width) / float(height), wp);
    auto mark = [&]() {
        if (timing) cudaEventRecord(r->event(wc->events++), stream);
    };
    // The learned guide: mixture outputs after each intersect, training records
    // from the shading kernel, then Adam steps on the wave's records.
    const bool guided = r->guide && r->pool.guide_out;
    if (guided) {
        const double per_wave = double(std::min<uint64_t>(plan.range, pixels)) * plan.spw * 3.0;
        GuideRecordSink sk{r->g_records.ptr, r->g_count.as<uint32_t>(), cenote_renderer::GUIDE_RECORDS,
                           float(std::min(1.0, cenote_renderer::GUIDE_RECORDS / std::max(1.0, per_wave))),
                           r->guide_fraction, 0};
        cudaError_t e = cudaMemcpyAsync(r->g_sink.ptr, &sk, sizeof sk, cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return e;
    }
    for (uint32_t done = 0; done < count;) {
        uint32_t s = std::min(plan.spw, count - done);
        for (uint64_t base = 0; base < pixels; base += plan.range) {
            wp.pixel_base = uint32_t(base);
            wp.pixel_count = uint32_t(std::min<uint64_t>(plan.range, pixels - base));
            wp.tile_width = CN_TILE_PIXELS && base == 0 && wp.pixel_count == pixels && width % 8 == 0 &&
                                    height % 4 == 0
                                ? width
                                : 0u;
            wp.samples = s;
            wp.sample_base = sample0 + done;
            const uint32_t n0 = wp.pixel_count * s;
            mark();
            if (guided) cudaMemsetAsync(r->g_count.ptr, 0, 4, stream);
            launch_wave_begin(r->pool, wp, ctx->shape, stream);
            mark();
            enqueue_bounces(r, sc, wp, n0, guided, stream, timing, counting, wc);
            launch_tally(r->pool, r->tally.as<unsigned long long>(), n0, max_bounces, stream);
            if (film)
                launch_accumulate(r->pool, *film, wp.pixel_base, wp.pixel_count, wp.tile_width, s,
                                  film_reset && done == 0, stream);
            else
                launch_copy_rad(r->pool, oneshot, wp.pixel_base, wp.pixel_count, wp.tile_width, stream);
            mark();
            if (guided) {
                guide::Record* recs = r->g_records.as<guide::Record>();
                const uint32_t* cnt = r->g_count.as<uint32_t>();
                guide::launch_resolve_records(recs, cnt, cenote_renderer::GUIDE_RECORDS, r->pool.rad, stream);
                const float3 bmin = make_float3(sc->ds.bbox_min[0], sc->ds.bbox_min[1], sc->ds.bbox_min[2]);
                for (uint32_t k = 0; k < r->guide_steps; ++k) {
                    r->guide->step++;
                    guide::launch_train_records(r->guide->view(), r->guide->scratch(cenote_renderer::GUIDE_BATCH), recs,
                                                cnt, cenote_renderer::GUIDE_RECORDS, k * cenote_renderer::GUIDE_BATCH,
                                                bmin, sc->ds.bbox_inv, r->guide_lr, r->guide->step, r->guide->sms,
                                                stream);
                }
            }
            wc->launches += 3 + 3 * max_bounces;
            wc->waves++;
        }
        done += s;
    }
    return cudaGetLastError();
}


}  // namespace cn
