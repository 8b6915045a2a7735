// The serving loop: progressive render jobs admitted by an HBM budget and
// multiplexed over a fixed set of CUDA streams.
//
// The reference renders one view at a time (render::Session,
// crates/cenote/src/render/session.rs:416: a render thread accumulating one
// film and publishing frames); serving many uneven jobs is this library's
// addition at the boundary (cenote_server_*, cenote_job_*). Design:
//  * A job is (scene, width, height, target spp, max bounces). Submission
//    only queues it; a server thread admits queued jobs in arrival order while
//    their resident footprint (film sums and averages, pinned frame buffer
//    excluded) fits in the budget and fewer than `max_active` are resident.
//  * `slots` streams each own a path pool of fixed capacity, allocated once
//    and counted against the budget. An admitted job is bound to the slot
//    with the fewest jobs; a slot runs one chunk (`frame_spp` samples, one
//    progressive frame) of one job at a time, so jobs on different slots
//    overlap on the device.
//  * First frames come first, device-wide: admitted jobs wait for their
//    first chunk in one arrival-order queue served by two slots that render
//    nothing else (so a first frame never waits for a busy slot) and by any
//    idle slot, and while first frames are queued or in flight no slot
//    starts another job's progressive chunk, so the chunks in flight drain
//    and the first frames get the device. Otherwise a slot round-robins the chunks of the
//    jobs bound to it. A job's full-size chunk is
//    captured once into a CUDA graph and replayed; the graph reads the job's
//    sample offset from device memory, advanced by a node at its end, so
//    replays need no parameter updates. A shorter final chunk is enqueued
//    directly.
//  * A finished job's film sums and averages and its pinned frame buffer go to
//    a cache keyed by size for the next jobs (the device bytes count against
//    the budget and are freed only when admission needs the room):
//    cudaFree and cudaFreeHost wait for the whole device, which stalled the
//    loop behind every chunk in flight (measured: first frames of jobs
//    submitted meanwhile waited 0.8 s).
//  * After the first frame, a frame's samples may run as several pieces of
//    about one path pool each, so progressive work in flight stays small.
//  * After each frame the film is resolved into the job's pinned buffer and
//    an event marks it; the server thread polls events and hands each frame
//    to the job's callback. Sample order within a film is ascending, so a
//    job's result is bitwise the same alone and in any mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <cstring>
#include <map>
#include <thread>

#include "runtime.h"

using namespace cn;

namespace {

double now_ms(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

struct Job {
    uint64_t id = 0;
    cenote_scene* scene = nullptr;
    uint32_t width = 0, height = 0, target = 0, max_bounces = 0;
    cenote_frame_fn fn = nullptr;
    void* user = nullptr;
    uint32_t state = CENOTE_JOB_QUEUED;
    int32_t error = CENOTE_OK;
    uint32_t samples = 0;   // completed
    uint32_t pending = 0;   // in the chunk in flight
    bool frame_pending = false;  // the chunk in flight ends a progressive frame
    int slot = -1;
    uint64_t bytes = 0;     // resident footprint counted against the budget
    DeviceBuffer sum, avg, offset;
    float* host = nullptr;  // pinned frame buffer
    cudaGraphExec_t graph = nullptr;
    cudaEvent_t done = nullptr;
    bool graph_tried = false;
    double t_submit = -1, t_admit = -1, t_first = -1, t_done = -1;

    void free_device() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        if (done) cudaEventDestroy(done);
        done = nullptr;
        if (host) cudaFreeHost(host);
        host = nullptr;
        sum.release();
        avg.release();
        offset.release();
    }
};

struct Slot {
    cudaStream_t stream = nullptr;
    cenote_renderer renderer;
    std::vector<uint64_t> jobs;  // resident jobs bound to this slot
    size_t next = 0;             // round-robin cursor
    uint64_t busy = 0;           // job whose chunk is in flight (0: idle)
    bool first_only = false;     // renders first frames only (no jobs bound to it)
};

// Slots that render first frames only (index 0 .. CN_FIRST_SLOTS-1).
#ifndef CN_FIRST_SLOTS
#define CN_FIRST_SLOTS 2
#endif

}  // namespace

struct cenote_server {
    cenote_context* ctx = nullptr;
    uint64_t budget = 0, used = 0;
    cenote_server_options opt{};
    std::vector<std::unique_ptr<Slot>> slots;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<uint64_t> queue;
    std::deque<uint64_t> first_queue;  // admitted jobs waiting for their first chunk
    std::multimap<size_t, void*> free_dev, free_host;  // retired jobs' buffers by size
    uint64_t cached = 0;                               // device bytes in free_dev
    uint32_t first_in_flight = 0;      // first chunks on the device
    std::map<uint64_t, std::unique_ptr<Job>> jobs;
    uint64_t next_id = 1;
    uint32_t active = 0;
    std::thread thread;
    bool stop = false;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    uint64_t submitted = 0, completed = 0, failed = 0, samples = 0;

    uint64_t job_bytes(uint32_t w, uint32_t h) const { return uint64_t(w) * h * 32 + 256; }

    // Fail a job and drop its resources (caller holds mu).
    void fail_job(Job& j, int32_t code) {
        j.error = code;
        j.state = CENOTE_JOB_FAILED;
        j.t_done = now_ms(t0);
        retire(j, false);
        failed++;
    }

    // A device buffer of `bytes` from the cache, else newly allocated.
    cudaError_t take_dev(DeviceBuffer& b, size_t bytes) {
        auto it = free_dev.find(bytes);
        if (it != free_dev.end()) {
            b.ptr = it->second;
            b.bytes = bytes;
            free_dev.erase(it);
            cached -= bytes;
            return cudaSuccess;
        }
        return b.alloc(bytes);
    }

    void give_dev(DeviceBuffer& b) {
        if (!b.ptr) return;
        free_dev.emplace(b.bytes, b.ptr);
        cached += b.bytes;
        b.ptr = nullptr;
        b.bytes = 0;
    }

    cudaError_t take_host(float** p, size_t bytes) {
        auto it = free_host.find(bytes);
        if (it != free_host.end()) {
            *p = static_cast<float*>(it->second);
            free_host.erase(it);
            return cudaSuccess;
        }
        return cudaMallocHost(reinterpret_cast<void**>(p), bytes);
    }

    void give_host(float*& p, size_t bytes) {
        if (!p) return;
        free_host.emplace(bytes, p);
        p = nullptr;
    }

    // Free cached device buffers until `need` more bytes fit the budget (or
    // none are left).
    void evict(uint64_t need) {
        while (used + cached + need > budget && !free_dev.empty()) {
            auto it = free_dev.begin();
            cudaFree(it->second);
            cached -= it->first;
            free_dev.erase(it);
        }
    }

    // `reuse`: the job's chunks have all completed, so its buffers can serve
    // the next jobs; a failed job's may still be in use by work enqueued
    // before the failure, so they are freed (which waits for the device).
    void retire(Job& j, bool reuse = true) {
        if (j.slot >= 0) {
            auto& v = slots[size_t(j.slot)]->jobs;
            v.erase(std::remove(v.begin(), v.end(), j.id), v.end());
        }
        first_queue.erase(std::remove(first_queue.begin(), first_queue.end(), j.id), first_queue.end());
        if (reuse) {
            give_dev(j.sum);
            give_dev(j.avg);
            give_dev(j.offset);
            give_host(j.host, size_t(j.width) * j.height * 16);
        }
        j.free_device();
        used -= j.bytes;
        j.bytes = 0;
        if (active) active--;
        cv.notify_all();
    }

    // Admit queued jobs in arrival order while budget and slots allow.
    void admit() {
        while (!queue.empty() && active < opt.max_active) {
            Job& j = *jobs[queue.front()];
            uint64_t bytes = job_bytes(j.width, j.height);
            if (used + bytes > budget) break;
            const size_t px = size_t(j.width) * j.height;
            // Cached buffers of this size serve it without new device bytes.
            const bool reuse = free_dev.count(px * 16) >= 2 && free_dev.count(16) >= 1;
            const uint64_t reusable = reuse ? uint64_t(px) * 32 + 16 : 0;
            if (used + cached + bytes - reusable > budget) {
                evict(bytes);
                if (used + cached + bytes > budget) break;
            }
            queue.pop_front();
            cudaError_t e;
            if ((e = take_dev(j.sum, px * 16)) || (e = take_dev(j.avg, px * 16)) || (e = take_dev(j.offset, 16)) ||
                (e = take_host(&j.host, px * 16)) ||
                (e = cudaEventCreateWithFlags(&j.done, cudaEventDisableTiming))) {
                j.free_device();
                j.error = e == cudaErrorMemoryAllocation ? CENOTE_E_ALLOCATION : CENOTE_E_DEVICE;
                j.state = CENOTE_JOB_FAILED;
                j.t_done = now_ms(t0);
                failed++;
                continue;
            }
            used += bytes;
            j.bytes = bytes;
            size_t best = CN_FIRST_SLOTS;
            for (size_t k = best + 1; k < slots.size(); ++k)
                if (slots[k]->jobs.size() < slots[best]->jobs.size()) best = k;
            j.slot = int(best);  // for its progressive chunks; its first chunk runs on any idle slot
            slots[best]->jobs.push_back(j.id);
            first_queue.push_back(j.id);
            j.state = CENOTE_JOB_RUNNING;
            j.t_admit = now_ms(t0);
            active++;
        }
    }

    // The slot's next progressive chunk: its bound jobs round-robin, past
    // those still waiting for a first frame.
    Job* pick(Slot& s) {
        for (size_t k = 0; k < s.jobs.size(); ++k) {
            s.next %= s.jobs.size();
            Job* j = jobs[s.jobs[s.next++]].get();
            if (j->samples > 0) return j;
        }
        return nullptr;
    }

    // Samples per progressive piece: as many as one path pool holds, at most
    // a frame's worth.
    uint32_t piece_spp(const Job& j) const {
        const uint64_t px = uint64_t(j.width) * j.height;
        return uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(opt.frame_spp, uint64_t(opt.pool_paths) / px)));
    }

    WavePlan plan_for(const Job& j, uint32_t n) const {
        const uint64_t px = uint64_t(j.width) * j.height;
        const uint64_t cap = opt.pool_paths;
        WavePlan p;
        if (px > cap) {
            p.range = uint32_t(cap);
            p.spw = 1;
        } else {
            p.range = uint32_t(px);
            p.spw = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(n, cap / px)));
        }
        p.need = uint64_t(p.range) * p.spw;
        return p;
    }

    // Enqueue the job's next chunk on slot `s` (no host waits). A first
    // chunk clears the job's sums and sample offset first and is launched
    // directly: the slot it runs on need not be the one whose path pool a
    // captured graph would bind.
    cudaError_t launch_chunk(Slot& s, Job& j) {
        const bool first = j.samples == 0;
        if (first) {
            const size_t px = size_t(j.width) * j.height;
            cudaError_t e0 = cudaMemsetAsync(j.sum.ptr, 0, px * 16, s.stream);
            if (e0 == cudaSuccess) e0 = cudaMemsetAsync(j.offset.ptr, 0, 16, s.stream);
            if (e0 != cudaSuccess) return e0;
        }
        // A first chunk is the whole first frame; later frames go in pieces
        // of about one path pool (frame_spp samples at most), so a new job's
        // first frame never waits long for progressive work in flight.
        const uint32_t remaining = j.target - j.samples;
        const uint32_t piece = piece_spp(j);
        const uint32_t n = first ? std::min(opt.frame_spp, remaining)
                                 : std::min({piece, remaining, opt.frame_spp - j.samples % opt.frame_spp});
        const bool frame = (j.samples + n) % opt.frame_spp == 0 || j.samples + n == j.target;
        FilmTargets film{j.sum.as<float4>(), nullptr, nullptr, nullptr};  // previews carry no guides
        WavePlan plan = plan_for(j, n);
        cudaError_t e = cudaSuccess;
        const bool full = n == piece;
        if (full && !first && opt.no_graphs == 0 && !j.graph && !j.graph_tried) {
            j.graph_tried = true;
            cudaGraph_t g = nullptr;
            WaveCounts wc;
            e = cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                cudaError_t e2 = enqueue_waves(&s.renderer, j.scene, j.width, j.height, 0, n, j.max_bounces, plan,
                                               &film, false, nullptr, j.offset.as<uint32_t>(), s.stream, false, false,
                                               &wc);
                launch_advance(j.offset.as<uint32_t>(), n, s.stream);
                e = cudaStreamEndCapture(s.stream, &g);
                if (e2 != cudaSuccess) e = e2;
            }
            if (e == cudaSuccess) e = cudaGraphInstantiate(&j.graph, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                cudaGetLastError();
                j.graph = nullptr;  // fall back to direct launches for this job
                e = cudaSuccess;
            }
        }
        if (full && !first && j.graph) {
            e = cudaGraphLaunch(j.graph, s.stream);
        } else {
            WaveCounts wc;
            e = enqueue_waves(&s.renderer, j.scene, j.width, j.height, 0, n, j.max_bounces, plan, &film, false,
                              nullptr, j.offset.as<uint32_t>(), s.stream, false, false, &wc);
            if (e == cudaSuccess) launch_advance(j.offset.as<uint32_t>(), n, s.stream);
        }
        if (e != cudaSuccess) return e;
        if (frame) {
            const uint32_t px = j.width * j.height;
            launch_resolve(j.sum.as<float4>(), j.avg.as<float4>(), px, float(j.samples + n), s.stream);
            if ((e = cudaMemcpyAsync(j.host, j.avg.ptr, size_t(px) * 16, cudaMemcpyDeviceToHost, s.stream))) return e;
        }
        if ((e = cudaEventRecord(j.done, s.stream))) return e;
        j.pending = n;
        j.frame_pending = frame;
        s.busy = j.id;
        if (first) first_in_flight++;
        return cudaGetLastError();
    }

    void loop() {
        cudaSetDevice(ctx->device);
        std::unique_lock<std::mutex> lock(mu);
        while (!stop) {
            admit();
            bool progressed = false;
            for (auto& sp : slots) {
                Slot& s = *sp;
                if (s.busy) {
                    Job& j = *jobs[s.busy];
                    cudaError_t q = cudaEventQuery(j.done);
                    if (q == cudaErrorNotReady) continue;
                    s.busy = 0;
                    progressed = true;
                    if (j.samples == 0 && first_in_flight) first_in_flight--;
                    if (q != cudaSuccess) {
                        cudaGetLastError();
                        fail_job(j, CENOTE_E_DEVICE);
                        continue;
                    }
                    j.samples += j.pending;
                    samples += uint64_t(j.pending) * j.width * j.height;
                    j.pending = 0;
                    if (j.frame_pending) {  // else a piece of a frame: nothing to deliver yet
                        if (j.t_first < 0) j.t_first = now_ms(t0);
                        if (j.fn) {
                            cenote_frame_fn fn = j.fn;
                            void* user = j.user;
                            uint64_t id = j.id;
                            uint32_t smp = j.samples, tgt = j.target, w = j.width, h = j.height;
                            const float* frame = j.host;
                            lock.unlock();
                            fn(user, id, smp, tgt, frame, w, h);
                            lock.lock();
                        }
                        if (j.samples >= j.target) {
                            j.state = CENOTE_JOB_DONE;
                            j.t_done = now_ms(t0);
                            // Keep the final averages on the host for cenote_job_result;
                            // release the device side.
                            const size_t px = size_t(j.width) * j.height;
                            float* keep = new float[px * 4];
                            std::memcpy(keep, j.host, px * 16);
                            results[j.id].reset(keep);
                            retire(j);
                            completed++;
                        }
                    }
                }
                if (!s.busy) {
                    Job* j = nullptr;
                    if (!first_queue.empty()) {
                        j = jobs[first_queue.front()].get();
                        first_queue.pop_front();
                    } else if (first_in_flight == 0 && !s.first_only) {
                        j = pick(s);
                    }
                    if (j) {
                        cudaError_t e = launch_chunk(s, *j);
                        progressed = true;
                        if (e != cudaSuccess) {
                            cudaGetLastError();
                            fail_job(*j, CENOTE_E_DEVICE);
                        }
                    }
                }
            }
            if (!progressed) {
                bool idle = queue.empty() && active == 0;
                if (idle)
                    cv.wait_for(lock, std::chrono::milliseconds(5));
                else {
                    lock.unlock();
                    std::this_thread::sleep_for(std::chrono::microseconds(20));
                    lock.lock();
                }
            }
        }
    }

    std::map<uint64_t, std::unique_ptr<float[]>> results;
};

extern "C" {

int32_t cenote_server_create(cenote_context* ctx, uint64_t hbm_budget, const cenote_server_options* options,
                             cenote_server** out) {
    CN_CHECK(ctx && out, CENOTE_E_INVALID_ARGUMENT, "null context or output handle");
    *out = nullptr;
    auto s = std::make_unique<cenote_server>();
    s->ctx = ctx;
    s->budget = hbm_budget;
    if (options) s->opt = *options;
    if (s->opt.slots == 0) s->opt.slots = 8;
    if (s->opt.frame_spp == 0) s->opt.frame_spp = 4;
    if (s->opt.max_active == 0) s->opt.max_active = 64;
    if (s->opt.pool_paths == 0) s->opt.pool_paths = 1u << 21;
    CN_CHECK(s->opt.slots <= 64 && s->opt.pool_paths < (1u << 30), CENOTE_E_INVALID_ARGUMENT,
             "at most 64 slots and 2^30 paths per pool");
    CN_CHECK(s->opt.light_sampling <= CENOTE_LIGHT_SAMPLING_NEE, CENOTE_E_INVALID_ARGUMENT, "unknown light sampling");
    CN_CUDA(cudaSetDevice(ctx->device));
    // Each slot's pool: path state + queues + shadow records, no guide lanes.
    const uint64_t pool_bytes = uint64_t(s->opt.pool_paths) * (16 * 5 + 8 + 4 + 8 + sizeof(ShadowRay));
    const uint32_t all_slots = CN_FIRST_SLOTS + s->opt.slots;
    CN_CHECK(pool_bytes * all_slots <= hbm_budget, CENOTE_E_BUDGET, "the slots' path pools exceed the budget");
    for (uint32_t k = 0; k < all_slots; ++k) {
        auto slot = std::make_unique<Slot>();
        slot->first_only = k < CN_FIRST_SLOTS;
        CN_CUDA(cudaStreamCreateWithFlags(&slot->stream, cudaStreamNonBlocking));
        cenote_renderer& r = slot->renderer;
        r.ctx = ctx;
        r.light_sampling = s->opt.light_sampling;
        CN_CUDA(r.ensure(s->opt.pool_paths));
        CN_CUDA(r.counters.alloc(CTR_COUNT * 4));
        CN_CUDA(r.tally.alloc(64));
        CN_CUDA(cudaMemset(r.tally.ptr, 0, 64));
        r.pool.counters = r.counters.as<uint32_t>();
        CN_CUDA(r.set_guides(false));
        s->slots.push_back(std::move(slot));
    }
    s->used = pool_bytes * all_slots;
    retain(ctx);
    cenote_server* raw = s.release();
    raw->thread = std::thread([raw] { raw->loop(); });
    *out = raw;
    return CENOTE_OK;
}

void cenote_server_destroy(cenote_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    s->thread.join();
    cudaSetDevice(s->ctx->device);
    for (auto& sp : s->slots) {
        cudaStreamSynchronize(sp->stream);
        cudaStreamDestroy(sp->stream);
    }
    for (auto& kv : s->jobs) kv.second->free_device();
    for (auto& kv : s->free_dev) cudaFree(kv.second);
    for (auto& kv : s->free_host) cudaFreeHost(kv.second);
    cenote_context* ctx = s->ctx;
    s->slots.clear();
    delete s;
    release(ctx);
}

int32_t cenote_job_submit(cenote_server* s, cenote_scene* scene, uint32_t width, uint32_t height, uint32_t target_spp,
                          uint32_t max_bounces, cenote_frame_fn fn, void* user, uint64_t* job) {
    CN_CHECK(s && scene && job, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(scene->ctx == s->ctx, CENOTE_E_INVALID_ARGUMENT, "scene from another context");
    CN_CHECK(width > 0 && height > 0 && target_spp > 0, CENOTE_E_INVALID_ARGUMENT, "zero-sized job");
    CN_CHECK(uint64_t(width) * height < (1ull << 31), CENOTE_E_INVALID_ARGUMENT, "target too large");
    CN_CHECK(max_bounces >= 1 && max_bounces <= MAX_BOUNCES, CENOTE_E_INVALID_ARGUMENT, "bounces outside 1..=255");
    std::lock_guard<std::mutex> lock(s->mu);
    const uint64_t bytes = s->job_bytes(width, height);
    uint64_t pools = uint64_t(s->opt.pool_paths) * (16 * 5 + 8 + 4 + 8 + sizeof(ShadowRay)) *
                     (CN_FIRST_SLOTS + s->opt.slots);
    CN_CHECK(pools + bytes <= s->budget, CENOTE_E_BUDGET, "the job alone exceeds the budget");
    auto j = std::make_unique<Job>();
    j->id = s->next_id++;
    j->scene = scene;
    j->width = width;
    j->height = height;
    j->target = target_spp;
    j->max_bounces = max_bounces;
    j->fn = fn;
    j->user = user;
    j->t_submit = now_ms(s->t0);
    *job = j->id;
    s->queue.push_back(j->id);
    s->jobs[j->id] = std::move(j);
    s->submitted++;
    s->cv.notify_all();
    return CENOTE_OK;
}

int32_t cenote_job_poll(cenote_server* s, uint64_t job, cenote_job_status* st) {
    CN_CHECK(s && st, CENOTE_E_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job);
    CN_CHECK(it != s->jobs.end(), CENOTE_E_INVALID_ARGUMENT, "unknown job");
    const Job& j = *it->second;
    *st = cenote_job_status{};
    st->state = j.state;
    st->samples = j.samples;
    st->target = j.target;
    st->error = j.error;
    st->submit_ms = j.t_submit;
    st->admit_ms = j.t_admit;
    st->first_frame_ms = j.t_first;
    st->done_ms = j.t_done;
    return CENOTE_OK;
}

int32_t cenote_job_wait(cenote_server* s, uint64_t job, double timeout_ms) {
    CN_CHECK(s, CENOTE_E_INVALID_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job);
    CN_CHECK(it != s->jobs.end(), CENOTE_E_INVALID_ARGUMENT, "unknown job");
    Job* j = it->second.get();
    bool ok = s->cv.wait_for(lock, std::chrono::duration<double, std::milli>(timeout_ms), [&] {
        return j->state == CENOTE_JOB_DONE || j->state == CENOTE_JOB_FAILED;
    });
    if (!ok) return fail(CENOTE_E_TIMEOUT, "job not finished within the wait bound");
    if (j->state == CENOTE_JOB_FAILED) return fail(j->error, "job failed on the device");
    return CENOTE_OK;
}

int32_t cenote_job_result(cenote_server* s, uint64_t job, float* rgba) {
    CN_CHECK(s && rgba, CENOTE_E_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job);
    CN_CHECK(it != s->jobs.end(), CENOTE_E_INVALID_ARGUMENT, "unknown job");
    const Job& j = *it->second;
    CN_CHECK(j.state == CENOTE_JOB_DONE, CENOTE_E_INVALID_ARGUMENT, "job not done");
    auto r = s->results.find(job);
    CN_CHECK(r != s->results.end(), CENOTE_E_INVALID_ARGUMENT, "result already released");
    std::memcpy(rgba, r->second.get(), size_t(j.width) * j.height * 16);
    return CENOTE_OK;
}

int32_t cenote_job_release(cenote_server* s, uint64_t job) {
    CN_CHECK(s, CENOTE_E_INVALID_ARGUMENT, "null server");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job);
    CN_CHECK(it != s->jobs.end(), CENOTE_E_INVALID_ARGUMENT, "unknown job");
    CN_CHECK(it->second->state == CENOTE_JOB_DONE || it->second->state == CENOTE_JOB_FAILED,
             CENOTE_E_INVALID_ARGUMENT, "job still queued or running");
    s->results.erase(job);
    s->jobs.erase(it);
    return CENOTE_OK;
}

int32_t cenote_server_stats(cenote_server* s, cenote_server_counters* st) {
    CN_CHECK(s && st, CENOTE_E_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    *st = cenote_server_counters{};
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->failed = s->failed;
    st->queued = s->queue.size();
    st->active = s->active;
    st->samples = s->samples;
    st->bytes_in_use = s->used + s->cached;
    st->budget = s->budget;
    st->wall_ms = now_ms(s->t0);
    return CENOTE_OK;
}

}  // extern "C"
