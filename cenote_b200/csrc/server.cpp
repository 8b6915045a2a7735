// The serving loop: progressive render jobs admitted by an HBM budget and
// traced together as one wavefront of job-tagged paths.
//
// The reference renders one view at a time (render::Session,
// crates/cenote/src/render/session.rs:416: a render thread accumulating one
// film and publishing frames); serving many uneven jobs is this library's
// addition at the boundary (cenote_server_*, cenote_job_*). Design:
//  * A job is (scene, width, height, target spp, max bounces). Submission
//    only queues it; the server thread admits queued jobs in arrival order
//    while the budget holds them: the path pool, every resident scene's
//    device bytes (BVH, triangles, records, textures, environment tables;
//    counted once while any admitted job renders it) and each job's film
//    (sums and averages) - and while fewer than `max_active` are resident.
//  * One or two lanes, each a path pool with a low- and a high-priority
//    stream; an idle lane takes the next wave (first-frame waves on the
//    high-priority stream), so the waves of two lanes overlap and hide each
//    other's tails and launch gaps. Each wave is a set of segments, each one
//    job's samples of its whole image, all of one (scene, max bounces)
//    group: raygen gives every path its job's image size, camera and sample
//    index from its segment (k_raygen_segments), the bounces run over the
//    mixed paths exactly as for one job, and accumulate adds each segment's
//    samples to its job's film in ascending order (k_accumulate_segments).
//    A path therefore traces what a standalone render of its job traces for
//    the same (pixel, sample), and the film adds the same values in the same
//    order: a job's result is bitwise the same alone and in any mix.
//  * First frames come first, cheapest first: the next wave is the group of
//    the job whose first frame is expected to take the least device time
//    (its paths over the group's measured rate), and it opens with that
//    group's waiting first frames, smallest first, up to the wave's time
//    budget, then fills with the group's progressive work unless other first
//    frames still wait. No progressive wave starts while first frames wait;
//    one may run on the other lane beside a first-frame wave. Other waves
//    round-robin the groups with progressive work, their jobs round-robin
//    inside, each taking at most the rest of its current frame. A progressive wave holds at most about
//    `CN_WAVE_MS` of device time (the group's paths per millisecond measured
//    on its earlier waves), so a new first frame waits at most about that
//    long for the wave in flight.
//  * Each group's wave is captured once into a CUDA graph per segment-table
//    slot; its kernels read the segment count, path count and accumulate
//    items from the table's header on the device, so one graph replays
//    every wave of the group (only the table is copied in per wave).
//  * A job is in at most one wave in flight, so its samples stay in order
//    and its pinned frame buffer is never overwritten while its callback
//    reads it. At a frame's end the wave also resolves the job's film into
//    its pinned buffer; the server thread polls the wave's event and hands
//    each frame to the job's callback.
//  * A finished job's film and pinned frame buffers go to a cache keyed by
//    size for the next jobs (the device bytes count against the budget and
//    are freed only when admission needs the room): cudaFree and
//    cudaFreeHost wait for the whole device.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <thread>

#include "runtime.h"

using namespace cn;

namespace cn {
void camera_basis(const cenote_camera& cam, float aspect, WaveParams& wp);
}

namespace {

// Device time a progressive wave aims at; a first frame waits about this
// long for the wave in flight.
// 1: a first-frame wave keeps the other lane idle. Measured at 64 jobs in
// flight, letting the other lane run progressive work beside it gave the
// better p99 time to first frame after the opening burst (47 against 49-289
// ms over runs) and throughput (653 against 607-642 Msamples/s), so it is 0.
#ifndef CN_FIRST_EXCLUSIVE
#define CN_FIRST_EXCLUSIVE 0
#endif
// A progressive wave's device time in ms. Measured at 64 jobs in flight: 7
// gives p99 time to first frame after the opening burst of 44.3, 44.2 and
// 48.4 ms (three runs) at 633, 631 and 608 Msamples/s, 10 gives 53.8, 48.5,
// 50.2 and 47.1 ms at 631, 658, 649 and 653: 7 keeps the first-frame target
// of 50 ms for about 4 % of throughput; 20 raises throughput about 11 % and
// the first-frame wait with it.
#ifndef CN_WAVE_MS
#define CN_WAVE_MS 7.0
#endif
constexpr uint32_t MAX_SEGMENTS = 512;

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
    uint32_t samples = 0;    // completed
    uint32_t scheduled = 0;  // enqueued (completed + in the wave in flight)
    bool in_flight = false;
    uint64_t bytes = 0;      // film bytes counted against the budget
    DeviceBuffer sum, avg;
    float* host = nullptr;   // pinned frame buffer
    WaveParams cam{};        // the camera basis at admission, for this image's aspect
    double t_submit = -1, t_admit = -1, t_first = -1, t_done = -1;

    void free_device() {
        if (host) cudaFreeHost(host);
        host = nullptr;
        sum.release();
        avg.release();
    }
};

// Jobs that can share a wave: one scene, one bounce count.
struct GroupKey {
    cenote_scene* scene;
    uint32_t max_bounces;
    bool operator<(const GroupKey& o) const {
        return scene != o.scene ? scene < o.scene : max_bounces < o.max_bounces;
    }
};

struct Group {
    std::vector<uint64_t> jobs;  // admitted, unfinished, in arrival order
    size_t cursor = 0;           // round-robin position for progressive work
    double paths_per_ms = 0.0;   // measured on this group's waves (0: none yet)
    // One captured wave per table slot (its kernels read the slot's header
    // and segments), with the scene record it was captured against: an edit
    // of the scene (a delta light added) captures it again.
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    DeviceScene captured[2]{};
    bool graph_failed = false;

    void drop_graphs() {
        for (auto& g : graph)
            if (g) cudaGraphExecDestroy(g);
        graph[0] = graph[1] = nullptr;
    }
};

// A segment table in memory: a 256-byte header (segments, paths, accumulate
// items) then the segments.
constexpr size_t TABLE_HEADER = 256;
constexpr size_t TABLE_BYTES = TABLE_HEADER + MAX_SEGMENTS * sizeof(WaveSegment);

struct WaveEntry {
    uint64_t job;
    uint32_t samples;
    bool frame;  // the wave ends one of the job's frames
};

struct Wave {
    GroupKey key{};
    std::vector<WaveEntry> entries;
    uint32_t paths = 0;
    bool first = false;  // opened with first frames
    cudaEvent_t start = nullptr, done = nullptr;
    bool active = false;
};

}  // namespace

struct cenote_server {
    cenote_context* ctx = nullptr;
    uint64_t budget = 0, used = 0;
    cenote_server_options opt{};
    // Lanes: each has its own path pool and a low- and a high-priority
    // stream (first-frame waves take the high one); one wave per lane is in
    // flight, and waves of different lanes overlap on the device.
    uint32_t lanes = 1;
    cudaStream_t streams[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    cenote_renderer renderers[2];
    uint64_t pool_bytes = 0;
    // Segment tables: host staging (pinned) and device copies, one per wave
    // in flight.
    uint8_t* seg_host[2] = {nullptr, nullptr};
    DeviceBuffer seg_dev[2];
    Wave waves[2];  // the wave in flight on each lane
    std::mutex mu;
    std::condition_variable cv;
    std::deque<uint64_t> queue;
    std::map<GroupKey, Group> groups;
    size_t group_cursor = 0;
    std::map<cenote_scene*, uint32_t> resident;  // scene -> admitted jobs rendering it
    std::multimap<size_t, void*> free_dev, free_host;
    uint64_t cached = 0;
    std::map<uint64_t, std::unique_ptr<Job>> jobs;
    uint64_t next_id = 1;
    uint32_t active = 0;
    std::thread thread;
    bool stop = false;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    uint64_t submitted = 0, completed = 0, failed = 0, samples = 0;
    uint64_t wave_count = 0, first_wave_count = 0, wave_paths = 0;
    double busy_ms = 0.0;
    std::map<uint64_t, std::unique_ptr<float[]>> results;

    static uint64_t job_bytes(uint32_t w, uint32_t h) { return uint64_t(w) * h * 32; }
    static uint64_t path_bytes() { return 16 * 5 + 8 + 4 + 8 + sizeof(ShadowRay) + 8; }

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

    // Drop a finished or failed job from its group, the budget and the
    // scene's residency. `reuse`: its buffers serve the next jobs; a failed
    // job's may still be in use by work enqueued before the failure, so
    // they are freed (which waits for the device).
    void retire(Job& j, bool reuse = true) {
        auto g = groups.find(GroupKey{j.scene, j.max_bounces});
        if (g != groups.end()) {
            auto& v = g->second.jobs;
            v.erase(std::remove(v.begin(), v.end(), j.id), v.end());
            if (v.empty()) {
            g->second.drop_graphs();
            groups.erase(g);
        }
        }
        if (reuse) {
            give_dev(j.sum);
            give_dev(j.avg);
            give_host(j.host, size_t(j.width) * j.height * 16);
        }
        j.free_device();
        used -= j.bytes;
        j.bytes = 0;
        auto r = resident.find(j.scene);
        if (r != resident.end() && --r->second == 0) {
            used -= j.scene->device_bytes;
            resident.erase(r);
        }
        if (active) active--;
        cv.notify_all();
    }

    void fail_job(Job& j, int32_t code) {
        j.error = code;
        j.state = CENOTE_JOB_FAILED;
        j.t_done = now_ms(t0);
        retire(j, false);
        failed++;
    }

    // Admit queued jobs in arrival order while budget and `max_active` allow.
    void admit() {
        while (!queue.empty() && active < opt.max_active) {
            Job& j = *jobs[queue.front()];
            const uint64_t bytes = job_bytes(j.width, j.height);
            const uint64_t scene_bytes = resident.count(j.scene) ? 0 : j.scene->device_bytes;
            const size_t px = size_t(j.width) * j.height;
            if (used + bytes + scene_bytes > budget) break;
            // Cached buffers of this size serve it without new device bytes.
            const uint64_t reusable = free_dev.count(px * 16) >= 2 ? uint64_t(px) * 32 : 0;
            if (used + cached + bytes + scene_bytes - reusable > budget) {
                evict(bytes + scene_bytes);
                if (used + cached + bytes + scene_bytes > budget) break;
            }
            queue.pop_front();
            cudaError_t e;
            if ((e = take_dev(j.sum, px * 16)) || (e = take_dev(j.avg, px * 16)) || (e = take_host(&j.host, px * 16))) {
                j.free_device();
                j.error = e == cudaErrorMemoryAllocation ? CENOTE_E_ALLOCATION : CENOTE_E_DEVICE;
                j.state = CENOTE_JOB_FAILED;
                j.t_done = now_ms(t0);
                failed++;
                continue;
            }
            used += bytes + scene_bytes;
            j.bytes = bytes;
            resident[j.scene]++;
            j.cam.width = j.width;
            j.cam.height = j.height;
            camera_basis(j.scene->camera, float(j.width) / float(j.height), j.cam);
            groups[GroupKey{j.scene, j.max_bounces}].jobs.push_back(j.id);
            j.state = CENOTE_JOB_RUNNING;
            j.t_admit = now_ms(t0);
            active++;
        }
    }

    // A job whose first frame is not yet all enqueued.
    bool wants_first(const Job& j) const { return !j.in_flight && j.scheduled < std::min(opt.frame_spp, j.target); }

    // The device time a job's first frame is expected to take: its paths
    // over its group's measured rate (paths alone until one is measured).
    double first_cost(const Job& j) const {
        const double paths = double(j.width) * j.height * std::min(opt.frame_spp, j.target);
        auto g = groups.find(GroupKey{j.scene, j.max_bounces});
        const double rate = g != groups.end() ? g->second.paths_per_ms : 0.0;
        return rate > 0.0 ? paths / rate : paths * 1e-6;
    }

    // First frames first, the cheapest first (so a burst of arrivals costs
    // the small jobs little), a job's wait counting against its cost (so
    // none starves): the group of the best job waiting for its first frame;
    // else, once no first frame waits or runs, the next group (round robin)
    // with progressive work; null when nothing should start.
    Group* pick_group(GroupKey* key, bool* first) {
        const Job* cheapest = nullptr;
        double best = 0.0;
        const double now = now_ms(t0);
        for (auto& kv : groups)
            for (uint64_t id : kv.second.jobs) {
                const Job& j = *jobs[id];
                if (!wants_first(j)) continue;
                const double c = first_cost(j) - (now - j.t_submit);
                if (!cheapest || c < best) {
                    cheapest = &j;
                    best = c;
                }
            }
        if (cheapest) {
            *key = GroupKey{cheapest->scene, cheapest->max_bounces};
            *first = true;
            return &groups[*key];
        }
        *first = false;
        if (groups.empty()) return nullptr;
        // With CN_FIRST_EXCLUSIVE, no progressive wave while a first-frame
        // wave runs: the first frames have the device to themselves.
        if (CN_FIRST_EXCLUSIVE)
            for (const Wave& w : waves)
                if (w.active && w.first) return nullptr;
        for (size_t n = 0; n < groups.size(); ++n) {
            auto it = groups.begin();
            std::advance(it, (group_cursor + n) % groups.size());
            for (uint64_t id : it->second.jobs) {
                const Job& j = *jobs[id];
                if (!j.in_flight && j.scheduled < j.target) {
                    group_cursor = (group_cursor + n + 1) % groups.size();
                    *key = it->first;
                    return &it->second;
                }
            }
        }
        return nullptr;
    }

    bool first_frames_waiting() const {
        for (auto& kv : groups)
            for (uint64_t id : kv.second.jobs)
                if (wants_first(*jobs.at(id))) return true;
        return false;
    }

    // Fill wave slot `w` from one group; false when there is nothing to run.
    bool build(Wave& w, WaveSegment* segs, uint32_t* nseg, uint32_t* items) {
        GroupKey key{};
        bool first = false;
        Group* g = pick_group(&key, &first);
        if (!g) return false;
        const uint64_t cap = opt.pool_paths;
        // Progressive work stops near the wave's time budget once the group's
        // rate is known; first frames fill what they need, up to the pool.
        const uint64_t soft = g->paths_per_ms > 0.0
                                  ? std::max<uint64_t>(1, std::min<uint64_t>(cap, uint64_t(g->paths_per_ms * CN_WAVE_MS)))
                                  : cap / 4;
        uint64_t paths = 0;
        uint32_t pixels = 0, n = 0;
        w.entries.clear();
        w.key = key;
        w.first = first;
        auto add = [&](Job& j, uint32_t count, bool frame) {
            WaveSegment& s = segs[n++];
            const uint32_t px = j.width * j.height;
            s.start = uint32_t(paths);
            s.pixel_start = pixels;
            s.width = j.width;
            s.height = j.height;
            s.pixel_base = 0;
            s.pixel_count = px;
            s.samples = count;
            s.sample_base = j.scheduled;
            s.cam_pos = j.cam.cam_pos;
            s.cam_right = j.cam.cam_right;
            s.cam_up = j.cam.cam_up;
            s.cam_fwd = j.cam.cam_fwd;
            s.aperture = j.cam.aperture;
            s.reset = j.scheduled == 0 ? 1u : 0u;
            s.film = j.sum.as<float4>();
            paths += uint64_t(px) * count;
            pixels += px;
            j.scheduled += count;
            j.in_flight = true;
            w.entries.push_back({j.id, count, frame});
        };
        // The rest of the job's current frame: frame_spp samples, the last
        // frame possibly shorter.
        auto frame_rest = [&](const Job& j) {
            return std::min(opt.frame_spp - j.scheduled % opt.frame_spp, j.target - j.scheduled);
        };
        if (first) {
            // The group's first frames, cheapest first, up to the wave's time
            // budget (the first always, up to the pool).
            std::vector<uint64_t> order;
            for (uint64_t id : g->jobs)
                if (wants_first(*jobs[id])) order.push_back(id);
            std::stable_sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) {
                return uint64_t(jobs[a]->width) * jobs[a]->height < uint64_t(jobs[b]->width) * jobs[b]->height;
            });
            for (uint64_t id : order) {
                Job& j = *jobs[id];
                if (n >= MAX_SEGMENTS || (n > 0 && paths >= soft)) break;
                const uint64_t px = uint64_t(j.width) * j.height;
                const uint32_t rest = frame_rest(j);
                const uint32_t count = uint32_t(std::min<uint64_t>(rest, (cap - paths) / px));
                if (count == 0) continue;
                add(j, count, count == rest);
            }
        }
        // Progressive work, round robin from the group's cursor, until the
        // wave's time budget; the first segment may pass it (never the pool).
        // A first-frame wave takes none while other first frames wait.
        const size_t m = first && first_frames_waiting() ? 0 : g->jobs.size();
        for (size_t k = 0; k < m && n < MAX_SEGMENTS && paths < soft; ++k) {
            const size_t at = (g->cursor + k) % m;
            Job& j = *jobs[g->jobs[at]];
            if (j.in_flight || j.scheduled == 0 || j.scheduled >= j.target) continue;
            const uint64_t px = uint64_t(j.width) * j.height;
            const uint32_t rest = frame_rest(j);
            const uint64_t room = n == 0 ? std::max<uint64_t>(soft, px) : soft - paths;
            const uint32_t count = uint32_t(std::min<uint64_t>(rest, std::min<uint64_t>(room, cap - paths) / px));
            if (count == 0) continue;
            add(j, count, count == rest);
            g->cursor = (at + 1) % m;
        }
        if (n == 0) return false;
        w.paths = uint32_t(paths);
        *nseg = n;
        *items = pixels;
        return true;
    }

    // The wave graph of `g` for lane `slot` (its pool and segment table),
    // captured on first use (or again after a scene edit); null if capture
    // failed (waves of the group then launch directly).
    cudaGraphExec_t wave_graph(Group& g, const GroupKey& key, uint32_t slot, cudaStream_t stream) {
        if (g.graph_failed) return nullptr;
        if (g.graph[slot] && std::memcmp(&g.captured[slot], &key.scene->ds, sizeof(DeviceScene)) == 0)
            return g.graph[slot];
        if (g.graph[slot]) cudaGraphExecDestroy(g.graph[slot]);
        g.graph[slot] = nullptr;
        cudaGraph_t graph = nullptr;
        WaveCounts wc;
        const uint32_t* hdr = seg_dev[slot].as<uint32_t>();
        const WaveSegment* segs = reinterpret_cast<const WaveSegment*>(seg_dev[slot].as<uint8_t>() + TABLE_HEADER);
        cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t e2 =
                enqueue_segments(&renderers[slot], key.scene, segs, 0, 0, 0, hdr, key.max_bounces, stream, &wc);
            e = cudaStreamEndCapture(stream, &graph);
            if (e2 != cudaSuccess) e = e2;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&g.graph[slot], graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            cudaGetLastError();
            g.graph[slot] = nullptr;
            g.graph_failed = true;
            return nullptr;
        }
        g.captured[slot] = key.scene->ds;
        return g.graph[slot];
    }

    // Build and enqueue the next wave on lane `slot`; false if idle.
    bool launch(uint32_t slot) {
        Wave& w = waves[slot];
        uint32_t nseg = 0, items = 0;
        WaveSegment* table = reinterpret_cast<WaveSegment*>(seg_host[slot] + TABLE_HEADER);
        if (!build(w, table, &nseg, &items)) return false;
        cudaStream_t stream = streams[slot][w.first ? 1 : 0];
        uint32_t* hdr = reinterpret_cast<uint32_t*>(seg_host[slot]);
        hdr[0] = nseg;
        hdr[1] = w.paths;
        hdr[2] = items;
        cudaError_t e = cudaEventRecord(w.start, stream);
        if (!e) e = cudaMemcpyAsync(seg_dev[slot].ptr, seg_host[slot], TABLE_HEADER + nseg * sizeof(WaveSegment),
                                    cudaMemcpyHostToDevice, stream);
        cudaGraphExec_t graph = nullptr;
        if (!e && opt.no_graphs == 0) graph = wave_graph(groups[w.key], w.key, slot, stream);
        if (!e && graph) {
            e = cudaGraphLaunch(graph, stream);
        } else if (!e) {
            WaveCounts wc;
            const WaveSegment* segs = reinterpret_cast<const WaveSegment*>(seg_dev[slot].as<uint8_t>() + TABLE_HEADER);
            e = enqueue_segments(&renderers[slot], w.key.scene, segs, nseg, w.paths, items, nullptr, w.key.max_bounces,
                                 stream, &wc);
        }
        // Frames that end here: the job's averages to its pinned buffer.
        for (const WaveEntry& en : w.entries) {
            if (e || !en.frame) continue;
            Job& j = *jobs[en.job];
            const uint32_t px = j.width * j.height;
            launch_resolve(j.sum.as<float4>(), j.avg.as<float4>(), px, float(j.scheduled), stream);
            e = cudaMemcpyAsync(j.host, j.avg.ptr, size_t(px) * 16, cudaMemcpyDeviceToHost, stream);
        }
        if (!e) e = cudaEventRecord(w.done, stream);
        w.active = true;
        if (e) {
            cudaGetLastError();
            // Nothing of this wave can be trusted: fail its jobs once it drains.
            cudaStreamSynchronize(stream);
            for (const WaveEntry& en : w.entries) fail_job(*jobs[en.job], CENOTE_E_DEVICE);
            w.active = false;
        }
        return true;
    }

    // A finished wave: its samples counted, its frames delivered.
    void finish(Wave& w, std::unique_lock<std::mutex>& lock) {
        w.active = false;
        cudaError_t q = cudaEventQuery(w.done);
        float ms = 0.0f;
        wave_count++;
        first_wave_count += w.first ? 1 : 0;
        wave_paths += w.paths;
        if (q == cudaSuccess && cudaEventElapsedTime(&ms, w.start, w.done) == cudaSuccess && ms > 0.0f) {
            busy_ms += ms;
            auto g = groups.find(w.key);
            if (g != groups.end()) {
                const double rate = double(w.paths) / double(ms);
                g->second.paths_per_ms = g->second.paths_per_ms > 0.0 ? 0.5 * (g->second.paths_per_ms + rate) : rate;
            }
        }
        for (const WaveEntry& en : w.entries) {
            auto it = jobs.find(en.job);
            if (it == jobs.end()) continue;
            Job& j = *it->second;
            j.in_flight = false;
            if (j.state != CENOTE_JOB_RUNNING) continue;
            if (q != cudaSuccess) {
                fail_job(j, CENOTE_E_DEVICE);
                continue;
            }
            j.samples += en.samples;
            samples += uint64_t(en.samples) * j.width * j.height;
            if (!en.frame) continue;
            if (j.t_first < 0) j.t_first = now_ms(t0);
            if (j.fn) {
                cenote_frame_fn fn = j.fn;
                void* user = j.user;
                uint64_t id = j.id;
                uint32_t smp = j.samples, tgt = j.target, wd = j.width, ht = j.height;
                const float* frame = j.host;
                lock.unlock();
                fn(user, id, smp, tgt, frame, wd, ht);
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
        if (q != cudaSuccess && q != cudaErrorNotReady) cudaGetLastError();
        cv.notify_all();
    }

    void loop() {
        cudaSetDevice(ctx->device);
        std::unique_lock<std::mutex> lock(mu);
        while (!stop) {
            admit();
            bool progressed = false;
            for (uint32_t k = 0; k < lanes; ++k) {
                Wave& w = waves[k];
                if (w.active && cudaEventQuery(w.done) != cudaErrorNotReady) {
                    finish(w, lock);
                    progressed = true;
                }
            }
            // Idle lanes take the next wave: first frames first.
            uint32_t in_flight = 0;
            for (uint32_t k = 0; k < lanes; ++k) {
                if (!waves[k].active && launch(k)) progressed = true;
                in_flight += waves[k].active ? 1u : 0u;
            }
            if (!progressed) {
                if (queue.empty() && active == 0 && in_flight == 0) {
                    cv.wait_for(lock, std::chrono::milliseconds(5));
                } else {
                    lock.unlock();
                    std::this_thread::sleep_for(std::chrono::microseconds(20));
                    lock.lock();
                }
            }
        }
    }
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
    if (s->opt.slots == 0) s->opt.slots = 2;
    if (s->opt.frame_spp == 0) s->opt.frame_spp = 4;
    if (s->opt.max_active == 0) s->opt.max_active = 64;
    if (s->opt.pool_paths == 0) s->opt.pool_paths = 1u << 24;
    CN_CHECK(s->opt.slots <= 64 && s->opt.pool_paths < (1u << 30), CENOTE_E_INVALID_ARGUMENT,
             "at most 2^30 paths in the pool");
    CN_CHECK(s->opt.light_sampling <= CENOTE_LIGHT_SAMPLING_NEE, CENOTE_E_INVALID_ARGUMENT, "unknown light sampling");
    CN_CUDA(cudaSetDevice(ctx->device));
    s->lanes = std::min(2u, std::max(1u, s->opt.slots));
    s->pool_bytes = uint64_t(s->opt.pool_paths) * cenote_server::path_bytes() * s->lanes;
    CN_CHECK(s->pool_bytes <= hbm_budget, CENOTE_E_BUDGET, "the path pools exceed the budget");
    int least = 0, greatest = 0;
    CN_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    for (uint32_t k = 0; k < s->lanes; ++k) {
        CN_CUDA(cudaStreamCreateWithPriority(&s->streams[k][0], cudaStreamNonBlocking, least));
        CN_CUDA(cudaStreamCreateWithPriority(&s->streams[k][1], cudaStreamNonBlocking, greatest));
        cenote_renderer& r = s->renderers[k];
        r.ctx = ctx;
        r.light_sampling = s->opt.light_sampling;
        CN_CUDA(r.ensure(s->opt.pool_paths));
        CN_CUDA(r.counters.alloc(CTR_COUNT * 4));
        CN_CUDA(r.tally.alloc(64));
        CN_CUDA(cudaMemset(r.tally.ptr, 0, 64));
        r.pool.counters = r.counters.as<uint32_t>();
        CN_CUDA(r.set_guides(false));
    }
    for (int k = 0; k < 2; ++k) {
        CN_CUDA(cudaMallocHost(reinterpret_cast<void**>(&s->seg_host[k]), TABLE_BYTES));
        CN_CUDA(s->seg_dev[k].alloc(TABLE_BYTES));
        CN_CUDA(cudaEventCreate(&s->waves[k].start));
        CN_CUDA(cudaEventCreate(&s->waves[k].done));
    }
    s->used = s->pool_bytes;
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
    for (auto& lane : s->streams)
        for (cudaStream_t st : lane)
            if (st) {
                cudaStreamSynchronize(st);
                cudaStreamDestroy(st);
            }
    for (int k = 0; k < 2; ++k) {
        if (s->seg_host[k]) cudaFreeHost(s->seg_host[k]);
        if (s->waves[k].start) cudaEventDestroy(s->waves[k].start);
        if (s->waves[k].done) cudaEventDestroy(s->waves[k].done);
    }
    for (auto& kv : s->groups) kv.second.drop_graphs();
    for (auto& kv : s->jobs) kv.second->free_device();
    for (auto& kv : s->free_dev) cudaFree(kv.second);
    for (auto& kv : s->free_host) cudaFreeHost(kv.second);
    cenote_context* ctx = s->ctx;
    delete s;
    release(ctx);
}

int32_t cenote_job_submit(cenote_server* s, cenote_scene* scene, uint32_t width, uint32_t height, uint32_t target_spp,
                          uint32_t max_bounces, cenote_frame_fn fn, void* user, uint64_t* job) {
    CN_CHECK(s && scene && job, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(scene->ctx == s->ctx, CENOTE_E_INVALID_ARGUMENT, "scene from another context");
    CN_CHECK(width > 0 && height > 0 && target_spp > 0, CENOTE_E_INVALID_ARGUMENT, "zero-sized job");
    CN_CHECK(uint64_t(width) * height <= s->opt.pool_paths, CENOTE_E_INVALID_ARGUMENT,
             "a job's image must fit the path pool (one sample of every pixel)");
    CN_CHECK(max_bounces >= 1 && max_bounces <= MAX_BOUNCES, CENOTE_E_INVALID_ARGUMENT, "bounces outside 1..=255");
    std::lock_guard<std::mutex> lock(s->mu);
    const uint64_t bytes = cenote_server::job_bytes(width, height) + scene->device_bytes;
    CN_CHECK(s->pool_bytes + bytes <= s->budget, CENOTE_E_BUDGET, "the job alone exceeds the budget");
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
    st->waves = s->wave_count;
    st->first_waves = s->first_wave_count;
    st->wave_paths = s->wave_paths;
    st->busy_ms = s->busy_ms;
    return CENOTE_OK;
}

}  // extern "C"
