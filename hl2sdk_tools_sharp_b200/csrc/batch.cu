// batch.cu -- many maps lit on one device (vrad_batch_*).  No counterpart
// in the reference, which lights one map per call (Vrad.RunAsync,
// MapTools/Rad/Vrad.cs:160-390).
//
// A batch is a persistent runner: `created` host threads, each owning one
// context (its own stream, device tables and pinned staging), wait for
// work.  A run hands them one queue of maps, ordered largest first (the
// longest-processing-time rule: the big maps start early and the small
// ones fill the tail).  Each worker lights whole maps through the same
// calls a single-map host makes, so the lumps are the single-map lumps byte
// for byte.  The overlap is between maps: while one worker's map is in its
// host set-up (SAH build, sample slots, patch tree), other workers' light
// passes keep the device busy, and the small maps' kernels, which fill few
// of the 148 SMs alone, run side by side on the workers' streams.  Each
// context waits only for its own stream, never for the device.  The
// uploads' streams have the device's greatest priority and the passes'
// the least, so an upload's short kernels are not queued behind another
// map's transfer build, and a worker sleeps while it waits for the device.
//
// The autotuner picks the two launch knobs a batch has: the gather's
// threads per CTA (timed on the largest map) and the number of maps in
// flight (the batch timed at each worker count).

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

#include "context.cuh"
#include "device_pool.h"
#include "sync_wait.h"

struct vrad_batch {
    int device = 0;
    int created = 0;
    int tuned_workers = 0;   // 0: not tuned (a run uses every worker)
    int block = 0;           // the gather's threads per CTA; 0: the contexts' default
    std::vector<vrad_ctx *> ctx;
    std::vector<std::thread> threads;

    std::mutex run_mu;       // one run at a time
    std::mutex mu;
    std::condition_variable cv, done_cv;
    uint64_t gen = 0;
    bool stop = false;
    int active = 0;          // workers taking part in the current run
    int finished = 0;
    vrad_batch_map *maps = nullptr;
    std::vector<int32_t> order;
    std::atomic<int32_t> next{0};
};

namespace {

using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point t0) {
    return std::chrono::duration<double>(Clock::now() - t0).count();
}

void note_error(vrad_ctx *ctx, vrad_batch_map &m, int32_t rc) {
    m.status = rc;
    vrad_last_error(ctx, m.error, (int32_t)sizeof m.error);
}

// The whole lighting stage of one map on one context, through the
// single-map entry points.
void light_map(vrad_ctx *ctx, vrad_batch_map &m, int block) {
    const Clock::time_point t0 = Clock::now();
    m.status = VRAD_OK;
    m.error[0] = 0;
    m.lighting_bytes = 0;
    memset(&m.pass, 0, sizeof m.pass);
    memset(&m.bounce_stats, 0, sizeof m.bounce_stats);
    m.scene_s = m.world_s = m.bounce_s = m.pass_s = 0.0;
    Clock::time_point t = t0;
    auto lap = [&t](double &into) {
        const Clock::time_point now = Clock::now();
        into = std::chrono::duration<double>(now - t).count();
        t = now;
    };
    // The launch shape and the supersampling passes first: the world upload
    // queues the direct gather ahead with them.
    int32_t rc = vrad_set_extra_passes(ctx, m.extra_passes < 0 ? 4 : m.extra_passes);
    if (rc == VRAD_OK && block) {
        std::lock_guard<std::mutex> g(ctx->mu);
        ctx->world.block = block;
    }
    if (rc == VRAD_OK) rc = vrad_scene_upload(ctx, m.triangles, m.ntriangles);
    lap(m.scene_s);
    if (rc == VRAD_OK) rc = vrad_world_upload(ctx, m.world);
    lap(m.world_s);
    if (rc == VRAD_OK && m.bounce) rc = vrad_bounce_upload(ctx, m.bounce);
    lap(m.bounce_s);
    if (rc == VRAD_OK) rc = vrad_lighting_size(ctx, &m.lighting_bytes);
    if (rc == VRAD_OK) rc = vrad_light_pass(ctx, m.lighting, m.capacity, m.lightofs, &m.pass);
    if (rc == VRAD_OK && m.bounce) rc = vrad_bounce_stats_get(ctx, &m.bounce_stats);
    lap(m.pass_s);
    if (rc != VRAD_OK) note_error(ctx, m, rc);
    const cudaError_t e = vrad::release_tables(ctx);
    if (e != cudaSuccess && m.status == VRAD_OK) {
        m.status = vrad_cuda_fail(ctx, e, "releasing the map's tables");
        vrad_last_error(ctx, m.error, (int32_t)sizeof m.error);
    }
    m.seconds = seconds_since(t0);
}

void worker_loop(vrad_batch *b, int w) {
    // While this worker waits for its map's kernels, its core serves the
    // other workers' host set-up.
    vrad::set_sleeping_waits(true);
    uint64_t seen = 0;
    std::unique_lock<std::mutex> g(b->mu);
    while (true) {
        b->cv.wait(g, [&] { return b->stop || b->gen != seen; });
        if (b->stop) {
            cudaSetDevice(b->device);
            vrad::set_sleeping_waits(false);
            return;
        }
        seen = b->gen;
        const bool takes_part = w < b->active;
        g.unlock();
        if (takes_part) {
            const int32_t n = (int32_t)b->order.size();
            for (int32_t k; (k = b->next.fetch_add(1)) < n;) {
                vrad_batch_map &m = b->maps[b->order[(size_t)k]];
                light_map(b->ctx[(size_t)w], m, b->block);
                m.worker = w;
            }
        }
        g.lock();
        if (++b->finished == b->created) b->done_cv.notify_all();
    }
}

// Work estimate for the queue order: the gather's rays scale with the
// samples, the transfers' with the patches, which follow the surface area
// the samples also measure.  Bounced maps weigh double.
int64_t weight_of(const vrad_batch_map &m) {
    const int64_t s = m.world ? m.world->nsamples : 0;
    return (m.bounce ? 2 : 1) * s + m.ntriangles;
}

int32_t check_maps(const vrad_batch_map *maps, int32_t nmaps) {
    if (nmaps < 0 || (nmaps > 0 && !maps)) return vrad_fail(nullptr, VRAD_ERR_ARG, "null or negative map list");
    for (int32_t i = 0; i < nmaps; i++) {
        const vrad_batch_map &m = maps[i];
        if (!m.triangles || m.ntriangles <= 0 || !m.world || !m.lighting || m.capacity < 0)
            return vrad_fail(nullptr, VRAD_ERR_ARG, "map %d lacks triangles, a world or a lump buffer", i);
    }
    return VRAD_OK;
}

// One run of the queue on `workers` workers; the caller holds run_mu.
int32_t run_locked(vrad_batch *b, vrad_batch_map *maps, int32_t nmaps, int workers, vrad_batch_stats *stats) {
    const Clock::time_point t0 = Clock::now();
    const vrad::PoolCounters pc0 = vrad::dev_counters();
    {
        std::lock_guard<std::mutex> g(b->mu);
        b->maps = maps;
        b->order.resize((size_t)nmaps);
        std::iota(b->order.begin(), b->order.end(), 0);
        std::stable_sort(b->order.begin(), b->order.end(),
                         [&](int32_t x, int32_t y) { return weight_of(maps[x]) > weight_of(maps[y]); });
        b->next.store(0);
        b->active = std::min(workers, std::max(1, (int)nmaps));
        b->finished = 0;
        b->gen++;
    }
    b->cv.notify_all();
    {
        std::unique_lock<std::mutex> g(b->mu);
        b->done_cv.wait(g, [&] { return b->finished == b->created; });
        b->maps = nullptr;
    }
    // Maps that ran out of device memory beside the others run again, one
    // at a time on an emptied pool.
    bool trimmed = false;
    for (int32_t k = 0; k < nmaps; k++) {
        vrad_batch_map &m = maps[b->order[(size_t)k]];
        if (m.status != VRAD_ERR_OOM) continue;
        if (!trimmed) {
            cudaSetDevice(b->device);
            vrad::dev_trim(b->device);
            trimmed = true;
        }
        const double first = m.seconds;
        light_map(b->ctx[0], m, b->block);
        m.worker = 0;
        m.seconds += first;
    }
    vrad_batch_stats st;
    memset(&st, 0, sizeof st);
    st.workers = std::min(workers, std::max(1, (int)nmaps));
    st.maps = nmaps;
    st.block = b->block;
    st.seconds = seconds_since(t0);
    const vrad::PoolCounters pc1 = vrad::dev_counters();
    st.device_mallocs = pc1.mallocs - pc0.mallocs;
    st.device_malloc_bytes = pc1.malloc_bytes - pc0.malloc_bytes;
    st.device_trims = pc1.trims - pc0.trims;
    int32_t rc = VRAD_OK;
    for (int32_t i = 0; i < nmaps; i++) {
        const vrad_batch_map &m = maps[i];
        st.busy_seconds += m.seconds;
        if (m.status != VRAD_OK) {
            st.failed++;
            if (rc == VRAD_OK) rc = m.status;
            continue;
        }
        st.rays += m.pass.visibility_rays + m.pass.sky_rays + m.bounce_stats.transfer_rays;
        st.luxels += m.pass.luxels;
        st.lighting_bytes += m.lighting_bytes;
    }
    if (stats) *stats = st;
    if (rc != VRAD_OK) {
        for (int32_t i = 0; i < nmaps; i++)
            if (maps[i].status != VRAD_OK) {
                vrad_fail(nullptr, maps[i].status, "batch map %d: %s", i, maps[i].error);
                break;
            }
    }
    return rc;
}

}  // namespace

extern "C" int32_t vrad_batch_create(int32_t device, int32_t workers, vrad_batch **out) {
    if (!out) return vrad_fail(nullptr, VRAD_ERR_ARG, "null output");
    *out = nullptr;
    if (workers < 1 || workers > VRAD_BATCH_MAX_WORKERS)
        return vrad_fail(nullptr, VRAD_ERR_ARG, "workers %d outside 1..%d", workers, VRAD_BATCH_MAX_WORKERS);
    vrad_batch *b = new vrad_batch();
    b->device = device;
    for (int32_t w = 0; w < workers; w++) {
        vrad_ctx *c = nullptr;
        int32_t rc = vrad_create(device, &c);
        if (rc == VRAD_OK) {
            const cudaError_t e = vrad::prioritise_uploads(c);
            if (e != cudaSuccess) {
                vrad_destroy(c);
                c = nullptr;
                rc = vrad_cuda_fail(nullptr, e, "batch stream priorities");
            }
        }
        if (rc != VRAD_OK) {
            for (vrad_ctx *x : b->ctx) vrad_destroy(x);
            delete b;
            return rc;
        }
        b->ctx.push_back(c);
    }
    b->created = workers;
    for (int32_t w = 0; w < workers; w++) b->threads.emplace_back(worker_loop, b, (int)w);
    *out = b;
    return VRAD_OK;
}

extern "C" int32_t vrad_batch_destroy(vrad_batch *b) {
    if (!b) return VRAD_OK;
    {
        std::lock_guard<std::mutex> run(b->run_mu);
        {
            std::lock_guard<std::mutex> g(b->mu);
            b->stop = true;
        }
        b->cv.notify_all();
        for (std::thread &t : b->threads) t.join();
    }
    for (vrad_ctx *c : b->ctx) vrad_destroy(c);
    delete b;
    return VRAD_OK;
}

extern "C" int32_t vrad_batch_run(vrad_batch *b, vrad_batch_map *maps, int32_t nmaps, int32_t workers,
                                  vrad_batch_stats *stats) {
    if (!b) return vrad_fail(nullptr, VRAD_ERR_ARG, "null batch");
    int32_t rc = check_maps(maps, nmaps);
    if (rc != VRAD_OK) return rc;
    if (workers < 0 || workers > b->created)
        return vrad_fail(nullptr, VRAD_ERR_ARG, "workers %d outside 0..%d", workers, b->created);
    if (workers == 0) workers = b->tuned_workers ? b->tuned_workers : b->created;
    std::lock_guard<std::mutex> run(b->run_mu);
    return run_locked(b, maps, nmaps, workers, stats);
}

extern "C" int32_t vrad_batch_autotune(vrad_batch *b, vrad_batch_map *maps, int32_t nmaps, int32_t *chosen_workers,
                                       int32_t *chosen_block, double *seconds) {
    if (!b) return vrad_fail(nullptr, VRAD_ERR_ARG, "null batch");
    int32_t rc = check_maps(maps, nmaps);
    if (rc != VRAD_OK) return rc;
    if (nmaps == 0) return vrad_fail(nullptr, VRAD_ERR_ARG, "no maps to tune on");
    std::lock_guard<std::mutex> run(b->run_mu);
    // The launch shape, on the largest map.
    int32_t big = 0;
    for (int32_t i = 1; i < nmaps; i++)
        if (weight_of(maps[i]) > weight_of(maps[big])) big = i;
    vrad_ctx *c = b->ctx[0];
    rc = vrad_scene_upload(c, maps[big].triangles, maps[big].ntriangles);
    if (rc == VRAD_OK) rc = vrad_world_upload(c, maps[big].world);
    if (rc == VRAD_OK) rc = vrad_set_extra_passes(c, maps[big].extra_passes < 0 ? 4 : maps[big].extra_passes);
    int32_t block = 0;
    if (rc == VRAD_OK) rc = vrad_direct_autotune(c, &block, nullptr);
    if (rc != VRAD_OK) {
        char msg[256];
        vrad_last_error(c, msg, (int32_t)sizeof msg);
        return vrad_fail(nullptr, rc, "batch autotune, map %d: %s", big, msg);
    }
    b->block = block;
    // The maps in flight.  One untimed run on every worker first: the
    // device pool and the pinned tables then hold what the largest count
    // needs, so no count is timed with its first allocations.
    rc = run_locked(b, maps, nmaps, b->created, nullptr);
    if (rc != VRAD_OK) return rc;
    double best = 1e300;
    int best_w = b->created;
    for (int w = 1; w <= b->created; w++) {
        vrad_batch_stats st;
        rc = run_locked(b, maps, nmaps, w, &st);
        if (rc != VRAD_OK) return rc;
        if (seconds) seconds[w - 1] = st.seconds;
        if (st.seconds < best) {
            best = st.seconds;
            best_w = w;
        }
    }
    b->tuned_workers = best_w;
    if (chosen_workers) *chosen_workers = best_w;
    if (chosen_block) *chosen_block = block;
    return VRAD_OK;
}
