// server.cpp - continuous batching of collision scenarios on one device.
//
// Scenarios (requests) arrive with their initial Stars and a step count.  Each
// scheduling round (gcs_server_tick):
//   1. admits queued scenarios in arrival order while the segment slots and
//      the particle capacity that the HBM budget buys allow;
//   2. if membership changed, lays the context out again: resident
//      scenarios keep their device state (moved on the device by
//      gcs_relayout), newly admitted ones are uploaded into their segments;
//   3. advances every resident scenario by one step with one launch per
//      stage over the concatenated segments (a CUDA graph, captured again
//      only after a membership change);
//   4. writes simulation.bin frames of scenarios that asked for one this
//      step, and retires scenarios that reached their step count: their
//      final Stars are kept for gcs_server_pop and, with an output
//      directory set, their last frame is appended to <dir>/<id>.bin.
// Segments are independent, so every scenario's result is byte-identical to
// running it alone with the same parameters.  At most two steps are queued
// on the device ahead of the host, so admission decisions are never more
// than two steps stale.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <deque>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/gcs.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Scenario {
    uint64_t id = 0;
    std::vector<Star> init;
    int64_t n = 0;
    int32_t steps = 0;
    int32_t done = 0;
    int32_t seg = -1;  // segment in the current layout, -1 until uploaded
    int32_t frames = 0;
    int32_t status = GCS_OK;
    Clock::time_point t_submit, t_admit, t_finish;
    std::vector<Star> result;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct gcs_server {
    gcs_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t step_done[2] = {nullptr, nullptr};
    int64_t ticks = 0;
    int64_t particle_steps = 0;  // progress counters (gcs_server_progress)
    int64_t peak_scenarios = 0, peak_particles = 0;
    gcs_params p;
    int64_t capacity = 0;
    int32_t max_segments = 0;
    std::deque<Scenario> queued;
    std::vector<Scenario> resident;  // in segment order
    std::deque<Scenario> finished;
    bool layout_dirty = false;
    std::string out_dir;
    int32_t frame_every = 0;
    std::vector<PlaybackStar> frame;
    std::string last_error;
};

namespace {

void release(gcs_server* s) {
    if (s->ctx) gcs_destroy(s->ctx);
    for (cudaEvent_t& e : s->step_done)
        if (e) cudaEventDestroy(e);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

int fail(gcs_server* s, int rc, const char* what) {
    s->last_error = what;
    if (s->ctx && gcs_last_error(s->ctx)[0]) {
        s->last_error += ": ";
        s->last_error += gcs_last_error(s->ctx);
    }
    return rc;
}

// Append scenario r's current state (segment r.seg) to <dir>/<id>.bin as one
// frame of PlaybackStar records, the reference's bake format.
int write_frame(gcs_server* s, Scenario& r) {
    s->frame.resize((size_t)r.n);
    int rc = gcs_download_playback(s->ctx, s->frame.data(), gcs_segment_offset(s->ctx, r.seg), r.n);
    if (rc) return fail(s, rc, "frame download");
    const std::string path = s->out_dir + "/" + std::to_string(r.id) + ".bin";
    FILE* f = std::fopen(path.c_str(), r.frames == 0 ? "wb" : "ab");
    if (!f) return fail(s, GCS_ERR_ARG, "cannot open the scenario's output file");
    const size_t put = std::fwrite(s->frame.data(), sizeof(PlaybackStar), (size_t)r.n, f);
    std::fclose(f);
    if (put != (size_t)r.n) return fail(s, GCS_ERR_ARG, "short write of a frame");
    ++r.frames;
    return GCS_OK;
}

}  // namespace

extern "C" {

int gcs_server_create(gcs_server** out, int32_t device, int64_t max_particles, int32_t max_segments,
                      double hbm_budget_bytes, const gcs_params* p) {
    if (!out || !p || max_particles < 1 || max_segments < 1 || !(hbm_budget_bytes > 0)) return GCS_ERR_ARG;
    *out = nullptr;
    gcs_server* s = new gcs_server();
    s->max_segments = max_segments;
    s->p = *p;
    // The largest particle capacity whose whole context fits the budget (the
    // footprint grows monotonically with the capacity).
    int64_t bytes = gcs_context_bytes(max_particles, max_segments, device);
    if (bytes < 0) {
        delete s;
        return (int)bytes;
    }
    int64_t cap = max_particles;
    if ((double)bytes > hbm_budget_bytes) {
        int64_t lo = 0, hi = max_particles;  // fits(lo) (or lo == 0), !fits(hi)
        while (hi - lo > 1) {
            const int64_t mid = lo + (hi - lo) / 2;
            if ((double)gcs_context_bytes(mid, max_segments, device) <= hbm_budget_bytes) lo = mid;
            else hi = mid;
        }
        cap = lo;
    }
    int rc = cap < 1 ? GCS_ERR_CAPACITY : gcs_create(&s->ctx, cap, max_segments, device);
    if (rc) {
        delete s;
        return rc;
    }
    s->capacity = cap;
    cudaSetDevice(device);
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->step_done[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->step_done[1], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        release(s);
        return GCS_ERR_CUDA;
    }
    gcs_set_stream(s->ctx, s->stream);
    rc = gcs_set_graphs(s->ctx, 1);
    if (rc) {
        release(s);
        return rc;
    }
    *out = s;
    return GCS_OK;
}

void gcs_server_destroy(gcs_server* s) {
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    release(s);
}

gcs_ctx* gcs_server_context(gcs_server* s) { return s ? s->ctx : nullptr; }

int64_t gcs_server_capacity(const gcs_server* s) { return s ? s->capacity : 0; }

const char* gcs_server_last_error(const gcs_server* s) { return s ? s->last_error.c_str() : "null server"; }

int gcs_server_set_output(gcs_server* s, const char* dir, int32_t frame_every) {
    if (!s || frame_every < 0) return GCS_ERR_ARG;
    s->out_dir = dir ? dir : "";
    s->frame_every = frame_every;
    return GCS_OK;
}

int gcs_server_submit(gcs_server* s, uint64_t id, const Star* stars, int64_t n, int32_t steps) {
    if (!s || !stars || n < 1 || steps < 1) return GCS_ERR_ARG;
    if (n > s->capacity) {
        s->last_error = "scenario larger than the particle capacity the HBM budget allows";
        return GCS_ERR_CAPACITY;
    }
    Scenario sc;
    sc.id = id;
    sc.init.assign(stars, stars + n);
    sc.n = n;
    sc.steps = steps;
    sc.t_submit = Clock::now();
    s->queued.push_back(std::move(sc));
    return GCS_OK;
}

int gcs_server_tick(gcs_server* s, int64_t out[4]) {
    if (!s) return GCS_ERR_ARG;
    int64_t particles = 0, admitted = 0, retired = 0;
    for (const Scenario& r : s->resident) particles += r.n;

    // 1. admission in arrival order (no overtaking: a large request at the
    //    head waits until it fits)
    while (!s->queued.empty()) {
        const Scenario& q = s->queued.front();
        if ((int32_t)s->resident.size() >= s->max_segments || particles + q.n > s->capacity) break;
        particles += q.n;
        s->resident.push_back(std::move(s->queued.front()));
        s->queued.pop_front();
        s->resident.back().t_admit = Clock::now();
        ++admitted;
        s->layout_dirty = true;
    }

    // 2. new layout: kept scenarios move on the device, new ones are uploaded
    if (s->layout_dirty && !s->resident.empty()) {
        std::vector<int64_t> counts;
        std::vector<int32_t> src;
        for (const Scenario& r : s->resident) {
            counts.push_back(r.n);
            src.push_back(r.seg);
        }
        int rc = gcs_relayout(s->ctx, (int32_t)counts.size(), counts.data(), src.data());
        if (rc) return fail(s, rc, "relayout");
        for (size_t i = 0; i < s->resident.size(); ++i) {
            Scenario& r = s->resident[i];
            if (r.seg < 0) {
                rc = gcs_upload_stars(s->ctx, r.init.data(), gcs_segment_offset(s->ctx, (int32_t)i), r.n);
                if (rc) return fail(s, rc, "upload");
                std::vector<Star>().swap(r.init);
            }
            r.seg = (int32_t)i;
        }
        s->layout_dirty = false;
    }

    if (!s->resident.empty()) {
        // 3. one step of every resident scenario, at most two steps in flight
        cudaEvent_t ev = s->step_done[s->ticks & 1];
        if (s->ticks >= 2 && cudaEventSynchronize(ev) != cudaSuccess) {
            cudaGetLastError();
            return fail(s, GCS_ERR_CUDA, "step event");
        }
        int rc = gcs_step(s->ctx, &s->p);
        if (rc) return fail(s, rc, "step");
        s->particle_steps += particles;
        s->peak_scenarios = std::max<int64_t>(s->peak_scenarios, (int64_t)s->resident.size());
        s->peak_particles = std::max(s->peak_particles, particles);
        if (cudaEventRecord(ev, s->stream) != cudaSuccess) {
            cudaGetLastError();
            return fail(s, GCS_ERR_CUDA, "step event");
        }
        ++s->ticks;

        // 4. frames and retirement
        bool any_done = false;
        for (Scenario& r : s->resident) {
            ++r.done;
            any_done |= r.done >= r.steps;
        }
        uint32_t dev = 0;
        if (any_done) {
            rc = gcs_device_status(s->ctx, &dev, 1);
            if (rc && rc != GCS_ERR_DEVICE) return fail(s, rc, "device status");
        }
        for (Scenario& r : s->resident) {
            const bool last = r.done >= r.steps;
            const bool frame = !s->out_dir.empty() &&
                               (last || (s->frame_every > 0 && r.done % s->frame_every == 0));
            if (frame) {
                rc = write_frame(s, r);
                if (rc) return rc;
            }
            if (!last) continue;
            r.result.resize((size_t)r.n);
            rc = gcs_download_stars(s->ctx, r.result.data(), gcs_segment_offset(s->ctx, r.seg), r.n);
            if (rc) return fail(s, rc, "result download");
            r.status = dev ? GCS_ERR_DEVICE : GCS_OK;
            r.t_finish = Clock::now();
        }
        std::vector<Scenario> keep;
        keep.reserve(s->resident.size());
        for (Scenario& r : s->resident) {
            if (r.done >= r.steps) {
                particles -= r.n;
                s->finished.push_back(std::move(r));
                ++retired;
            } else {
                keep.push_back(std::move(r));
            }
        }
        if (retired) {
            s->resident.swap(keep);
            s->layout_dirty = true;
        }
        if (dev) {
            s->last_error = "a kernel raised a device status bit";
            if (out) out[0] = (int64_t)s->resident.size(), out[1] = particles, out[2] = admitted, out[3] = retired;
            return GCS_ERR_DEVICE;
        }
    }
    if (out) {
        out[0] = (int64_t)s->resident.size();
        out[1] = particles;
        out[2] = admitted;
        out[3] = retired;
    }
    return GCS_OK;
}

int gcs_server_counts(const gcs_server* s, int64_t out[3]) {
    if (!s || !out) return GCS_ERR_ARG;
    out[0] = (int64_t)s->queued.size();
    out[1] = (int64_t)s->resident.size();
    out[2] = (int64_t)s->finished.size();
    return GCS_OK;
}

int gcs_server_progress(const gcs_server* s, int64_t out[4]) {
    if (!s || !out) return GCS_ERR_ARG;
    out[0] = s->particle_steps;
    out[1] = s->ticks;
    out[2] = s->peak_scenarios;
    out[3] = s->peak_particles;
    return GCS_OK;
}

int gcs_server_pop(gcs_server* s, gcs_server_result* info, Star* host, int64_t host_capacity) {
    if (!s || !info) return GCS_ERR_ARG;
    if (s->finished.empty()) return 0;
    Scenario& r = s->finished.front();
    if (host && host_capacity < r.n) return GCS_ERR_CAPACITY;
    info->id = r.id;
    info->n = r.n;
    info->steps = r.steps;
    info->status = r.status;
    info->queued_ms = ms_between(r.t_submit, r.t_admit);
    info->latency_ms = ms_between(r.t_submit, r.t_finish);
    if (host) std::memcpy(host, r.result.data(), sizeof(Star) * (size_t)r.n);
    s->finished.pop_front();
    return 1;
}

}  // extern "C"
