// engine.cu - the gcs_ctx context behind include/gcs.h: device buffers,
// segment layout, the per-step stage sequence and the C ABI.
//
// Replaces the reference's file-scope globals and cuda_physics_step
// (cuda_engine.cu:16-44, 219-451).  Differences in structure, not in
// results: state lives in a context (so several scenarios can share a
// device), all work is asynchronous on the context's stream with no device
// synchronisation between stages, and every failure is a status code.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda.h>  // driver API types for the pointer-range query (entry point fetched at run time)

#include "gcs_internal.h"

using namespace gcs;

struct gcs_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    int64_t capacity = 0;
    int32_t max_segments = 1;
    size_t device_bytes = 0;  // bytes this context holds on the device
    bool dry_run = false;      // count allocations without making them

    // layout
    int32_t n = 0, nseg = 0, n_internal = 0;
    std::vector<int64_t> h_seg_off;
    std::vector<int32_t> h_group_start;  // first particle of each walk group (host copy)
    std::vector<int64_t> h_chunk_first;  // first particle of each bounds chunk, then n (host copy)
    int n_groups = 0, n_chunks = 0;

    // device state
    float4* pos[2] = {nullptr, nullptr};
    float4* vel[2] = {nullptr, nullptr};
    float4* acc = nullptr;
    int cur = 0;
    uint64_t* keys[2] = {nullptr, nullptr};
    uint32_t* idx[2] = {nullptr, nullptr};
    int sorted_buf = 0;
    BvhNodeTraverse* tr = nullptr;
    BvhNodeBuild* bd = nullptr;
    // Walk records (one per internal node) and what they were written for:
    // the aggregation of generation wn_gen with G = wn_G and leaf size wn_L.
    // tree_gen counts enqueued aggregations and layout changes, so a walk
    // whose records are older than the tree, or were written for another G
    // or leaf size, first rewrites them from the traverse records.
    WalkNode* wn = nullptr;
    uint64_t tree_gen = 1;
    uint64_t wn_gen = 0;
    float wn_G = 0.0f;
    int32_t wn_L = 0;
    double4* com64 = nullptr;
    int32_t* leaf_parent = nullptr;
    int64_t* seg_off = nullptr;
    int32_t* seg_id = nullptr;
    WalkGroup* groups = nullptr;
    // walk frontiers: super-groups of consecutive groups, their lists
    SuperGroup* supers = nullptr;
    int32_t* sg_list = nullptr;
    int32_t* sg_src = nullptr;
    int4* sg_meta = nullptr;
    int n_supers = 0;
    size_t supers_cap = 0;
    int32_t* perm = nullptr;              // walk targets in group order (full super-groups partitioned)
    // second stream and events for the partition beside the frontier pass
    // (created at the first partitioned walk and kept)
    cudaStream_t part_stream = nullptr;
    cudaEvent_t part_fork = nullptr, part_join = nullptr;
    // the gather runs on part_stream beside the tree build (both need only
    // the sort); the build stage joins it
    cudaEvent_t gather_fork = nullptr, gather_join = nullptr;
    bool gather_pending = false;
    std::vector<int32_t> h_group_super;   // super-group of each walk group (host copy)
    Chunk* chunks = nullptr;
    float2* seg_bounds = nullptr;
    Star* staging = nullptr;
    PlaybackStar* pb_staging = nullptr;
    unsigned char* scratch = nullptr;
    size_t scratch_cap = 0;
    uint32_t* status = nullptr;
    double* diag = nullptr;
    int64_t* targets = nullptr;
    int64_t targets_cap = 0;
    double* direct_out = nullptr;
    unsigned long long* counts = nullptr;  // walk interaction counters (count mode)
    int2* walk_stack = nullptr;            // per-warp global bottoms of the walk stacks
    // splat renderer: fixed-point accumulator and RGBA staging, sized for
    // render_pixels_cap pixels (allocated at the first gcs_render_frame)
    unsigned long long* render_acc = nullptr;
    uint8_t* render_rgba = nullptr;
    int64_t render_pixels_cap = 0;
    // bake: two pinned frame buffers (bake_frames_cap records each), a copy
    // stream and its events, created at the first gcs_bake and kept
    PlaybackStar* bake_host[2] = {nullptr, nullptr};
    int64_t bake_frames_cap = 0;
    cudaStream_t bake_stream = nullptr;
    cudaEvent_t bake_packed[2] = {nullptr, nullptr};
    cudaEvent_t bake_copied[2] = {nullptr, nullptr};
    // host step with the Star copy overlapped with the walk (gcs_step_host):
    // a copy stream, an event after the walk, per-chunk completion flags in
    // mapped host memory (written by the walk's epilogue) and their device
    // counters; created at the first such step and kept
    cudaStream_t star_stream = nullptr;
    cudaEvent_t up_landed[8] = {};       // chunks of the step's Star upload (gcs_step_host_io)
    cudaEvent_t star_walked = nullptr;
    uint32_t* star_flags = nullptr;      // mapped host memory, kMaxStarChunks words
    uint32_t* star_flags_dev = nullptr;  // its device address
    uint32_t* star_chunk_done = nullptr;
    uint32_t star_epoch = 0;
    size_t walk_stack_entries = 0;
    int32_t group_width = 32;              // targets per walk group (<= 64; two per lane above 32)
    bool walk_frontier = true;             // super-group frontier pass before the walk
    // particles the walk and the kick/drift cover (sorted order; count < 0:
    // all): one rank's slice when one scenario is stepped across devices
    int64_t range_first = 0;
    int64_t range_count = -1;
    size_t groups_cap = 0;
    bool count_walk = false;

    // CUDA graphs of one full step, one per ping-pong parity of the particle
    // arrays (the gather flips it every step); rebuilt when the parameters,
    // the layout or the stream change.
    bool use_graphs = false;
    bool graphs_valid = false;
    gcs_params graph_params;
    cudaStream_t graph_stream = nullptr;
    cudaGraphExec_t graph_exec[2] = {nullptr, nullptr};
    int graph_after[2] = {1, 0};  // parity of the particle arrays after the graph of each parity
    int graph_builds = 0;
    // caller's events recorded around the walk stage (gcs_set_walk_events);
    // in a captured step they are event-record nodes, pointed at the events
    // set now before each launch
    cudaEvent_t walk_ev[2] = {nullptr, nullptr};
    cudaGraph_t graph[2] = {nullptr, nullptr};  // kept: their nodes address the exec graphs' nodes
    cudaGraphNode_t walk_ev_node[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [parity][start, end]
    cudaEvent_t walk_ev_bound[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};

    std::string last_error;
};

namespace {

constexpr int kChunkSize = 2048;  // particles per bounds block
constexpr int kCountWords = 17;  // counting-walk outputs: gcs_count_interactions, stack peak, lane use
constexpr int kMinGroupWidth = 8;

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

void set_error(gcs_ctx* c, const char* what, cudaError_t e) {
    char buf[256];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    c->last_error = buf;
}

#define GCS_CUDA(ctx, call)                                  \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) {                             \
            set_error((ctx), #call, e_);                     \
            return GCS_ERR_CUDA;                             \
        }                                                    \
    } while (0)

int check_launch(gcs_ctx* c, const char* stage) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(c, stage, e);
        return GCS_ERR_CUDA;
    }
    return GCS_OK;
}

Layout layout_of(const gcs_ctx* c) {
    Layout L;
    L.n = c->n;
    L.nseg = c->nseg;
    L.n_internal = c->n_internal;
    L.seg_off = c->seg_off;
    L.seg_id = c->seg_id;
    return L;
}

int seg_passes(int nseg) { return nseg <= 1 ? 0 : (nseg <= 256 ? 1 : 2); }

// Byte offsets of the scratch regions for n particles in nseg segments.
ScratchLayout scratch_layout(int32_t max_segments, int64_t n, int nseg) {
    ScratchLayout s;
    s.hist = 0;
    s.walk_q = round256(sizeof(uint32_t) * kMaxPasses * kRadix);
    s.bounds = s.walk_q + 256;
    s.tiles = s.bounds + round256(sizeof(uint32_t) * 2 * (size_t)max_segments);
    s.lookback = s.tiles + 256;
    s.end = s.lookback + sizeof(uint32_t) * sort_lookback_words(n, kKeyPasses + seg_passes(nseg));
    return s;
}
template <typename T>
T* scratch_at(gcs_ctx* c, size_t off) {
    return reinterpret_cast<T*>(c->scratch + off);
}

template <typename T>
int dalloc(gcs_ctx* c, T** p, size_t count) {
    if (c->dry_run) {  // footprint only (gcs_context_bytes)
        c->device_bytes += sizeof(T) * (count > 0 ? count : 1);
        return GCS_OK;
    }
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * (count > 0 ? count : 1));
    if (e != cudaSuccess) {
        set_error(c, "cudaMalloc", e);
        *p = nullptr;
        return GCS_ERR_NOMEM;
    }
    c->device_bytes += sizeof(T) * (count > 0 ? count : 1);
    return GCS_OK;
}

void drop_graphs(gcs_ctx* c) {
    for (auto& g : c->graph_exec) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    for (auto& g : c->graph) {
        if (g) cudaGraphDestroy(g);
        g = nullptr;
    }
    for (int k = 0; k < 2; ++k)
        for (int e = 0; e < 2; ++e) {
            c->walk_ev_node[k][e] = nullptr;
            c->walk_ev_bound[k][e] = nullptr;
        }
    c->graphs_valid = false;
}

// Record a caller's event on the context stream; under stream capture it
// becomes an event-record node of the graph.
cudaError_t record_event(cudaEvent_t ev, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const cudaError_t e = cudaStreamIsCapturing(st, &cs);
    if (e != cudaSuccess) return e;
    return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal)
                                               : cudaEventRecord(ev, st);
}

void free_all(gcs_ctx* c) {
    drop_graphs(c);
    if (c->bake_stream) {
        cudaStreamSynchronize(c->bake_stream);
        cudaStreamDestroy(c->bake_stream);
    }
    for (int b = 0; b < 2; ++b) {
        if (c->bake_packed[b]) cudaEventDestroy(c->bake_packed[b]);
        if (c->bake_copied[b]) cudaEventDestroy(c->bake_copied[b]);
        if (c->bake_host[b]) cudaFreeHost(c->bake_host[b]);
    }
    if (c->star_stream) {
        cudaStreamSynchronize(c->star_stream);
        cudaStreamDestroy(c->star_stream);
    }
    if (c->star_walked) cudaEventDestroy(c->star_walked);
    for (cudaEvent_t e : c->up_landed)
        if (e) cudaEventDestroy(e);
    if (c->part_stream) {
        cudaStreamSynchronize(c->part_stream);
        cudaStreamDestroy(c->part_stream);
    }
    if (c->part_fork) cudaEventDestroy(c->part_fork);
    if (c->part_join) cudaEventDestroy(c->part_join);
    if (c->gather_fork) cudaEventDestroy(c->gather_fork);
    if (c->gather_join) cudaEventDestroy(c->gather_join);
    if (c->star_flags) cudaFreeHost(c->star_flags);
    void* ptrs[] = {c->pos[0], c->pos[1], c->vel[0], c->vel[1], c->acc, c->keys[0], c->keys[1],
                    c->idx[0], c->idx[1], c->tr, c->bd, c->wn, c->com64, c->leaf_parent, c->seg_off,
                    c->seg_id, c->groups, c->supers, c->sg_list, c->sg_src, c->sg_meta, c->perm, c->chunks,
                    c->seg_bounds, c->staging, c->pb_staging,
                    c->scratch, c->status, c->diag, c->targets, c->direct_out, c->counts,
                    c->walk_stack, c->render_acc, c->render_rgba, c->star_chunk_done};
    for (void* p : ptrs)
        if (p) cudaFree(p);
}

int validate_params(gcs_ctx* c, const gcs_params* p) {
    if (!p) {
        c->last_error = "null params";
        return GCS_ERR_ARG;
    }
    if (p->leaf_size < 1 || p->leaf_size > 32) {
        c->last_error = "leaf_size must be in [1, 32]";
        return GCS_ERR_ARG;
    }
    if (p->bounds_mode != GCS_BOUNDS_CALLER && p->bounds_mode != GCS_BOUNDS_DEVICE) {
        c->last_error = "bounds_mode must be GCS_BOUNDS_CALLER or GCS_BOUNDS_DEVICE";
        return GCS_ERR_ARG;
    }
    if (!(p->theta >= 0.0f) || !(p->epsilon_sq >= 0.0f)) {
        c->last_error = "theta and epsilon_sq must be >= 0";
        return GCS_ERR_ARG;
    }
    return GCS_OK;
}

int default_walk_batch() { return 32; }

WalkNodeParams walk_node_params(const gcs_ctx* c, const gcs_params* p) {
    WalkNodeParams w;
    w.wn = c->wn;
    w.G = p->G;
    w.leaf_size = std::min(std::max(p->leaf_size, 1), 32);
    return w;
}

// Walk work units: runs of <= group_width consecutive particles that never
// straddle a segment, so a segment's groups are the same alone or batched.
// First particle and count the walk and the kick/drift cover.
int64_t range_first(const gcs_ctx* c) { return c->range_count < 0 ? 0 : std::min<int64_t>(c->range_first, c->n); }
int64_t range_count(const gcs_ctx* c) {
    const int64_t f = range_first(c);
    return c->range_count < 0 ? c->n : std::max<int64_t>(0, std::min<int64_t>(c->range_count, c->n - f));
}

// Groups per super-group for a group width: whole groups of at most
// kSuperTargets targets (at least one group).
int groups_per_super(int width) { return std::max(1, kSuperTargets / width); }

// Bisection levels that split a full super-group into its groups (0: the
// width does not halve kSuperTargets down to itself, targets stay in Morton
// order).
int split_levels(int width) {
    int levels = 0;
    for (int part = kSuperTargets; part > width; part >>= 1) ++levels;
    return (kSuperTargets >> levels) == width ? levels : 0;
}

// Whether the walk takes its targets through a partition of each super-group.
bool partitioned(const gcs_ctx* c) { return c->walk_frontier && split_levels(c->group_width) > 0; }

// A range boundary must be the end of the particles or the first particle
// of a walk group (so that no group is split between ranges) - of a
// super-group when groups take their targets through a partition of their
// super-group (so that no target moves between ranges).
bool range_boundary_ok(const gcs_ctx* c, int64_t b) {
    if (b == c->n) return true;
    const int64_t unit = partitioned(c) ? (int64_t)groups_per_super(c->group_width) * c->group_width : c->group_width;
    for (int s = 0; s < c->nseg; ++s)
        if (b >= c->h_seg_off[s] && b < c->h_seg_off[s + 1]) return (b - c->h_seg_off[s]) % unit == 0;
    return false;
}

int upload_groups(gcs_ctx* c) {
    std::vector<WalkGroup> groups;
    std::vector<SuperGroup> supers;
    groups.reserve((size_t)(c->n / c->group_width + c->nseg + 1));
    const int64_t rf = range_first(c), rl = rf + range_count(c);
    // Super-groups are aligned to the segment start and always cover all of
    // their targets, also where a step range cuts one: its box, and so its
    // frontier and every group's sums, are then the same in each slice of a
    // scenario stepped across devices as in the whole scenario.
    const int per = groups_per_super(c->group_width);
    const int64_t span = (int64_t)per * c->group_width;  // targets of a full super-group
    for (int s = 0; s < c->nseg; ++s) {
        const int64_t a = c->h_seg_off[s], e = c->h_seg_off[s + 1];
        int64_t cur = -1;  // first target of the current super-group
        for (int64_t g = a; g < e; g += c->group_width) {
            if (g < rf || g >= rl) continue;  // outside this context's step range
            WalkGroup w;
            w.start = (int32_t)g;
            w.count = (int32_t)std::min<int64_t>(c->group_width, e - g);
            w.seg = s;
            const int64_t sg_first = a + (g - a) / span * span;
            if (sg_first != cur) {
                SuperGroup sg;
                sg.start = (int32_t)sg_first;
                sg.count = (int32_t)std::min<int64_t>(span, e - sg_first);
                sg.seg = s;
                sg.pad = 0;
                supers.push_back(sg);
                cur = sg_first;
            }
            w.super = (int32_t)supers.size() - 1;
            groups.push_back(w);
        }
    }
    if (groups.size() > c->groups_cap || supers.size() > c->supers_cap) {
        c->last_error = "group table capacity exceeded";
        return GCS_ERR_CAPACITY;
    }
    cudaSetDevice(c->device);
    GCS_CUDA(c, cudaStreamSynchronize(c->stream));
    GCS_CUDA(c, cudaMemcpyAsync(c->groups, groups.data(), sizeof(WalkGroup) * groups.size(),
                                cudaMemcpyHostToDevice, c->stream));
    if (!supers.empty())
        GCS_CUDA(c, cudaMemcpyAsync(c->supers, supers.data(), sizeof(SuperGroup) * supers.size(),
                                    cudaMemcpyHostToDevice, c->stream));
    c->n_supers = (int)supers.size();
    c->n_groups = (int)groups.size();
    c->h_group_super.resize(groups.size());
    for (size_t g = 0; g < groups.size(); ++g) c->h_group_super[g] = groups[g].super;
    c->h_group_start.resize(groups.size());
    for (size_t g = 0; g < groups.size(); ++g) c->h_group_start[g] = groups[g].start;
    return GCS_OK;
}

}  // namespace

// The partition's second stream and its fork/join events, created once per
// context (before any capture of the step: build_step_graphs calls it too).
static int ensure_part_stream(gcs_ctx* c) {
    if (c->part_stream) return GCS_OK;
    cudaSetDevice(c->device);
    if (cudaStreamCreateWithFlags(&c->part_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->part_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->part_join, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->gather_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->gather_join, cudaEventDisableTiming) != cudaSuccess) {
        set_error(c, "partition stream", cudaGetLastError());
        return GCS_ERR_CUDA;
    }
    return GCS_OK;
}

// ---------------------------------------------------------------------------
// stage sequence
// ---------------------------------------------------------------------------
// The walk stage, with an optional epilogue (the fused kick/drift and Star
// records of the overlapped host step).
static int walk_stage(gcs_ctx* c, const gcs_params* p, const WalkEpilogue& ep) {
    cudaStream_t st = c->stream;
    const Layout L = layout_of(c);
    const ScratchLayout sl = scratch_layout(c->max_segments, c->n, c->nseg);
    WalkParams wp;
    wp.G = p->G;
    wp.eps2 = p->epsilon_sq;
    wp.theta2 = p->theta * p->theta;
    wp.leaf_size = p->leaf_size;
    wp.batch = p->walk_batch > 0 ? p->walk_batch : default_walk_batch();
    wp.with_potential = p->with_potential ? 1 : 0;
    const WalkNodeParams wnp = walk_node_params(c, p);
    if (c->wn_gen != c->tree_gen || c->wn_G != wnp.G || c->wn_L != wnp.leaf_size) {
        launch_walk_nodes(L, c->tr, wnp, c->status, st);
        c->wn_gen = c->tree_gen;
        c->wn_G = wnp.G;
        c->wn_L = wnp.leaf_size;
    }
    WalkFrontier fr;
    fr.supers = c->walk_frontier ? c->supers : nullptr;
    fr.n_supers = c->n_supers;
    fr.list = c->sg_list;
    fr.src = c->sg_src;
    fr.meta = c->sg_meta;
    fr.perm = partitioned(c) ? c->perm : nullptr;
    fr.split_levels = split_levels(c->group_width);
    if (fr.perm) {
        const int rc = ensure_part_stream(c);
        if (rc) return rc;
        fr.side = c->part_stream;
        fr.fork = c->part_fork;
        fr.join = c->part_join;
    }
    launch_walk(L, wp, c->pos[c->cur], c->wn, c->groups, c->n_groups, c->group_width > 32 ? 2 : 1, c->acc,
                scratch_at<uint32_t>(c, sl.walk_q), c->status, p->walk_blocks_per_sm, c->sm_count,
                c->count_walk ? c->counts : nullptr, c->walk_stack, c->walk_stack_entries, st, ep, fr);
    return check_launch(c, "walk");
}

// gather_beside_build: the gather runs on the side stream while the build
// runs on the context stream (set when both stages run in one call; the
// build stage then joins the side stream, so later stages see both).
// kick_in_walk: the walk's warps apply the kick/drift to their groups as they
// finish them (out of place, into the other particle arrays) and the
// integrate stage has nothing left to do (set when both stages run in one
// call over all particles).
static int run_stage(gcs_ctx* c, const gcs_params* p, int stage, bool gather_beside_build = false,
                     bool kick_in_walk = false) {
    cudaStream_t st = c->stream;
    const Layout L = layout_of(c);
    const int passes = kKeyPasses + seg_passes(c->nseg);
    const ScratchLayout sl = scratch_layout(c->max_segments, c->n, c->nseg);
    uint32_t* hist = scratch_at<uint32_t>(c, sl.hist);
    switch (stage) {
        case GCS_STAGE_BOUNDS: {
            if (p->bounds_mode == GCS_BOUNDS_DEVICE) {
                uint32_t* enc = scratch_at<uint32_t>(c, sl.bounds);
                GCS_CUDA(c, cudaMemsetAsync(enc, 0, sizeof(uint32_t) * 2 * (size_t)c->nseg, st));
                launch_bounds(L, c->pos[c->cur], c->chunks, c->n_chunks, enc, c->status, st);
                launch_bounds_decode(enc, c->seg_bounds, c->nseg, st);
            }
            return check_launch(c, "bounds");
        }
        case GCS_STAGE_ENCODE:
            GCS_CUDA(c, cudaMemsetAsync(hist, 0, sizeof(uint32_t) * kRadix * (size_t)passes, st));
            launch_encode(L, c->pos[c->cur], p->bounds_mode, p->global_min, p->global_max,
                          c->seg_bounds, c->keys[0], c->idx[0], hist, seg_passes(c->nseg), st);
            return check_launch(c, "encode");
        case GCS_STAGE_SORT: {
            GCS_CUDA(c, cudaMemsetAsync(c->scratch + sl.tiles, 0, sl.end - sl.tiles, st));
            for (int pass = 0; pass < passes; ++pass) {
                const int in = pass & 1;
                launch_sort_pass(L, pass, c->keys[in], c->idx[in], c->keys[in ^ 1], c->idx[in ^ 1],
                                 hist, scratch_at<uint32_t>(c, sl.tiles),
                                 scratch_at<uint32_t>(c, sl.lookback), c->status, st);
            }
            c->sorted_buf = passes & 1;
            return check_launch(c, "sort");
        }
        case GCS_STAGE_GATHER: {
            cudaStream_t gs = st;
            if (gather_beside_build && ensure_part_stream(c) == GCS_OK &&
                cudaEventRecord(c->gather_fork, st) == cudaSuccess &&
                cudaStreamWaitEvent(c->part_stream, c->gather_fork, 0) == cudaSuccess)
                gs = c->part_stream;
            launch_gather(c->idx[c->sorted_buf], c->pos[c->cur], c->vel[c->cur], c->pos[c->cur ^ 1],
                          c->vel[c->cur ^ 1], c->n, gs);
            if (gs != st) {
                GCS_CUDA(c, cudaEventRecord(c->gather_join, gs));
                c->gather_pending = true;
            }
            c->cur ^= 1;
            return check_launch(c, "gather");
        }
        case GCS_STAGE_BUILD:
            launch_build(L, c->keys[c->sorted_buf], c->tr, c->bd, c->leaf_parent, c->status, st);
            if (c->gather_pending) {  // later stages read the gathered records
                GCS_CUDA(c, cudaStreamWaitEvent(st, c->gather_join, 0));
                c->gather_pending = false;
            }
            return check_launch(c, "build");
        case GCS_STAGE_AGGREGATE: {
            const WalkNodeParams wnp = walk_node_params(c, p);
            launch_aggregate(L, c->pos[c->cur], c->tr, c->bd, c->com64, c->leaf_parent, p->com_fp64, wnp,
                             c->status, st);
            c->tree_gen++;
            c->wn_gen = c->tree_gen;
            c->wn_G = wnp.G;
            c->wn_L = wnp.leaf_size;
            return check_launch(c, "aggregate");
        }
        case GCS_STAGE_WALK: {
            if (c->walk_ev[0]) GCS_CUDA(c, record_event(c->walk_ev[0], st));
            WalkEpilogue ep;
            if (kick_in_walk) {
                ep.vel_in = c->vel[c->cur];
                ep.pos_out = c->pos[c->cur ^ 1];
                ep.vel_out = c->vel[c->cur ^ 1];
                ep.dt = p->dt;
                ep.recolor = p->recolor;
            }
            const int rc = walk_stage(c, p, ep);
            if (rc) return rc;
            if (kick_in_walk) c->cur ^= 1;  // the stepped state is in the other arrays
            if (c->walk_ev[1]) GCS_CUDA(c, record_event(c->walk_ev[1], st));
            return GCS_OK;
        }
        case GCS_STAGE_INTEGRATE: {
            if (kick_in_walk) return GCS_OK;  // the walk applied it
            const int64_t f = range_first(c);
            launch_integrate(c->pos[c->cur] + f, c->vel[c->cur] + f, c->acc + f, p->dt, p->recolor, range_count(c),
                             st);
            return check_launch(c, "integrate");
        }
        default:
            c->last_error = "unknown stage";
            return GCS_ERR_ARG;
    }
}

static int run_stages(gcs_ctx* c, const gcs_params* p, int first, int last) {
    if (!c) return GCS_ERR_ARG;
    int rc = validate_params(c, p);
    if (rc) return rc;
    if (first < GCS_STAGE_BOUNDS || last > GCS_STAGE_INTEGRATE || first > last) {
        c->last_error = "bad stage range";
        return GCS_ERR_ARG;
    }
    if (c->n <= 0) {
        c->last_error = "no particles";
        return GCS_ERR_STATE;
    }
    const bool gather_beside_build = first <= GCS_STAGE_GATHER && last >= GCS_STAGE_BUILD;
    const bool kick_in_walk = first <= GCS_STAGE_WALK && last >= GCS_STAGE_INTEGRATE && c->range_count < 0;
    for (int s = first; s <= last; ++s) {
        rc = run_stage(c, p, s, gather_beside_build, kick_in_walk);
        if (rc) return rc;
    }
    return GCS_OK;
}

int gcs::pack_to_device(gcs_ctx* c, Star* dst) {
    if (!c || !dst) return GCS_ERR_ARG;
    cudaSetDevice(c->device);
    launch_pack_stars(c->pos[c->cur], c->vel[c->cur], dst, c->n, c->stream);
    int rc = check_launch(c, "pack_to_device");
    if (rc) return rc;
    GCS_CUDA(c, cudaStreamSynchronize(c->stream));
    return GCS_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

void gcs_params_reference(gcs_params* p) {
    if (!p) return;
    memset(p, 0, sizeof *p);
    p->G = 1.0f;
    p->epsilon_sq = 10.0f;
    p->theta = 1.0f;
    p->dt = 0.01f;
    p->leaf_size = 1;
    p->bounds_mode = GCS_BOUNDS_CALLER;
    p->global_min = -10000.0f;
    p->global_max = 10000.0f;
    p->recolor = 1;
    p->com_fp64 = 0;
    p->walk_batch = 0;
    p->walk_blocks_per_sm = 0;
}

const char* gcs_status_string(int status) {
    switch (status) {
        case GCS_OK: return "ok";
        case GCS_ERR_ARG: return "invalid argument";
        case GCS_ERR_CUDA: return "CUDA runtime error";
        case GCS_ERR_NOMEM: return "out of memory";
        case GCS_ERR_CAPACITY: return "capacity exceeded";
        case GCS_ERR_DEVICE: return "device status word set";
        case GCS_ERR_STATE: return "invalid state";
        case GCS_ERR_NO_DEVICE: return "no usable CUDA device";
        default: return "unknown status";
    }
}

const char* gcs_last_error(const gcs_ctx* c) { return c ? c->last_error.c_str() : "null context"; }

static int allocate_state(gcs_ctx* c);

int gcs_create(gcs_ctx** out, int64_t capacity, int32_t max_segments, int32_t device) {
    if (!out || capacity < 1 || capacity > (int64_t)(1 << 30) - 1 || max_segments < 1 ||
        max_segments > 65536)
        return GCS_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) {
        cudaGetLastError();
        return GCS_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return GCS_ERR_NO_DEVICE;
    if (prop.major != 10) return GCS_ERR_NO_DEVICE;  // built for sm_100a only
    if (cudaSetDevice(device) != cudaSuccess) return GCS_ERR_NO_DEVICE;

    gcs_ctx* c = new gcs_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    c->capacity = capacity;
    c->max_segments = max_segments;
    int rc = allocate_state(c);
    if (rc) {
        free_all(c);
        delete c;
        return GCS_ERR_NOMEM;
    }
    cudaMemset(c->scratch, 0, c->scratch_cap);  // the walk queue starts (and stays) at zero
    cudaMemset(c->status, 0, sizeof(uint32_t));
    cudaMemset(c->wn, 0, sizeof(WalkNode) * (size_t)capacity);  // codes of unwritten records stay in range
    cudaMemset(c->acc, 0, sizeof(float4) * (size_t)capacity);
    int64_t cnt = capacity;
    rc = gcs_set_segments(c, 1, &cnt);
    if (rc) {
        free_all(c);
        delete c;
        return rc;
    }
    *out = c;
    return GCS_OK;
}

int64_t gcs_context_bytes(int64_t capacity, int32_t max_segments, int32_t device) {
    if (capacity < 1 || capacity > (int64_t)(1 << 30) - 1 || max_segments < 1 || max_segments > 65536)
        return GCS_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) {
        cudaGetLastError();
        return GCS_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) return GCS_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return GCS_ERR_NO_DEVICE;
    gcs_ctx c;
    c.device = device;
    c.sm_count = prop.multiProcessorCount;
    c.capacity = capacity;
    c.max_segments = max_segments;
    c.dry_run = true;
    allocate_state(&c);
    return (int64_t)c.device_bytes;
}

// Every device array of a context, sized for its capacity and max_segments
// (with dry_run set, only the bytes are counted).
static int allocate_state(gcs_ctx* c) {
    const int64_t capacity = c->capacity;
    const int32_t max_segments = c->max_segments;
    const size_t N = (size_t)capacity;
    // groups as narrow as kMinGroupWidth targets (the autotuner's smallest)
    const size_t max_groups = N / kMinGroupWidth + (size_t)max_segments + 1;
    c->groups_cap = max_groups;
    const size_t max_chunks = N / kChunkSize + (size_t)max_segments + 1;
    int rc = GCS_OK;
    for (int b = 0; b < 2 && !rc; ++b) {
        rc |= dalloc(c, &c->pos[b], N);
        rc |= dalloc(c, &c->vel[b], N);
        rc |= dalloc(c, &c->keys[b], N);
        rc |= dalloc(c, &c->idx[b], N);
    }
    if (!rc) rc |= dalloc(c, &c->acc, N);
    if (!rc) rc |= dalloc(c, &c->tr, N);
    if (!rc) rc |= dalloc(c, &c->bd, N);
    if (!rc) rc |= dalloc(c, &c->wn, N);
    if (!rc) rc |= dalloc(c, &c->com64, N);
    if (!rc) rc |= dalloc(c, &c->leaf_parent, N);
    if (!rc) rc |= dalloc(c, &c->seg_off, (size_t)max_segments + 1);
    if (!rc) rc |= dalloc(c, &c->seg_id, N);
    if (!rc) rc |= dalloc(c, &c->groups, max_groups);
    // super-groups: full ones hold more than kSuperTargets - kGroupSize
    // targets; a segment (or a step range within it) ends at most one
    // partial one
    const size_t max_supers = N / (size_t)(kSuperTargets - kGroupSize) + (size_t)max_segments + 1;
    c->supers_cap = max_supers;
    if (!rc) rc |= dalloc(c, &c->supers, max_supers);
    if (!rc) rc |= dalloc(c, &c->sg_list, max_supers * (size_t)kSuperCap);
    if (!rc) rc |= dalloc(c, &c->sg_src, max_supers * (size_t)kSuperSrcCap);
    if (!rc) rc |= dalloc(c, &c->sg_meta, max_supers);
    if (!rc) rc |= dalloc(c, &c->perm, N);
    if (!rc) rc |= dalloc(c, &c->chunks, max_chunks);
    if (!rc) rc |= dalloc(c, &c->seg_bounds, (size_t)max_segments);
    if (!rc) rc |= dalloc(c, &c->staging, N);
    if (!rc) rc |= dalloc(c, &c->pb_staging, N);
    if (!rc) rc |= dalloc(c, &c->status, 1);
    if (!rc) rc |= dalloc(c, &c->diag, 8);
    if (!rc) rc |= dalloc(c, &c->counts, kCountWords);
    if (!rc) {
        // enough per-warp stack regions for the largest persistent walk grid
        const int64_t gb = std::max(walk_grid_blocks((int)max_groups, 0, c->sm_count, 0),
                                    walk_grid_blocks((int)max_groups, 0, c->sm_count, 1));
        c->walk_stack_entries = walk_stack_entries(gb);
        rc |= dalloc(c, &c->walk_stack, c->walk_stack_entries);
    }
    if (!rc) {
        // worst case: every particle, the most segment-id sort passes
        c->scratch_cap = scratch_layout(max_segments, capacity, max_segments).end;
        rc |= dalloc(c, &c->scratch, c->scratch_cap);
    }
    return rc;
}

void gcs_destroy(gcs_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    else cudaDeviceSynchronize();
    free_all(c);
    delete c;
}

int gcs_set_stream(gcs_ctx* c, void* stream) {
    if (!c) return GCS_ERR_ARG;
    c->stream = reinterpret_cast<cudaStream_t>(stream);
    drop_graphs(c);
    return GCS_OK;
}

void* gcs_get_stream(const gcs_ctx* c) { return c ? reinterpret_cast<void*>(c->stream) : nullptr; }

// Segment tables for a new layout; the particle arrays are not touched.
static int apply_layout(gcs_ctx* c, int32_t num_segments, const int64_t* counts) {
    if (!c || num_segments < 1 || !counts) return GCS_ERR_ARG;
    if (num_segments > c->max_segments) {
        c->last_error = "more segments than max_segments";
        return GCS_ERR_CAPACITY;
    }
    std::vector<int64_t> off((size_t)num_segments + 1, 0);
    for (int s = 0; s < num_segments; ++s) {
        if (counts[s] < 1) {
            c->last_error = "every segment needs at least one particle";
            return GCS_ERR_ARG;
        }
        off[s + 1] = off[s] + counts[s];
    }
    if (off[num_segments] > c->capacity) {
        c->last_error = "segments exceed the context capacity";
        return GCS_ERR_CAPACITY;
    }
    const int64_t n = off[num_segments];
    std::vector<Chunk> chunks;
    for (int s = 0; s < num_segments; ++s) {
        for (int64_t g = off[s]; g < off[s + 1]; g += kChunkSize) {
            Chunk ch;
            ch.start = (int32_t)g;
            ch.count = (int32_t)std::min<int64_t>(kChunkSize, off[s + 1] - g);
            ch.seg = s;
            ch.pad = 0;
            chunks.push_back(ch);
        }
    }
    cudaSetDevice(c->device);
    // The tables are read by steps already queued on the context stream:
    // let those finish, then write the new tables in stream order (pageable
    // sources are staged before each copy call returns).
    GCS_CUDA(c, cudaStreamSynchronize(c->stream));
    GCS_CUDA(c, cudaMemcpyAsync(c->seg_off, off.data(), sizeof(int64_t) * off.size(),
                                cudaMemcpyHostToDevice, c->stream));
    launch_fill_segment_ids(c->seg_off, num_segments, c->seg_id, n, c->stream);
    int rc = check_launch(c, "fill_segment_ids");
    if (rc) return rc;
    GCS_CUDA(c, cudaMemcpyAsync(c->chunks, chunks.data(), sizeof(Chunk) * chunks.size(),
                                cudaMemcpyHostToDevice, c->stream));
    c->h_seg_off = off;
    c->h_chunk_first.clear();
    for (const Chunk& ch : chunks) c->h_chunk_first.push_back(ch.start);
    c->h_chunk_first.push_back(n);
    c->n = (int32_t)n;
    c->nseg = num_segments;
    c->n_internal = (int32_t)(n - num_segments);
    c->n_chunks = (int)chunks.size();
    c->tree_gen++;  // the tree (and its walk records) belong to the old layout
    c->range_first = 0;  // a new layout steps every particle until a range is set again
    c->range_count = -1;
    drop_graphs(c);
    return upload_groups(c);
}

int gcs_set_segments(gcs_ctx* c, int32_t num_segments, const int64_t* counts) {
    const int rc = apply_layout(c, num_segments, counts);
    if (!rc) c->cur = 0;
    return rc;
}

int gcs_relayout(gcs_ctx* c, int32_t num_segments, const int64_t* counts, const int32_t* src_segment) {
    if (!c || num_segments < 1 || !counts || !src_segment) return GCS_ERR_ARG;
    const std::vector<int64_t> old_off = c->h_seg_off;
    const int old_nseg = c->nseg;
    int64_t dst = 0;
    std::vector<int64_t> dst_off((size_t)num_segments);
    for (int s = 0; s < num_segments; ++s) {
        const int src = src_segment[s];
        if (src >= old_nseg || (src >= 0 && old_off[src + 1] - old_off[src] != counts[s])) {
            c->last_error = "relayout: a kept segment must keep its particle count";
            return GCS_ERR_ARG;
        }
        for (int t = 0; t < s; ++t)
            if (src >= 0 && src_segment[t] == src) {
                c->last_error = "relayout: a segment is kept twice";
                return GCS_ERR_ARG;
            }
        dst_off[s] = dst;
        dst += counts[s];
    }
    if (dst > c->capacity || num_segments > c->max_segments) {
        c->last_error = "relayout exceeds the context capacity";
        return GCS_ERR_CAPACITY;
    }
    cudaSetDevice(c->device);
    bool in_place = true;
    for (int s = 0; s < num_segments; ++s)
        if (src_segment[s] >= 0 && dst_off[s] != old_off[src_segment[s]]) in_place = false;
    if (in_place) return apply_layout(c, num_segments, counts);
    // kept segments move into the other ping-pong buffer at their new offsets
    const int from = c->cur, to = c->cur ^ 1;
    for (int s = 0; s < num_segments; ++s) {
        const int src = src_segment[s];
        if (src < 0) continue;
        const size_t bytes = sizeof(float4) * (size_t)counts[s];
        GCS_CUDA(c, cudaMemcpyAsync(c->pos[to] + dst_off[s], c->pos[from] + old_off[src], bytes,
                                    cudaMemcpyDeviceToDevice, c->stream));
        GCS_CUDA(c, cudaMemcpyAsync(c->vel[to] + dst_off[s], c->vel[from] + old_off[src], bytes,
                                    cudaMemcpyDeviceToDevice, c->stream));
    }
    const int rc = apply_layout(c, num_segments, counts);
    if (rc) return rc;
    c->cur = to;
    return GCS_OK;
}

int64_t gcs_segment_offset(const gcs_ctx* c, int32_t segment) {
    if (!c || segment < 0 || segment > c->nseg) return -1;
    return c->h_seg_off[segment];
}

int gcs_set_group_width(gcs_ctx* c, int32_t width) {
    if (!c || width < kMinGroupWidth || width > kGroupSize) return GCS_ERR_ARG;
    const int32_t old = c->group_width;
    c->group_width = width;
    if (c->range_count >= 0 &&
        (!range_boundary_ok(c, c->range_first) || !range_boundary_ok(c, c->range_first + c->range_count))) {
        c->group_width = old;
        c->last_error = "group width would split a walk group across the step range";
        return GCS_ERR_STATE;
    }
    drop_graphs(c);
    return upload_groups(c);
}

int32_t gcs_group_width(const gcs_ctx* c) { return c ? c->group_width : 0; }

int gcs_set_walk_frontier(gcs_ctx* c, int32_t enable) {
    if (!c) return GCS_ERR_ARG;
    const bool old = c->walk_frontier;
    c->walk_frontier = enable != 0;
    if (c->range_count >= 0 &&
        (!range_boundary_ok(c, c->range_first) || !range_boundary_ok(c, c->range_first + c->range_count))) {
        c->walk_frontier = old;
        c->last_error = "walk frontiers partition super-groups that the step range would split";
        return GCS_ERR_STATE;
    }
    if (old != c->walk_frontier) drop_graphs(c);
    return GCS_OK;
}

int64_t gcs_num_particles(const gcs_ctx* c) { return c ? c->n : 0; }
int32_t gcs_num_segments(const gcs_ctx* c) { return c ? c->nseg : 0; }
int64_t gcs_num_internal_nodes(const gcs_ctx* c) { return c ? c->n_internal : 0; }
int64_t gcs_device_bytes(const gcs_ctx* c) { return c ? (int64_t)c->device_bytes : 0; }

int gcs_upload_stars(gcs_ctx* c, const Star* host, int64_t offset, int64_t n) {
    if (!c || !host || offset < 0 || n < 0 || offset + n > c->n) return GCS_ERR_ARG;
    if (n == 0) return GCS_OK;
    cudaSetDevice(c->device);
    GCS_CUDA(c, cudaMemcpyAsync(c->staging + offset, host, sizeof(Star) * (size_t)n,
                                cudaMemcpyHostToDevice, c->stream));
    launch_unpack_stars(c->staging + offset, c->pos[c->cur] + offset, c->vel[c->cur] + offset, n,
                        c->stream);
    int rc = check_launch(c, "unpack");
    if (rc) return rc;
    GCS_CUDA(c, cudaStreamSynchronize(c->stream));
    return GCS_OK;
}

int gcs_download_stars(gcs_ctx* c, Star* host, int64_t offset, int64_t n) {
    if (!c || !host || offset < 0 || n < 0 || offset + n > c->n) return GCS_ERR_ARG;
    if (n == 0) return GCS_OK;
    cudaSetDevice(c->device);
    launch_pack_stars(c->pos[c->cur] + offset, c->vel[c->cur] + offset, c->staging + offset, n,
                      c->stream);
    int rc = check_launch(c, "pack");
    if (rc) return rc;
    GCS_CUDA(c, cudaMemcpyAsync(host, c->staging + offset, sizeof(Star) * (size_t)n,
                                cudaMemcpyDeviceToHost, c->stream));
    GCS_CUDA(c, cudaStreamSynchronize(c->stream));
    return GCS_OK;
}

int gcs_download_playback(gcs_ctx* c, PlaybackStar* host, int64_t offset, int64_t n) {
    if (!c || !host || offset < 0 || n < 0 || offset + n > c->n) return GCS_ERR_ARG;
    if (n == 0) return GCS_OK;
    cudaSetDevice(c->device);
    launch_pack_playback(c->pos[c->cur] + offset, c->vel[c->cur] + offset, c->pb_staging + offset,
                         n, c->stream);
    int rc = check_launch(c, "pack_playback");
    if (rc) return rc;
    GCS_CUDA(c, cudaMemcpyAsync(host, c->pb_staging + offset, sizeof(PlaybackStar) * (size_t)n,
                                cudaMemcpyDeviceToHost, c->stream));
    GCS_CUDA(c, cudaStreamSynchronize(c->stream));
    return GCS_OK;
}

// Capture the full step twice, once from each ping-pong parity of the
// particle arrays, into executable graphs.  The stage launches are the ones
// an eager step makes; capture runs on the context stream in thread-local
// mode, so other threads' CUDA calls are unaffected.
static int build_step_graphs(gcs_ctx* c, const gcs_params* p) {
    drop_graphs(c);
    const int cur0 = c->cur;
    int rc = ensure_part_stream(c);  // created outside the capture
    if (rc) return rc;
    for (int k = 0; k < 2 && !rc; ++k) {
        const int parity = cur0 ^ k;
        c->cur = parity;
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            c->last_error = "cudaStreamBeginCapture failed";
            rc = GCS_ERR_CUDA;
            break;
        }
        rc = run_stages(c, p, GCS_STAGE_BOUNDS, GCS_STAGE_INTEGRATE);
        c->graph_after[parity] = c->cur;
        const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
        if (!rc && e != cudaSuccess) {
            set_error(c, "cudaStreamEndCapture", e);
            rc = GCS_ERR_CUDA;
        }
        if (!rc) {
            const cudaError_t ei = cudaGraphInstantiate(&c->graph_exec[parity], graph, 0);
            if (ei != cudaSuccess) {
                set_error(c, "cudaGraphInstantiate", ei);
                rc = GCS_ERR_CUDA;
            }
        }
        if (!rc && (c->walk_ev[0] || c->walk_ev[1])) {
            // the event-record nodes of the caller's walk events
            size_t count = 0;
            if (cudaGraphGetNodes(graph, nullptr, &count) == cudaSuccess && count > 0) {
                std::vector<cudaGraphNode_t> nodes(count);
                if (cudaGraphGetNodes(graph, nodes.data(), &count) == cudaSuccess) {
                    for (size_t i = 0; i < count; ++i) {
                        cudaGraphNodeType type;
                        cudaEvent_t ev = nullptr;
                        if (cudaGraphNodeGetType(nodes[i], &type) != cudaSuccess ||
                            type != cudaGraphNodeTypeEventRecord ||
                            cudaGraphEventRecordNodeGetEvent(nodes[i], &ev) != cudaSuccess)
                            continue;
                        for (int e = 0; e < 2; ++e)
                            if (ev && ev == c->walk_ev[e]) {
                                c->walk_ev_node[parity][e] = nodes[i];
                                c->walk_ev_bound[parity][e] = ev;
                            }
                    }
                }
            }
            for (int e = 0; e < 2; ++e)
                if (c->walk_ev[e] && !c->walk_ev_node[parity][e]) {
                    c->last_error = "walk event node missing from the captured step";
                    rc = GCS_ERR_CUDA;
                }
        }
        c->graph[parity] = graph;  // destroyed with the exec graphs
    }
    c->cur = cur0;
    if (rc) {
        drop_graphs(c);
        cudaGetLastError();
        return rc;
    }
    c->graph_params = *p;
    c->graph_stream = c->stream;
    c->graphs_valid = true;
    ++c->graph_builds;
    return GCS_OK;
}

int gcs_step(gcs_ctx* c, const gcs_params* p) {
    if (!c) return GCS_ERR_ARG;
    if (!c->use_graphs) return run_stages(c, p, GCS_STAGE_BOUNDS, GCS_STAGE_INTEGRATE);
    int rc = validate_params(c, p);
    if (rc) return rc;
    if (c->n <= 0) {
        c->last_error = "no particles";
        return GCS_ERR_STATE;
    }
    if (!c->graphs_valid || c->graph_stream != c->stream ||
        memcmp(&c->graph_params, p, sizeof(gcs_params)) != 0) {
        rc = build_step_graphs(c, p);
        if (rc) return rc;
    }
    cudaSetDevice(c->device);
    for (int e = 0; e < 2; ++e) {
        // point the graph's walk-event nodes at the events set now
        cudaGraphNode_t node = c->walk_ev_node[c->cur][e];
        if (node && c->walk_ev[e] && c->walk_ev_bound[c->cur][e] != c->walk_ev[e]) {
            GCS_CUDA(c, cudaGraphExecEventRecordNodeSetEvent(c->graph_exec[c->cur], node, c->walk_ev[e]));
            c->walk_ev_bound[c->cur][e] = c->walk_ev[e];
        }
    }
    GCS_CUDA(c, cudaGraphLaunch(c->graph_exec[c->cur], c->stream));
    c->cur = c->graph_after[c->cur];  // the flips the captured step made (gather, kick/drift in the walk)
    c->sorted_buf = (kKeyPasses + seg_passes(c->nseg)) & 1;
    return GCS_OK;
}

int gcs_set_walk_events(gcs_ctx* c, void* start, void* end) {
    if (!c) return GCS_ERR_ARG;
    cudaEvent_t ev[2] = {static_cast<cudaEvent_t>(start), static_cast<cudaEvent_t>(end)};
    // graphs hold event-record nodes only for events present at capture
    if ((ev[0] != nullptr) != (c->walk_ev[0] != nullptr) || (ev[1] != nullptr) != (c->walk_ev[1] != nullptr))
        drop_graphs(c);
    c->walk_ev[0] = ev[0];
    c->walk_ev[1] = ev[1];
    return GCS_OK;
}

int gcs_set_graphs(gcs_ctx* c, int32_t enable) {
    if (!c) return GCS_ERR_ARG;
    if (enable && c->stream == nullptr) {
        c->last_error = "graph capture needs a non-default stream (gcs_set_stream)";
        return GCS_ERR_STATE;
    }
    c->use_graphs = enable != 0;
    if (!c->use_graphs) drop_graphs(c);
    return GCS_OK;
}

int32_t gcs_graph_builds(const gcs_ctx* c) { return c ? c->graph_builds : 0; }

// The device address of the `bytes` at host pointer p when all of them lie in
// one pinned, device-mapped host allocation (cudaMallocHost, cudaHostAlloc,
// cudaHostRegister with UVA), 16-byte aligned; nullptr otherwise.  The range
// comes from the driver (cuPointerGetAttribute, RANGE_START_ADDR / _SIZE),
// fetched through the runtime's entry-point query, so the library does not
// link the driver library.
static void* mapped_host_range(const void* p, size_t bytes) {
    using GetAttr = CUresult (*)(void*, CUpointer_attribute, CUdeviceptr);
    static GetAttr get_attr = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuPointerGetAttribute", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_attr = reinterpret_cast<GetAttr>(f);
        cudaGetLastError();
    });
    if (!p || !get_attr) return nullptr;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // not memory the runtime knows: pageable
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost || !a.devicePointer) return nullptr;
    const CUdeviceptr d = reinterpret_cast<CUdeviceptr>(a.devicePointer);
    CUdeviceptr start = 0;
    size_t size = 0;
    if (get_attr(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, d) != CUDA_SUCCESS ||
        get_attr(&size, CU_POINTER_ATTRIBUTE_RANGE_SIZE, d) != CUDA_SUCCESS)
        return nullptr;
    if (d < start || d - start > size || bytes > size - (d - start) || (d & 15u)) return nullptr;
    return a.devicePointer;
}

// Resources of the overlapped host step, created at its first use.
static int ensure_star_pipeline(gcs_ctx* c) {
    if (!c->star_stream) GCS_CUDA(c, cudaStreamCreateWithFlags(&c->star_stream, cudaStreamNonBlocking));
    if (!c->star_walked) GCS_CUDA(c, cudaEventCreateWithFlags(&c->star_walked, cudaEventDisableTiming));
    for (cudaEvent_t& e : c->up_landed)
        if (!e) GCS_CUDA(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    if (!c->star_flags) {
        GCS_CUDA(c, cudaHostAlloc(reinterpret_cast<void**>(&c->star_flags), sizeof(uint32_t) * kMaxStarChunks,
                                  cudaHostAllocMapped));
        memset(c->star_flags, 0, sizeof(uint32_t) * kMaxStarChunks);
        GCS_CUDA(c, cudaHostGetDevicePointer(reinterpret_cast<void**>(&c->star_flags_dev), c->star_flags, 0));
    }
    if (!c->star_chunk_done) {
        const int rc = dalloc(c, &c->star_chunk_done, kMaxStarChunks);
        if (rc) return rc;
    }
    return GCS_OK;
}

// One step whose Stars land in `host`, with the transfer overlapped with the
// walk: the walk's epilogue applies the kick/drift out of place and writes
// each group's Star records, straight into `host` when it is pinned and
// device-mapped, else into device staging, from which the host copies every
// chunk of groups as soon as its flag arrives.  Groups handed out before the work queue runs dry go
// in up to kMaxStarHeadChunks large chunks; the last groups (twice the
// walk's resident warps, one group each) are all in flight at the end and
// finish together, so they go in up to kMaxStarTailChunks small chunks whose
// completions, and copies, spread over the walk's last phase.  The result is the
// same bits as the plain stage sequence followed by gcs_download_stars.  A
// step range (one slice of the scenario) takes that plain sequence.
static int step_host_overlapped(gcs_ctx* c, const gcs_params* p, Star* host, int first_stage = GCS_STAGE_BOUNDS) {
    int rc = run_stages(c, p, first_stage, GCS_STAGE_AGGREGATE);
    if (rc) return rc;
    // A pinned, device-mapped host array: the epilogue writes each group's
    // Stars straight into it over PCIe while the walk goes on (no copies, no
    // flags); the stream's completion makes them visible to the host.
    void* direct = mapped_host_range(host, sizeof(Star) * (size_t)c->n);
    if (direct) {
        WalkEpilogue ep;
        ep.vel_in = c->vel[c->cur];
        ep.pos_out = c->pos[c->cur ^ 1];
        ep.vel_out = c->vel[c->cur ^ 1];
        ep.stars = reinterpret_cast<float4*>(direct);
        ep.dt = p->dt;
        ep.recolor = p->recolor;
        rc = walk_stage(c, p, ep);
        if (rc) return rc;
        c->cur ^= 1;  // the epilogue wrote the stepped state into the other arrays
        GCS_CUDA(c, cudaStreamSynchronize(c->stream));
        return GCS_OK;
    }
    rc = ensure_star_pipeline(c);
    if (rc) return rc;
    const int ng = c->n_groups;
    const int64_t resident = walk_grid_blocks(ng, p->walk_blocks_per_sm, c->sm_count, p->with_potential) *
                             (int64_t)kWalkBlockWarps;
    const int tail_groups = (int)std::min<int64_t>(ng, 2 * resident);
    const int head_groups = ng - tail_groups;
    const int hpc = head_groups > 0 ? (head_groups + kMaxStarHeadChunks - 1) / kMaxStarHeadChunks : 1;
    const int tpc = (tail_groups + kMaxStarTailChunks - 1) / kMaxStarTailChunks;
    // chunk boundaries (group indices): large chunks over the head, small
    // ones over the tail; with partitioned super-groups each boundary moves
    // up to the next super-group edge, so a chunk's particles stay one range
    std::vector<int32_t> bound;
    bound.push_back(0);
    const bool snap = partitioned(c);
    auto add_bound = [&](int g) {
        if (snap)
            while (g < ng && g > 0 && c->h_group_super[(size_t)g] == c->h_group_super[(size_t)g - 1]) ++g;
        if (g > bound.back()) bound.push_back(g);
    };
    for (int g = hpc; g < head_groups; g += hpc) add_bound(g);
    add_bound(head_groups);
    for (int g = head_groups + tpc; g < ng; g += tpc) add_bound(g);
    add_bound(ng);
    const int chunks = (int)bound.size() - 1;
    if (chunks < 1 || chunks > kMaxStarChunks) {
        c->last_error = "host step: chunk table out of range";
        return GCS_ERR_STATE;
    }
    if (++c->star_epoch == 0) c->star_epoch = 1;
    const uint32_t epoch = c->star_epoch;
    GCS_CUDA(c, cudaMemsetAsync(c->star_chunk_done, 0, sizeof(uint32_t) * (size_t)chunks, c->stream));
    WalkEpilogue ep;
    ep.vel_in = c->vel[c->cur];
    ep.pos_out = c->pos[c->cur ^ 1];
    ep.vel_out = c->vel[c->cur ^ 1];
    ep.stars = reinterpret_cast<float4*>(c->staging);
    ep.dt = p->dt;
    ep.recolor = p->recolor;
    ep.n_chunks = chunks;
    for (int k = 0; k <= chunks; ++k) ep.chunk_bound[k] = bound[(size_t)k];
    ep.chunk_done = c->star_chunk_done;
    ep.host_flags = c->star_flags_dev;
    ep.epoch = epoch;
    rc = walk_stage(c, p, ep);
    if (rc) return rc;
    c->cur ^= 1;  // the epilogue wrote the stepped state into the other arrays
    GCS_CUDA(c, cudaEventRecord(c->star_walked, c->stream));
    // Copy each chunk once its flag is up; when the walk has finished, copy
    // what is left (a chunk that was never signalled is reported).
    bool missing = false;
    for (int k = 0; k < chunks && !rc; ++k) {
        const int g0 = bound[(size_t)k], g1 = bound[(size_t)k + 1];
        const int64_t first = c->h_group_start[(size_t)g0];
        const int64_t end = g1 < ng ? c->h_group_start[(size_t)g1] : c->n;
        for (uint32_t polls = 1;; ++polls) {
            if (__atomic_load_n(c->star_flags + k, __ATOMIC_ACQUIRE) == epoch) break;
            if ((polls & 63u) == 0u) {
                const cudaError_t q = cudaEventQuery(c->star_walked);
                if (q == cudaSuccess) {
                    if (__atomic_load_n(c->star_flags + k, __ATOMIC_ACQUIRE) != epoch) missing = true;
                    break;
                }
                if (q != cudaErrorNotReady) {
                    set_error(c, "walk", q);
                    rc = GCS_ERR_CUDA;
                    break;
                }
            }
        }
        if (rc) break;
        const cudaError_t e = cudaMemcpyAsync(host + first, c->staging + first, sizeof(Star) * (size_t)(end - first),
                                              cudaMemcpyDeviceToHost, c->star_stream);
        if (e != cudaSuccess) {
            set_error(c, "cudaMemcpyAsync (Stars)", e);
            rc = GCS_ERR_CUDA;
        }
    }
    // no copy into the caller's buffer may outlive this call
    const cudaError_t e1 = cudaStreamSynchronize(c->star_stream);
    const cudaError_t e2 = cudaStreamSynchronize(c->stream);
    if (rc) return rc;
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
        set_error(c, "cudaStreamSynchronize (host step)", e1 != cudaSuccess ? e1 : e2);
        return GCS_ERR_CUDA;
    }
    if (missing) {
        c->last_error = "host step: a chunk of Star records was not signalled by the walk";
        return GCS_ERR_STATE;
    }
    return GCS_OK;
}

// One step from host Stars to host Stars.  The upload goes in up to 8 chunks
// (whole bounds chunks) on the copy stream; the context stream unpacks each
// chunk, and reduces it into the segment bounds when the bounds come from
// the device, as soon as it has landed, so the PCIe copy overlaps that work
// and no host synchronisation separates the upload from the step; the rest
// is gcs_step_host's step (Stars back while the walk runs).
int gcs_step_host_io(gcs_ctx* c, const gcs_params* p, const Star* in, Star* out) {
    if (!c || !in || !out) return GCS_ERR_ARG;
    cudaSetDevice(c->device);
    int rc = validate_params(c, p);
    if (rc) return rc;
    if (c->range_count >= 0 || c->n_groups <= 0 || c->n <= 0 || c->n_chunks <= 0) {
        rc = gcs_upload_stars(c, in, 0, c->n);
        return rc ? rc : gcs_step_host(c, p, out);
    }
    rc = ensure_star_pipeline(c);
    if (rc) return rc;
    const bool device_bounds = p->bounds_mode == GCS_BOUNDS_DEVICE;
    const Layout L = layout_of(c);
    const ScratchLayout sl = scratch_layout(c->max_segments, c->n, c->nseg);
    uint32_t* enc = scratch_at<uint32_t>(c, sl.bounds);
    if (device_bounds) GCS_CUDA(c, cudaMemsetAsync(enc, 0, sizeof(uint32_t) * 2 * (size_t)c->nseg, c->stream));
    // the copy stream starts after everything queued so far (the previous
    // step may still be reading the staging buffer and the particle arrays)
    GCS_CUDA(c, cudaEventRecord(c->up_landed[0], c->stream));
    GCS_CUDA(c, cudaStreamWaitEvent(c->star_stream, c->up_landed[0], 0));
    constexpr int kUpChunks = (int)(sizeof(c->up_landed) / sizeof(c->up_landed[0]));
    const int per = (c->n_chunks + kUpChunks - 1) / kUpChunks;
    for (int u = 0, e0 = 0; e0 < c->n_chunks; ++u, e0 += per) {
        const int e1 = std::min(e0 + per, c->n_chunks);
        const int64_t a = c->h_chunk_first[(size_t)e0], b = c->h_chunk_first[(size_t)e1];
        GCS_CUDA(c, cudaMemcpyAsync(c->staging + a, in + a, sizeof(Star) * (size_t)(b - a), cudaMemcpyHostToDevice,
                                    c->star_stream));
        GCS_CUDA(c, cudaEventRecord(c->up_landed[u], c->star_stream));
        GCS_CUDA(c, cudaStreamWaitEvent(c->stream, c->up_landed[u], 0));
        launch_unpack_stars(c->staging + a, c->pos[c->cur] + a, c->vel[c->cur] + a, b - a, c->stream);
        if (device_bounds) launch_bounds(L, c->pos[c->cur], c->chunks + e0, e1 - e0, enc, c->status, c->stream);
        rc = check_launch(c, "upload chunk");
        if (rc) return rc;
    }
    if (device_bounds) {
        launch_bounds_decode(enc, c->seg_bounds, c->nseg, c->stream);
        rc = check_launch(c, "bounds");
        if (rc) return rc;
    }
    return step_host_overlapped(c, p, out, GCS_STAGE_ENCODE);
}

int gcs_step_host(gcs_ctx* c, const gcs_params* p, Star* host) {
    if (!c || !host) return GCS_ERR_ARG;
    cudaSetDevice(c->device);
    if (c->range_count < 0 && c->n_groups > 0 && c->n > 0)
        return step_host_overlapped(c, p, host);
    int rc = run_stages(c, p, GCS_STAGE_BOUNDS, GCS_STAGE_INTEGRATE);
    if (rc) return rc;
    return gcs_download_stars(c, host, 0, c->n);
}

int gcs_compute_accels(gcs_ctx* c, const gcs_params* p) {
    if (!c) return GCS_ERR_ARG;
    return run_stages(c, p, GCS_STAGE_BOUNDS, GCS_STAGE_WALK);
}

int gcs_kick(gcs_ctx* c, float dt) {
    if (!c) return GCS_ERR_ARG;
    const int64_t f = range_first(c);
    launch_kick(c->vel[c->cur] + f, c->acc + f, dt, range_count(c), c->stream);
    return check_launch(c, "kick");
}

int gcs_set_step_range(gcs_ctx* c, int64_t first, int64_t count) {
    if (!c) return GCS_ERR_ARG;
    if (count < 0) {
        c->range_first = 0;
        c->range_count = -1;
    } else {
        if (first < 0 || first > c->n || count > c->n - first || !range_boundary_ok(c, first) ||
            !range_boundary_ok(c, first + count)) {
            c->last_error = "step range: bounds must be walk-group starts within the particles";
            return GCS_ERR_ARG;
        }
        c->range_first = first;
        c->range_count = count;
    }
    drop_graphs(c);
    return upload_groups(c);
}

void* gcs_device_array(gcs_ctx* c, int32_t which) {
    if (!c) return nullptr;
    switch (which) {
        case GCS_BUF_POS: return c->pos[c->cur];
        case GCS_BUF_VEL: return c->vel[c->cur];
        case GCS_BUF_ACCEL: return c->acc;
        default: return nullptr;
    }
}

int gcs_run_stages(gcs_ctx* c, const gcs_params* p, int32_t first, int32_t last) {
    return run_stages(c, p, first, last);
}

int gcs_device_status(gcs_ctx* c, uint32_t* status, int32_t clear) {
    if (!c || !status) return GCS_ERR_ARG;
    cudaSetDevice(c->device);
    GCS_CUDA(c, cudaStreamSynchronize(c->stream));
    GCS_CUDA(c, cudaMemcpy(status, c->status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (clear) GCS_CUDA(c, cudaMemsetAsync(c->status, 0, sizeof(uint32_t), c->stream));
    return GCS_OK;
}

int gcs_synchronize(gcs_ctx* c) {
    uint32_t s = 0;
    int rc = gcs_device_status(c, &s, 0);
    if (rc) return rc;
    if (s) {
        char buf[96];
        snprintf(buf, sizeof buf, "device status word 0x%x", s);
        c->last_error = buf;
        return GCS_ERR_DEVICE;
    }
    return GCS_OK;
}

int gcs_read_buffer(gcs_ctx* c, int32_t which, void* host, int64_t first, int64_t count) {
    if (!c || !host || first < 0 || count < 0) return GCS_ERR_ARG;
    const void* src = nullptr;
    size_t elem = 0;
    int64_t limit = 0;
    switch (which) {
        case GCS_BUF_KEYS: src = c->keys[c->sorted_buf]; elem = 8; limit = c->n; break;
        case GCS_BUF_INDEX: src = c->idx[c->sorted_buf]; elem = 4; limit = c->n; break;
        case GCS_BUF_NODES: src = c->tr; elem = sizeof(BvhNodeTraverse); limit = c->n_internal; break;
        case GCS_BUF_BUILD: src = c->bd; elem = sizeof(BvhNodeBuild); limit = c->n_internal; break;
        case GCS_BUF_LEAF_PARENT: src = c->leaf_parent; elem = 4; limit = c->n; break;
        case GCS_BUF_ACCEL: src = c->acc; elem = 16; limit = c->n; break;
        case GCS_BUF_POS: src = c->pos[c->cur]; elem = 16; limit = c->n; break;
        case GCS_BUF_VEL: src = c->vel[c->cur]; elem = 16; limit = c->n; break;
        case GCS_BUF_BOUNDS: src = c->seg_bounds; elem = 8; limit = c->nseg; break;
        case GCS_BUF_KEYS_UNSORTED: src = c->keys[0]; elem = 8; limit = c->n; break;
        default: return GCS_ERR_ARG;
    }
    if (first + count > limit) return GCS_ERR_ARG;
    if (count == 0) return GCS_OK;
    cudaSetDevice(c->device);
    GCS_CUDA(c, cudaStreamSynchronize(c->stream));
    GCS_CUDA(c, cudaMemcpy(host, static_cast<const char*>(src) + elem * (size_t)first,
                           elem * (size_t)count, cudaMemcpyDeviceToHost));
    return GCS_OK;
}

int gcs_diagnostics(gcs_ctx* c, int32_t segment, double out[6]) {
    return gcs_diagnostics_kicked(c, segment, 0.0, out);
}

int gcs_diagnostics_kicked(gcs_ctx* c, int32_t segment, double kick, double out[6]) {
    if (!c || !out || segment < 0 || segment >= c->nseg) return GCS_ERR_ARG;
    cudaSetDevice(c->device);
    const int64_t first = c->h_seg_off[segment];
    const int64_t n = c->h_seg_off[segment + 1] - first;
    GCS_CUDA(c, cudaMemsetAsync(c->diag, 0, sizeof(double) * 6, c->stream));
    launch_diag(c->pos[c->cur], c->vel[c->cur], c->acc, first, n, kick, c->diag, c->stream);
    int rc = check_launch(c, "diag");
    if (rc) return rc;
    GCS_CUDA(c, cudaMemcpyAsync(out, c->diag, sizeof(double) * 6, cudaMemcpyDeviceToHost, c->stream));
    GCS_CUDA(c, cudaStreamSynchronize(c->stream));
    return GCS_OK;
}

int gcs_count_interactions(gcs_ctx* c, const gcs_params* p, uint64_t out[8]) {
    if (!c || !p || !out) return GCS_ERR_ARG;
    cudaSetDevice(c->device);
    GCS_CUDA(c, cudaMemsetAsync(c->counts, 0, kCountWords * sizeof(unsigned long long), c->stream));
    c->count_walk = true;
    const int rc = run_stages(c, p, GCS_STAGE_BOUNDS, GCS_STAGE_WALK);
    c->count_walk = false;
    if (rc) return rc;
    GCS_CUDA(c, cudaMemcpyAsync(out, c->counts, 8 * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                c->stream));
    GCS_CUDA(c, cudaStreamSynchronize(c->stream));
    return GCS_OK;
}

int gcs_walk_stack_peak(gcs_ctx* c, int64_t out[2]) {
    if (!c || !out) return GCS_ERR_ARG;
    cudaSetDevice(c->device);
    uint64_t peak = 0;
    GCS_CUDA(c, cudaMemcpyAsync(&peak, c->counts + 8, sizeof peak, cudaMemcpyDeviceToHost, c->stream));
    GCS_CUDA(c, cudaStreamSynchronize(c->stream));
    out[0] = (int64_t)peak;
    out[1] = kWalkGlobalStack;
    return GCS_OK;
}

int gcs_walk_lane_use(gcs_ctx* c, uint64_t out[8]) {
    if (!c || !out) return GCS_ERR_ARG;
    cudaSetDevice(c->device);
    GCS_CUDA(c, cudaMemcpyAsync(out, c->counts + 9, 8 * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream));
    GCS_CUDA(c, cudaStreamSynchronize(c->stream));
    return GCS_OK;
}

int gcs_autotune(gcs_ctx* c, gcs_params* p, double* best_walk_ms) {
    if (!c || !p) return GCS_ERR_ARG;
    int rc = run_stages(c, p, GCS_STAGE_BOUNDS, GCS_STAGE_AGGREGATE);
    if (rc) return rc;
    cudaSetDevice(c->device);
    cudaEvent_t e0, e1;
    GCS_CUDA(c, cudaEventCreate(&e0));
    GCS_CUDA(c, cudaEventCreate(&e1));
    const int widths[] = {64, 32, 16};
    const int leaves[] = {1, 2, 4, 8, 16, 32};
    const int batches[] = {16, 32, 64};
    const int occupancy[] = {0, 4};
    gcs_params best = *p;
    int best_width = c->group_width;
    float best_ms = 3.0e38f;
    for (int gw : widths) {
        rc = gcs_set_group_width(c, gw);
        if (rc) break;
        for (int L : leaves) {
            if (L > p->leaf_size || L < p->tune_leaf_min) continue;
            for (int b : batches) {
                for (int occ : occupancy) {
                    gcs_params q = *p;
                    q.leaf_size = L;
                    q.walk_batch = b;
                    q.walk_blocks_per_sm = occ;
                    if ((rc = run_stage(c, &q, GCS_STAGE_WALK))) break;  // warm
                    cudaEventRecord(e0, c->stream);
                    for (int r = 0; r < 2 && !rc; ++r) rc = run_stage(c, &q, GCS_STAGE_WALK);
                    cudaEventRecord(e1, c->stream);
                    if (rc) break;
                    cudaEventSynchronize(e1);
                    float ms = 0.0f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    ms *= 0.5f;
                    if (ms < best_ms) {
                        best_ms = ms;
                        best = q;
                        best_width = gw;
                    }
                }
                if (rc) break;
            }
            if (rc) break;
        }
        if (rc) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    rc = gcs_set_group_width(c, best_width);
    if (rc) return rc;
    *p = best;
    if (best_walk_ms) *best_walk_ms = best_ms;
    return gcs_synchronize(c);
}

int gcs_direct_accels_fp64(gcs_ctx* c, const gcs_params* p, int32_t segment,
                           const int64_t* targets, int64_t n_targets, double* out) {
    if (!c || !p || !targets || !out || segment < 0 || segment >= c->nseg || n_targets < 0)
        return GCS_ERR_ARG;
    if (n_targets == 0) return GCS_OK;
    const int64_t first = c->h_seg_off[segment];
    const int64_t n = c->h_seg_off[segment + 1] - first;
    for (int64_t i = 0; i < n_targets; ++i)
        if (targets[i] < 0 || targets[i] >= n) return GCS_ERR_ARG;
    cudaSetDevice(c->device);
    if (n_targets > c->targets_cap) {
        if (c->targets) cudaFree(c->targets);
        if (c->direct_out) cudaFree(c->direct_out);
        c->targets = nullptr;
        c->direct_out = nullptr;
        c->targets_cap = 0;
        if (dalloc(c, &c->targets, (size_t)n_targets) || dalloc(c, &c->direct_out, 3 * (size_t)n_targets))
            return GCS_ERR_NOMEM;
        c->targets_cap = n_targets;
    }
    GCS_CUDA(c, cudaMemcpyAsync(c->targets, targets, sizeof(int64_t) * (size_t)n_targets,
                                cudaMemcpyHostToDevice, c->stream));
    launch_direct_fp64(c->pos[c->cur], first, n, c->targets, n_targets, (double)p->G,
                       (double)p->epsilon_sq, c->direct_out, c->stream);
    int rc = check_launch(c, "direct_fp64");
    if (rc) return rc;
    GCS_CUDA(c, cudaMemcpyAsync(out, c->direct_out, sizeof(double) * 3 * (size_t)n_targets,
                                cudaMemcpyDeviceToHost, c->stream));
    GCS_CUDA(c, cudaStreamSynchronize(c->stream));
    return GCS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// headless point-splat renderer (renderer.cpp:97-148, 202-204, 248, 262-263)
// ---------------------------------------------------------------------------
extern "C" {

void gcs_camera_reference(gcs_camera* cam) {
    if (!cam) return;
    const float pos[3] = {0.0f, 150.0f, 600.0f}, front[3] = {0.0f, -0.2f, -1.0f}, up[3] = {0.0f, 1.0f, 0.0f};
    for (int k = 0; k < 3; ++k) {
        cam->pos[k] = pos[k];
        cam->front[k] = front[k];
        cam->up[k] = up[k];
    }
    cam->fovy_deg = 45.0f;
    cam->z_near = 0.1f;
    cam->z_far = 5000.0f;
}

int gcs_camera_look_at(gcs_camera* cam, const float target[3]) {
    if (!cam || !target) return GCS_ERR_ARG;
    const float d[3] = {target[0] - cam->pos[0], target[1] - cam->pos[1], target[2] - cam->pos[2]};
    const float len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (!(len > 0.0f) || !std::isfinite(len)) return GCS_ERR_ARG;
    for (int k = 0; k < 3; ++k) cam->front[k] = d[k] * (1.0f / len);
    return GCS_OK;
}

// View = lookAt(eye, eye + front, up): rows s, u, -f (s = normalize(f x up),
// u = s x f, f = normalize(front)) with translations -s.eye, -u.eye, f.eye.
// Proj = perspective(fovy, aspect, near, far), OpenGL clip depth [-1, 1].
// Formed in double, stored as float.
int gcs_camera_matrices(const gcs_camera* cam, int32_t width, int32_t height, float view[16], float proj[16]) {
    if (!cam || !view || !proj || width < 1 || height < 1) return GCS_ERR_ARG;
    if (!(cam->fovy_deg > 0.0f && cam->fovy_deg < 180.0f) || !(cam->z_near > 0.0f) ||
        !(cam->z_far > cam->z_near))
        return GCS_ERR_ARG;
    double f[3] = {cam->front[0], cam->front[1], cam->front[2]};
    const double fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    if (!(fl > 0.0)) return GCS_ERR_ARG;
    for (double& x : f) x /= fl;
    const double up[3] = {cam->up[0], cam->up[1], cam->up[2]};
    double sv[3] = {f[1] * up[2] - f[2] * up[1], f[2] * up[0] - f[0] * up[2], f[0] * up[1] - f[1] * up[0]};
    const double sl = std::sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
    if (!(sl > 0.0)) return GCS_ERR_ARG;  // up parallel to the view direction
    for (double& x : sv) x /= sl;
    const double u[3] = {sv[1] * f[2] - sv[2] * f[1], sv[2] * f[0] - sv[0] * f[2], sv[0] * f[1] - sv[1] * f[0]};
    const double e[3] = {cam->pos[0], cam->pos[1], cam->pos[2]};
    const double V[16] = {sv[0], sv[1], sv[2], -(sv[0] * e[0] + sv[1] * e[1] + sv[2] * e[2]),
                          u[0],  u[1],  u[2],  -(u[0] * e[0] + u[1] * e[1] + u[2] * e[2]),
                          -f[0], -f[1], -f[2], (f[0] * e[0] + f[1] * e[1] + f[2] * e[2]),
                          0.0,   0.0,   0.0,   1.0};
    const double t = std::tan(0.5 * (double)cam->fovy_deg * 3.14159265358979323846 / 180.0);
    const double aspect = (double)width / (double)height;
    const double n = cam->z_near, fa = cam->z_far;
    const double P[16] = {1.0 / (aspect * t), 0.0, 0.0, 0.0,
                          0.0, 1.0 / t, 0.0, 0.0,
                          0.0, 0.0, -(fa + n) / (fa - n), -2.0 * fa * n / (fa - n),
                          0.0, 0.0, -1.0, 0.0};
    for (int k = 0; k < 16; ++k) {
        view[k] = (float)V[k];
        proj[k] = (float)P[k];
    }
    return GCS_OK;
}

int gcs_render_frame(gcs_ctx* c, const gcs_camera* cam, int32_t segment, int32_t width, int32_t height,
                     uint8_t* rgba, int32_t rgba_on_host) {
    if (!c || !cam || !rgba || width < 1 || height < 1) return GCS_ERR_ARG;
    if (segment < -1 || segment >= c->nseg) {
        c->last_error = "render: segment out of range";
        return GCS_ERR_ARG;
    }
    const int64_t pixels = (int64_t)width * height;
    if (pixels > ((int64_t)1 << 28)) {
        c->last_error = "render: frame larger than 2^28 pixels";
        return GCS_ERR_ARG;
    }
    float view[16], proj[16];
    if (gcs_camera_matrices(cam, width, height, view, proj)) {
        c->last_error = "render: degenerate camera";
        return GCS_ERR_ARG;
    }
    cudaSetDevice(c->device);
    if (pixels > c->render_pixels_cap) {
        // buffers in use by queued frames are released only once those are done
        GCS_CUDA(c, cudaStreamSynchronize(c->stream));
        if (c->render_acc) cudaFree(c->render_acc);
        if (c->render_rgba) cudaFree(c->render_rgba);
        c->render_acc = nullptr;
        c->render_rgba = nullptr;
        c->render_pixels_cap = 0;
        GCS_CUDA(c, cudaMalloc(reinterpret_cast<void**>(&c->render_acc), sizeof(unsigned long long) * 3 * pixels));
        GCS_CUDA(c, cudaMalloc(reinterpret_cast<void**>(&c->render_rgba), 4 * (size_t)pixels));
        c->render_pixels_cap = pixels;
    }
    const int64_t first = segment < 0 ? 0 : c->h_seg_off[segment];
    const int64_t n = segment < 0 ? c->n : c->h_seg_off[segment + 1] - first;
    GCS_CUDA(c, cudaMemsetAsync(c->render_acc, 0, sizeof(unsigned long long) * 3 * pixels, c->stream));
    launch_splat_posvel(c->pos[c->cur] + first, c->vel[c->cur] + first, n, view, proj, width, height, c->render_acc,
                        c->stream);
    uint8_t* target = rgba_on_host ? c->render_rgba : rgba;
    launch_resolve(c->render_acc, pixels, target, c->stream);
    int rc = check_launch(c, "render");
    if (rc) return rc;
    if (rgba_on_host) {
        GCS_CUDA(c, cudaMemcpyAsync(rgba, c->render_rgba, 4 * (size_t)pixels, cudaMemcpyDeviceToHost, c->stream));
        GCS_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    return GCS_OK;
}

int gcs_render_stars(const Star* stars, int64_t n, const gcs_camera* cam, int32_t width, int32_t height,
                     uint64_t* accum, uint8_t* rgba, void* stream) {
    if (n < 0 || (n > 0 && !stars) || !cam || !accum || width < 1 || height < 1) return GCS_ERR_ARG;
    const int64_t pixels = (int64_t)width * height;
    if (pixels > ((int64_t)1 << 28)) return GCS_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(accum) & 7u) || (reinterpret_cast<uintptr_t>(rgba) & 3u) ||
        (reinterpret_cast<uintptr_t>(stars) & 15u))
        return GCS_ERR_ARG;
    float view[16], proj[16];
    if (gcs_camera_matrices(cam, width, height, view, proj)) return GCS_ERR_ARG;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    launch_splat_stars(stars, n, view, proj, width, height, reinterpret_cast<unsigned long long*>(accum), st);
    if (rgba) launch_resolve(reinterpret_cast<const unsigned long long*>(accum), pixels, rgba, st);
    return cudaGetLastError() == cudaSuccess ? GCS_OK : GCS_ERR_CUDA;
}

int gcs_render_playback(const PlaybackStar* frame, int64_t n, const gcs_camera* cam, int32_t width, int32_t height,
                        uint64_t* accum, uint8_t* rgba, void* stream) {
    if (n < 0 || (n > 0 && !frame) || !cam || !accum || width < 1 || height < 1) return GCS_ERR_ARG;
    const int64_t pixels = (int64_t)width * height;
    if (pixels > ((int64_t)1 << 28)) return GCS_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(accum) & 7u) || (reinterpret_cast<uintptr_t>(rgba) & 3u) ||
        (reinterpret_cast<uintptr_t>(frame) & 15u))
        return GCS_ERR_ARG;
    float view[16], proj[16];
    if (gcs_camera_matrices(cam, width, height, view, proj)) return GCS_ERR_ARG;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    launch_splat_playback(frame, n, view, proj, width, height, reinterpret_cast<unsigned long long*>(accum), st);
    if (rgba) launch_resolve(reinterpret_cast<const unsigned long long*>(accum), pixels, rgba, st);
    return cudaGetLastError() == cudaSuccess ? GCS_OK : GCS_ERR_CUDA;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// bake: steps written as simulation.bin frames (main.cpp:119-297)
// ---------------------------------------------------------------------------
// The reference's Bake loop steps synchronously, copies the Star array to
// the host, converts it to PlaybackStar records on the host and hands the
// frame to a writer thread.  Here each frame is packed on the device
// (launch_pack_playback, the same records gcs_download_playback returns),
// copied on a second stream into one of two pinned buffers while the next
// step computes, and written by a writer thread in frame order.
namespace {

struct BakeWriter {
    std::mutex mu;
    std::condition_variable cv;
    int64_t queued = 0;   // frames handed to the writer
    int64_t written = 0;  // frames written (or abandoned after an error)
    bool stop = false;
    int error = 0;
};

}  // namespace

extern "C" int gcs_bake(gcs_ctx* c, const gcs_params* p, int32_t frames, const char* path, int32_t append,
                        double* seconds) {
    if (!c || !p || !path || frames < 0) return GCS_ERR_ARG;
    int rc = validate_params(c, p);
    if (rc) return rc;
    const auto t0 = std::chrono::steady_clock::now();
    FILE* f = std::fopen(path, append ? "ab" : "wb");
    if (!f) {
        c->last_error = std::string("bake: cannot open ") + path;
        return GCS_ERR_ARG;
    }
    cudaSetDevice(c->device);
    const int64_t n = c->n;
    const size_t bytes = sizeof(PlaybackStar) * (size_t)n;
    // pinned buffers, copy stream and events live with the context
    bool ok = true;
    if (!c->bake_stream) {
        ok = cudaStreamCreateWithFlags(&c->bake_stream, cudaStreamNonBlocking) == cudaSuccess;
        for (int b = 0; b < 2 && ok; ++b)
            ok = cudaEventCreateWithFlags(&c->bake_packed[b], cudaEventDisableTiming) == cudaSuccess &&
                 cudaEventCreateWithFlags(&c->bake_copied[b], cudaEventDisableTiming) == cudaSuccess;
    }
    if (ok && n > c->bake_frames_cap) {
        for (int b = 0; b < 2; ++b) {
            if (c->bake_host[b]) cudaFreeHost(c->bake_host[b]);
            c->bake_host[b] = nullptr;
        }
        c->bake_frames_cap = 0;
        ok = cudaMallocHost(reinterpret_cast<void**>(&c->bake_host[0]), bytes) == cudaSuccess &&
             cudaMallocHost(reinterpret_cast<void**>(&c->bake_host[1]), bytes) == cudaSuccess;
        if (ok) c->bake_frames_cap = n;
    }
    PlaybackStar* const host[2] = {c->bake_host[0], c->bake_host[1]};
    const cudaStream_t copy = c->bake_stream;
    cudaEvent_t* const packed = c->bake_packed;
    cudaEvent_t* const copied = c->bake_copied;
    BakeWriter W;
    std::thread writer;
    if (ok) {
        writer = std::thread([&]() {
            for (int64_t k = 0;; ++k) {
                {
                    std::unique_lock<std::mutex> lk(W.mu);
                    W.cv.wait(lk, [&] { return W.queued > k || W.stop; });
                    if (W.queued <= k) return;
                }
                int err = 0;
                if (cudaEventSynchronize(copied[k & 1]) != cudaSuccess) err = GCS_ERR_CUDA;
                else if (n > 0 && std::fwrite(host[k & 1], sizeof(PlaybackStar), (size_t)n, f) != (size_t)n)
                    err = GCS_ERR_ARG;
                {
                    std::lock_guard<std::mutex> lk(W.mu);
                    if (err && !W.error) W.error = err;
                    W.written = k + 1;
                }
                W.cv.notify_all();
            }
        });
    } else {
        c->last_error = "bake: pinned buffers, copy stream or events could not be created";
        rc = GCS_ERR_NOMEM;
    }
    for (int32_t k = 0; ok && k < frames; ++k) {
        if ((rc = gcs_step(c, p))) break;
        // the staging buffer is free again once the previous frame's copy is done
        if (k >= 1 && cudaStreamWaitEvent(c->stream, copied[(k - 1) & 1], 0) != cudaSuccess) {
            rc = GCS_ERR_CUDA;
            break;
        }
        if (n > 0) launch_pack_playback(c->pos[c->cur], c->vel[c->cur], c->pb_staging, n, c->stream);
        if ((rc = check_launch(c, "bake pack")) || cudaEventRecord(packed[k & 1], c->stream) != cudaSuccess) {
            rc = rc ? rc : GCS_ERR_CUDA;
            break;
        }
        {
            // host buffer k & 1 is free once frame k - 2 has been written
            std::unique_lock<std::mutex> lk(W.mu);
            W.cv.wait(lk, [&] { return W.written >= (int64_t)k - 1 || W.error; });
            if (W.error) break;
        }
        if (cudaStreamWaitEvent(copy, packed[k & 1], 0) != cudaSuccess ||
            (n > 0 && cudaMemcpyAsync(host[k & 1], c->pb_staging, bytes, cudaMemcpyDeviceToHost, copy) != cudaSuccess) ||
            cudaEventRecord(copied[k & 1], copy) != cudaSuccess) {
            rc = GCS_ERR_CUDA;
            break;
        }
        {
            std::lock_guard<std::mutex> lk(W.mu);
            W.queued = (int64_t)k + 1;
        }
        W.cv.notify_all();
    }
    if (writer.joinable()) {
        {
            std::lock_guard<std::mutex> lk(W.mu);
            W.stop = true;
        }
        W.cv.notify_all();
        writer.join();
    }
    if (!rc && W.error) {
        rc = W.error;
        c->last_error = rc == GCS_ERR_CUDA ? "bake: frame copy failed" : "bake: short write of a frame";
    }
    if (std::fclose(f) != 0 && !rc) {
        rc = GCS_ERR_ARG;
        c->last_error = "bake: closing the output failed";
    }
    if (copy) cudaStreamSynchronize(copy);
    if (!rc) rc = gcs_synchronize(c);
    if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}
