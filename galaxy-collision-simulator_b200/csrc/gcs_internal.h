// gcs_internal.h - declarations shared by the engine's translation units.
//
// Device arrays (one context, N particles in S segments, n_internal = N - S):
//   pos[2]   float4 x,y,z,mass           (ping-pong across the gather)
//   vel[2]   float4 vx,vy,vz,bits(tcol)  (tcol = type | r<<8 | g<<16 | b<<24,
//                                         the byte order of Star bytes 28..31)
//   acc      float4 ax,ay,az,potential
//   keys[2]  u64 Morton codes, idx[2] u32 positions (radix-sort ping-pong)
//   nodes_tr BvhNodeTraverse[n_internal], nodes_bd BvhNodeBuild[n_internal],
//   wn       WalkNode[n_internal] (walk records: com, G*mass, width^2, codes)
//   com64    double4 [n_internal] FP64 mass-weighted position sums
//   leaf_parent i32[N]
//   seg_off  i64[S+1], seg_id i32[N], groups int4[n_groups]
//   scratch  zeroed once per step (sort histograms, tile counters, look-back,
//            walk work counter, device bounds)
#pragma once
#include <cstdint>
#include <mutex>
#include <utility>
#include <cuda_runtime.h>
#include "../../include/gcs_types.h"
#include "../../include/gcs.h"

namespace gcs {

// ---- per-device set-up ------------------------------------------------------
// Kernel attributes (the dynamic shared-memory opt-in above 48 KB) belong to
// a device's context, not to the process: a process that drives several
// devices must set them on each.  once_per_device runs `set` once for the
// current device, thread-safe; devices beyond kMaxDevices run it every time.
constexpr int kMaxDevices = 64;
int current_device();      // the current device, or -1
int current_sm_count();    // its SM count (cached per device; 148 if unknown)
template <class F>
void once_per_device(std::once_flag (&flags)[kMaxDevices], F&& set) {
    const int dev = current_device();
    if (dev < 0 || dev >= kMaxDevices) {
        set();
        return;
    }
    std::call_once(flags[dev], std::forward<F>(set));
}

constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kKeyPasses = 8;          // 63 Morton bits in 8-bit digits
constexpr int kMaxPasses = 10;         // + up to two segment-id digits
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys per tile
constexpr int kGroupSize = 64;         // walk targets per warp group (two per lane above 32)

// Work unit of the walk: up to kGroupSize consecutive sorted particles of one
// segment; `super` is its super-group (walk frontiers, below).
struct WalkGroup {
    int32_t start;
    int32_t count;
    int32_t seg;
    int32_t super;
};

// Per-segment bounds chunk: a range of particles of one segment.
struct Chunk {
    int32_t start;
    int32_t count;
    int32_t seg;
    int32_t pad;
};

// Layout of the concatenated segments as the kernels see it.
struct Layout {
    int32_t n;            // particles
    int32_t nseg;         // segments
    int32_t n_internal;   // n - nseg
    const int64_t* seg_off;  // device [nseg+1]
    const int32_t* seg_id;   // device [n]
};

// Per-step scratch, one device allocation.  Each stage zeroes only the
// region it accumulates into, so any stage can be run on its own:
//   hist      u32[kMaxPasses][256]  radix digit histograms   (zeroed by encode)
//   walk_q    u32[2]                walk work queue          (self-resetting)
//   bounds    u32[2 * max_segments] ordered min/max          (zeroed by bounds)
//   tiles     u32[kMaxPasses]       onesweep tile tickets    (zeroed by sort,
//   lookback  u32[passes][tiles][256] decoupled look-back      with lookback)
struct ScratchLayout {
    size_t hist, walk_q, bounds, tiles, lookback, end;
};

// ---- launchers (one per stage; all asynchronous on `st`) ----------------
void launch_fill_segment_ids(const int64_t* seg_off, int nseg, int32_t* seg_id, int64_t n,
                             cudaStream_t st);
void launch_unpack_stars(const Star* stars, float4* pos, float4* vel, int64_t n, cudaStream_t st);
void launch_pack_stars(const float4* pos, const float4* vel, Star* out, int64_t n, cudaStream_t st);
void launch_pack_playback(const float4* pos, const float4* vel, PlaybackStar* out, int64_t n,
                          cudaStream_t st);

void launch_bounds(const Layout& L, const float4* pos, const Chunk* chunks, int n_chunks,
                   uint32_t* bounds_enc, uint32_t* status, cudaStream_t st);
void launch_bounds_decode(const uint32_t* bounds_enc, float2* bounds, int nseg, cudaStream_t st);
void launch_encode(const Layout& L, const float4* pos, int bounds_mode, float gmin, float gmax,
                   const float2* seg_bounds, uint64_t* keys, uint32_t* idx, uint32_t* hist,
                   int n_seg_passes, cudaStream_t st);

size_t sort_lookback_words(int64_t n, int passes);
void launch_sort_pass(const Layout& L, int pass, const uint64_t* keys_in, const uint32_t* vals_in,
                      uint64_t* keys_out, uint32_t* vals_out, const uint32_t* hist,
                      uint32_t* tile_counter, uint32_t* lookback, uint32_t* status,
                      cudaStream_t st);

void launch_gather(const uint32_t* idx, const float4* pos_in, const float4* vel_in, float4* pos_out,
                   float4* vel_out, int64_t n, cudaStream_t st);
void launch_build(const Layout& L, const uint64_t* keys, BvhNodeTraverse* tr, BvhNodeBuild* bd,
                  int32_t* leaf_parent, uint32_t* status, cudaStream_t st);
struct WalkNodeParams;
void launch_aggregate(const Layout& L, const float4* pos, BvhNodeTraverse* tr, BvhNodeBuild* bd,
                      double4* com64, const int32_t* leaf_parent, int com_fp64, const WalkNodeParams& wnp,
                      uint32_t* status, cudaStream_t st);

struct WalkParams {
    float G, eps2, theta2;
    int32_t leaf_size;
    int32_t batch;
    int32_t with_potential;
};

// Walk record of one internal node (32 bytes, two 16-byte loads), written
// beside the node's BvhNodeTraverse record for a given G and leaf size L:
//   cm    com.x, com.y, com.z, G*mass
//   link  bits(width^2), code_a, code_b, 0 where
//           code_b >= kWalkBucketTag  the node holds <= L particles, summed
//                                     directly: [code_a, code_a + code_b - tag)
//           code_b == kWalkSkipTag    malformed links: nothing below it
//           otherwise                 children: >= 0 internal node,
//                                     < 0 particle ~code
// Every code names an index below the context's capacity, so a walk over
// stale records reads inside its arrays.
struct WalkNode {
    float4 cm;
    int4 link;
};
static_assert(sizeof(WalkNode) == 32, "WalkNode must be 32 bytes");
constexpr int kWalkBucketTag = 1 << 30;
constexpr int kWalkSkipTag = 0x7FFFFFFF;
// G and leaf size of the walk records an aggregation writes (wn null: none).
struct WalkNodeParams {
    WalkNode* wn;
    float G;
    int32_t leaf_size;  // 1..32
};
// Walk records of every internal node from the traverse records (when the
// walk runs with a G or leaf size other than the aggregation's).
void launch_walk_nodes(const Layout& L, const BvhNodeTraverse* tr, WalkNodeParams wnp, uint32_t* status,
                       cudaStream_t st);
// Global-memory stack entries (int2) per walk warp: the shared-memory stack
// spills its bottom here.  A round adds at most `batch` entries per tree
// level, so 8192 covers batch 64 on trees 128 levels deep.
constexpr int kWalkGlobalStack = 8192;
constexpr int kWalkMaxBatch = 64;  // nodes popped per walk round
// targets_per_lane: 1 for groups of <= 32 targets, 2 for groups of <= 64.
// Optional epilogue of the walk: each warp, once its group's accelerations
// are written, applies the kick/drift to the group's particles out of place
// (pos/vel_in -> pos_out/vel_out, so the walk's other warps keep reading the
// step's positions) and writes their Star records.  Groups are counted in
// chunks of consecutive groups: chunk k is groups [chunk_bound[k],
// chunk_bound[k + 1]) of n_chunks (the host makes large chunks over the groups
// handed out early and small ones over the groups still in flight when the
// work queue runs dry, which finish together at the end of the walk, and
// puts every boundary at a super-group edge, so that a chunk's particles are
// one contiguous range also when groups take their targets through a
// partition of their super-group).  The warp that completes a chunk stores `epoch` into
// host_flags[chunk] (mapped host memory, after a system-scope fence), so the
// host can copy that chunk's Stars while the walk continues; with
// host_flags == nullptr nothing is counted (the records go straight to
// pinned host memory).  vel_in == nullptr: no epilogue.  chunk_done must be
// zero at launch.
struct WalkEpilogue {
    const float4* vel_in = nullptr;
    float4* pos_out = nullptr;
    float4* vel_out = nullptr;
    float4* stars = nullptr;  // Star records as float4 pairs
    float dt = 0.0f;
    int32_t recolor = 0;
    int32_t n_chunks = 0;
    uint32_t* chunk_done = nullptr;
    uint32_t* host_flags = nullptr;
    uint32_t epoch = 0;
    int32_t chunk_bound[65] = {};  // kMaxStarChunks + 1 group indices
};
constexpr int kMaxStarHeadChunks = 16;
constexpr int kMaxStarTailChunks = 48;
constexpr int kMaxStarChunks = kMaxStarHeadChunks + kMaxStarTailChunks;
static_assert(kMaxStarChunks + 1 == sizeof(WalkEpilogue::chunk_bound) / sizeof(int32_t), "chunk table size");
constexpr int kWalkBlockWarps = 8;  // warps per walk block

// ---- walk frontiers ------------------------------------------------------
// Consecutive walk groups of one segment form a super-group of at most
// kSuperTargets targets.  Before the walk, a frontier pass walks the tree once
// per super-group against the super-group's bounding box (the same box test
// as the group walk, which never contradicts a target's own opening test):
// nodes every target of the super-group accepts go to its take list, the
// particles of nodes every target opens and sums directly (leaf children,
// small nodes) to its source list, the children of other nodes every target
// opens are visited, and nodes the box cannot decide end the pass as its
// frontier.  Every target of the super-group reaches each of those nodes with
// every ancestor opened, so a group's walk evaluates the take list and the
// sources for all its targets and then starts from the frontier with full
// masks: each target's terms are exactly those of its walk from the root.
// A super-group whose lists do not fit (kSuperCap, kSuperSrcCap) is marked
// invalid and its groups walk from the root.
constexpr int kSuperTargets = 256;
constexpr int kSuperCap = 2048;     // take nodes (from the front) + frontier nodes (from the back)
constexpr int kSuperSrcCap = 256;   // particle sources of a super-group
// Targets [start, start + count) of segment seg (a run of whole groups).
struct SuperGroup {
    int32_t start;
    int32_t count;
    int32_t seg;
    int32_t pad;
};
struct WalkFrontier {
    const SuperGroup* supers = nullptr;  // null: every group walks from its root
    int n_supers = 0;
    int32_t* list = nullptr;  // [n_supers][kSuperCap]
    int32_t* src = nullptr;   // [n_supers][kSuperSrcCap] sorted particle indices
    int4* meta = nullptr;     // per super-group: n_take, n_src, n_front, valid
    // Targets in group order (null: Morton order).  A full super-group of
    // kSuperTargets targets is split into its groups by recursive median
    // bisection along the longest axis of each part's box, so the groups are
    // spatially tighter than runs of the Morton order (fewer nodes that
    // only some of a group's targets accept); group g takes targets
    // perm[start .. start + count).  Partial super-groups keep Morton order.
    int32_t* perm = nullptr;
    int32_t split_levels = 0;  // bisection levels: kSuperTargets >> levels == group width
    // Optional second stream for the partition: forked from the walk's stream
    // with `fork`, joined back with `join` before the walk, so it runs beside
    // the frontier pass (both are short latency chains).
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};

void launch_walk(const Layout& L, const WalkParams& wp, const float4* pos,
                 const WalkNode* wn, const WalkGroup* groups, int n_groups, int targets_per_lane,
                 float4* acc, uint32_t* queue, uint32_t* status, int blocks_per_sm,
                 int sm_count, unsigned long long* counts, int2* gstack, size_t gstack_entries,
                 cudaStream_t st, const WalkEpilogue& ep = WalkEpilogue(),
                 const WalkFrontier& fr = WalkFrontier());
int walk_max_blocks_per_sm(int batch, int with_potential, int targets_per_lane);
// Persistent walk grid (blocks) for n_groups groups, and the global stack
// entries that grid needs.
int64_t walk_grid_blocks(int n_groups, int blocks_per_sm, int sm_count, int with_potential);
size_t walk_stack_entries(int64_t grid_blocks);

void launch_integrate(float4* pos, float4* vel, const float4* acc, float dt, int recolor,
                      int64_t n, cudaStream_t st);
void launch_kick(float4* vel, const float4* acc, float dt, int64_t n, cudaStream_t st);

void launch_diag(const float4* pos, const float4* vel, const float4* acc, int64_t first, int64_t n,
                 double kick, double* out6, cudaStream_t st);
// Pack the context's current particles as Star[] into a device buffer and
// wait for it (the headless interop target of the drop-in API).
int pack_to_device(gcs_ctx* c, Star* dst);

// Headless point-splat renderer (k_render.cu): fixed-point fragment sums
// into acc (width*height*3 u64, zeroed by the caller), then RGBA8.
void launch_splat_posvel(const float4* pos, const float4* vel, int64_t n, const float* view, const float* proj,
                         int width, int height, unsigned long long* acc, cudaStream_t st);
void launch_splat_stars(const Star* stars, int64_t n, const float* view, const float* proj, int width, int height,
                        unsigned long long* acc, cudaStream_t st);
void launch_splat_playback(const PlaybackStar* recs, int64_t n, const float* view, const float* proj, int width,
                           int height, unsigned long long* acc, cudaStream_t st);
void launch_resolve(const unsigned long long* acc, int64_t pixels, uint8_t* rgba, cudaStream_t st);

void launch_direct_fp64(const float4* pos, int64_t seg_first, int64_t seg_n, const int64_t* targets,
                        int64_t n_targets, double G, double eps2, double* out, cudaStream_t st);

}  // namespace gcs
