// k_walk.cu - Barnes-Hut tree walk: accelerations (and optionally potentials)
// of every particle from its segment's tree.
//
// Semantics (per target particle, as query_gravity_bvh_kernel,
// cuda_engine.cu:91-161, extended with theta and a leaf size L):
//   * an internal node with softened distance d2 = |com - x|^2 + eps^2 is
//     used as a monopole iff width^2 < theta^2 * d2;
//   * otherwise it is opened: if it holds <= L particles they are summed
//     one by one, else its two children are visited;
//   * a leaf (one particle) is always summed directly, skipping sources with
//     d2 <= 1.01 eps^2 (the reference's self-exclusion, cuda_engine.cu:134);
//   * a term adds G m d / d2^{3/2}, with the hardware 1/sqrt.
// With theta = 1 and L = 1 every target sees exactly the reference's set of
// terms; only the order of the FP32 sums differs.
//
// Execution: a persistent grid of warps pulls groups of <= 32*T consecutive
// (Morton-adjacent) targets of one segment from a global work queue; lane l
// holds targets l and l+32 (T = 2) of its group.  The warp walks the tree once
// for its group with one stack; each stack entry carries, for each of the T
// target slots, the mask of lanes that still need that subtree, and each
// target takes its own opening decision, so the group walk is the union of
// the per-target walks with no change to any target's terms.  Nodes are read
// from walk records (WalkNode: centre of mass and G*mass, width^2, and the
// children or the bucket range for the step's leaf size), which the
// aggregation writes beside the traverse records.  Each round:
//   1. up to `batch` (<= 32*H) entries are popped; lane k fetches the
//      records of nodes k and k+32 (two 16-byte loads each);
//   2. each node is classified against the group's bounding box with a
//      2^-16 relative margin: "take" if every target of the box must accept
//      it, "open" if every target must open it, else "mixed" (the margin is
//      far above the few-ulp rounding of any target's own d2, so a class
//      never contradicts a target's own test);
//   3. take nodes whose masks hold every live target go through a monopole
//      loop without masks, other take nodes through a masked one, mixed
//      nodes through the per-target opening test (a predicated monopole and
//      a ballot of opening lanes per target slot); open nodes skip
//      evaluation altogether.  Every node loaded from shared memory is
//      evaluated for the lane's T targets;
//   4. in parallel, each lane pushes its nodes' internal children and
//      appends their particle sources (leaf children, or the whole range of
//      a small node) at offsets from one warp prefix scan;
//   5. particle sources accumulate in a per-warp list; when it fills, the
//      lanes fetch up to 64 source records in parallel into shared memory and
//      every lane sums them for its targets.
// The stack's top lives in shared memory; when it passes a threshold its
// bottom is spilled to a per-warp region of global memory (L2) and read back
// when the top runs low, so batches are never throttled and the logical
// stack order is that of an unbounded stack.  A global region that would
// overflow sets GCS_DEV_WALK_STACK_OVERFLOW (entries are dropped, nothing is
// written out of bounds); a walk that pops more nodes than the tree holds
// stops with GCS_DEV_TREE_MALFORMED.  The work queue resets itself: the last
// warp to find it empty zeroes it.
//
// With an epilogue (WalkEpilogue), a warp that has written its group's
// accelerations also applies the step's kick/drift to those particles, out of
// place, and writes their Star records (when given); the warp that completes a chunk of
// groups raises that chunk's flag in mapped host memory (chunks are large
// over the groups handed out early and small over the last ones, which are
// all in flight together at the end).  The host copies
// finished chunks to its Star array while the walk is still running (the
// reference copies all Stars after the step, cuda_engine.cu:442-448).  When
// the Star array is pinned host memory mapped into the device, the records
// go straight into it and no chunk is counted (host_flags == nullptr).
#include <algorithm>
#include <atomic>

#include "gcs_internal.h"
#include "device_math.cuh"

namespace gcs {

namespace {

constexpr int kWalkWarps = kWalkBlockWarps;
constexpr int kWalkThreads = kWalkWarps * 32;
constexpr int kSpillCount = 128;  // entries moved per spill / refill
constexpr int kSrcCap = 64;
constexpr uint32_t kFull = 0xFFFFFFFFu;
// Node codes come from the walk records (WalkNode: code_a / code_b with
// kWalkBucketTag and kWalkSkipTag).

// Classes of a batch node against the group's bounding box.
constexpr int kClassNone = 0;      // lane holds no node
constexpr int kClassTake = 1;      // every target of the group accepts it
constexpr int kClassOpen = 2;      // every target of the group opens it
constexpr int kClassMixed = 3;     // targets decide one by one
constexpr int kClassTakeFull = 4;  // kClassTake, and every live target is in its masks
constexpr float kBoxLo = 1.0f - 1.0f / 65536.0f;
constexpr float kBoxHi = 1.0f + 1.0f / 65536.0f;

// Class of a node (centre of mass c, width^2 w2) against a box of targets:
// the squared softened distances from c to the nearest and farthest points
// of the box bound every target's own d2, and the 2^-16 margins in k_take =
// theta^2 (1 - 2^-16) and k_open = theta^2 (1 + 2^-16) are far above the
// few-ulp rounding of a target's own d2, so "take" means every target of the
// box accepts the node (w2 < theta^2 d2) and "open" that every target opens
// it.
__device__ __forceinline__ int box_class(float4 c, float w2, float3 lo, float3 hi, float eps2, float k_take,
                                         float k_open) {
    float s2min = eps2, s2max = eps2;
    const float dl[3] = {lo.x - c.x, lo.y - c.y, lo.z - c.z};
    const float dh[3] = {c.x - hi.x, c.y - hi.y, c.z - hi.z};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const float near = fmaxf(fmaxf(dl[ax], dh[ax]), 0.0f);
        const float far = fmaxf(fabsf(dl[ax]), fabsf(dh[ax]));
        s2min = fmaf(near, near, s2min);
        s2max = fmaf(far, far, s2max);
    }
    if (w2 < s2min * k_take) return kClassTake;
    if (w2 >= s2max * k_open) return kClassOpen;
    return kClassMixed;
}

// Stack entry: node index and one lane mask per target slot.
template <int T>
struct EntryOf;
template <>
struct EntryOf<1> {
    using type = int2;
};
template <>
struct EntryOf<2> {
    using type = int4;
};
__device__ __forceinline__ int2 make_entry(int node, const uint32_t (&m)[1]) { return make_int2(node, (int)m[0]); }
__device__ __forceinline__ int4 make_entry(int node, const uint32_t (&m)[2]) {
    return make_int4(node, (int)m[0], (int)m[1], 0);
}
__device__ __forceinline__ void entry_masks(int2 e, uint32_t (&m)[1]) { m[0] = (uint32_t)e.y; }
__device__ __forceinline__ void entry_masks(int4 e, uint32_t (&m)[2]) {
    m[0] = (uint32_t)e.y;
    m[1] = (uint32_t)e.z;
}

// Per-warp shared memory for H nodes per lane per round and T targets per
// lane.  Nodes and sources to evaluate are stored in pairs (slot 2q and 2q+1
// side by side), so that one packed FP32 instruction (sm_100 f32x2) evaluates
// two of them: full-mask take nodes fill slots [0, n_full), other take nodes
// and mixed nodes each start at the next even slot, and an odd list is padded
// with an empty entry (mass 0 at 1e30 in every coordinate, lane masks 0).
template <int H, int T>
struct WarpSmem {
    using Entry = typename EntryOf<T>::type;
    static constexpr int kBatch = 32 * H;
    static constexpr int kPairs = kBatch / 2 + 2;  // three padded lists
    static_assert(2 * kPairs >= kBatch, "a source descriptor per popped node fits sdesc and pmask");
    // A round starts with top <= kSpillAbove (or < kBatch before a refill of
    // <= kSpillCount) and pushes <= 2 * batch; one spill of kSpillCount
    // brings top back to <= kSpillAbove.
    static constexpr int kStackCap = T == 1 ? 256 + 64 * H : kSpillCount + 2 * kBatch + 32;
    static constexpr int kSpillAbove = kStackCap - 2 * kBatch;
    static_assert(kSpillAbove >= kSpillCount && kBatch <= kSpillCount, "stack sizing");
    static_assert(2 * kBatch + kSpillCount - 1 <= kStackCap, "refill then push must fit");
    Entry stk[kStackCap];           // node, lane masks
    union {
        struct {
            float4 pxy[kPairs];     // x0 x1 y0 y1 of the centres of mass of slots 2q, 2q+1
            float4 pzm[kPairs];     // z0 z1 Gm0 Gm1
        };
        // after a round's evaluation: one descriptor per node with particle
        // sources (first source in the round, its two child codes), in source
        // order; the lane masks go to pmask
        int4 sdesc[2 * kPairs];
    };
    float2 pw2[kPairs];             // width^2 of both slots
    uint2 pmask[T][kPairs];         // lane masks of both slots, per target slot
    uint2 pnopen[T][kPairs];        // opening lanes of both slots (mixed nodes)
    float4 sxy[kSrcCap / 2];        // particle sources in pairs: x0 x1 y0 y1
    float4 szm[kSrcCap / 2];        // z0 z1 Gm0 Gm1
    uint2 smask[T][kSrcCap / 2];    // lane masks
    int srcp[kSrcCap];              // the list before its fetch: particle
    uint32_t srcm[T][kSrcCap];      //   and its lane masks
};

// Store one entry's coordinates at pair slot `slot` of a pair-interleaved list.
__device__ __forceinline__ void put_pair(float4* xy, float4* zm, int slot, float4 c) {
    const int q = slot >> 1, e = slot & 1;
    float* fxy = reinterpret_cast<float*>(xy + q);
    float* fzm = reinterpret_cast<float*>(zm + q);
    fxy[e] = c.x;
    fxy[2 + e] = c.y;
    fzm[e] = c.z;
    fzm[2 + e] = c.w;
}
__device__ __forceinline__ void put_mask(uint2* mk, int slot, uint32_t mask) {
    reinterpret_cast<uint32_t*>(mk + (slot >> 1))[slot & 1] = mask;
}

// Resident blocks per SM the register budget is set for (T=1: H=1 48
// registers a thread, 40 warps; H=2 64 registers, 32 warps; T=2: 80
// registers, 24 warps).
template <int H, int T>
struct WalkOcc {
    static constexpr int kMinBlocks = T == 2 ? 3 : (H == 1 ? 5 : 4);
};

// Sums of one target: two partial sums per component (even / odd slots).
struct Accum {
    float2 ax, ay, az, pot;
    uint32_t n_mono, n_part;  // interaction counts (count mode only)
};
// Warp-wide counters (count mode only).
struct WarpCount {
    uint32_t w_node, w_src;       // warp-wide node / source evaluations
    uint32_t rounds, spills;      // pop rounds, stack spills to global memory
    uint32_t all_open, all_take;  // nodes classified open / take by the box test
    uint32_t peak;                // deepest stack (shared top + global bottom), entries
    // lane use: evaluated rows (one node or source for every target slot of
    // the warp) by kind, and the target slots each kind served
    uint32_t r_list, r_full, r_part, r_mixed;  // take list, full-mask take, other take, mixed
    uint32_t l_part, l_mixed, l_accept, l_src;  // lanes in masks; mixed: lanes accepting; sources
};

// Sum over the warp of popc(m) where `in` holds.
__device__ __forceinline__ uint32_t warp_popc_sum(bool in, uint32_t m) {
    return (uint32_t)__reduce_add_sync(0xFFFFFFFFu, in ? (uint32_t)__popc(m) : 0u);
}

// Two evaluation entries for one target, packed (sm_100 f32x2): d = c - x
// and the softened d2 of both.  Each element is rounded exactly as the
// scalar forms round it (softened_d2), so opening decisions are the
// reference's.
struct PairD {
    float2 dx, dy, dz, d2;
};

__device__ __forceinline__ PairD pair_d(float4 xy, float4 zm, float2 npx, float2 npy, float2 npz, float2 e2) {
    PairD r;
    r.dx = __fadd2_rn(make_float2(xy.x, xy.y), npx);
    r.dy = __fadd2_rn(make_float2(xy.z, xy.w), npy);
    r.dz = __fadd2_rn(make_float2(zm.x, zm.y), npz);
    r.d2 = softened_d2_x2(r.dx, r.dy, r.dz, e2);
    return r;
}

// pair_d for nodes every target of the entry accepts: no opening decision
// depends on d2 here, so eps^2 starts the FMA chain (d2 differs from the
// decision form by rounding only).
__device__ __forceinline__ PairD pair_d_take(float4 xy, float4 zm, float2 npx, float2 npy, float2 npz, float2 e2) {
    PairD r;
    r.dx = __fadd2_rn(make_float2(xy.x, xy.y), npx);
    r.dy = __fadd2_rn(make_float2(xy.z, xy.w), npy);
    r.dz = __fadd2_rn(make_float2(zm.x, zm.y), npz);
    r.d2 = __ffma2_rn(r.dz, r.dz, __ffma2_rn(r.dy, r.dy, __ffma2_rn(r.dx, r.dx, e2)));
    return r;
}

// Terms of the two entries whose `use` is set: the hardware 1/sqrt, inv^3,
// G m inv^3, one FMA per component.
template <bool kPot>
__device__ __forceinline__ void pair_add(Accum& A, const PairD& d, float4 zm, bool use0, bool use1) {
    const float2 inv = make_float2(rsqrt_approx(d.d2.x), rsqrt_approx(d.d2.y));
    const float2 inv3 = __fmul2_rn(__fmul2_rn(inv, inv), inv);
    float2 f = __fmul2_rn(make_float2(zm.z, zm.w), inv3);
    f.x = use0 ? f.x : 0.0f;
    f.y = use1 ? f.y : 0.0f;
    A.ax = __ffma2_rn(d.dx, f, A.ax);
    A.ay = __ffma2_rn(d.dy, f, A.ay);
    A.az = __ffma2_rn(d.dz, f, A.az);
    if (kPot) {
        const float2 t = __ffma2_rn(make_float2(-zm.z, -zm.w), inv, A.pot);
        A.pot.x = use0 ? t.x : A.pot.x;
        A.pot.y = use1 ? t.y : A.pot.y;
    }
}

// The lane's targets: position as packed negatives (for d = c - x).
template <int T>
struct Targets {
    float2 npx[T], npy[T], npz[T];
};

// Sum the listed particle sources into every target whose lane bit is in
// the source's mask for its slot (leaf rule: skip d2 <= 1.01 eps^2).
template <int H, int T, bool kPot, bool kCount>
__device__ __forceinline__ void flush_sources(WarpSmem<H, T>& W, int nsrc, int lane, uint32_t lane_bit,
                                              const float4* __restrict__ pos, float G, const Targets<T>& X,
                                              float2 e2, float leaf_thr, Accum (&A)[T], WarpCount& WC) {
    __syncwarp();
    const int padded = (nsrc + 1) & ~1;
    for (int e = lane; e < padded; e += 32) {
        float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
        uint32_t m[T];
#pragma unroll
        for (int t = 0; t < T; ++t) m[t] = 0u;
        if (e < nsrc) {
            q = __ldg(pos + W.srcp[e]);
            q.w = __fmul_rn(G, q.w);
#pragma unroll
            for (int t = 0; t < T; ++t) m[t] = W.srcm[t][e];
        }
        put_pair(W.sxy, W.szm, e, q);
#pragma unroll
        for (int t = 0; t < T; ++t) put_mask(W.smask[t], e, m[t]);
    }
    __syncwarp();
#pragma unroll 4
    for (int q = 0; q < (padded >> 1); ++q) {
        const float4 zm = W.szm[q];
        const float4 xy = W.sxy[q];
#pragma unroll
        for (int t = 0; t < T; ++t) {
            const uint2 mk = W.smask[t][q];
            const PairD d = pair_d(xy, zm, X.npx[t], X.npy[t], X.npz[t], e2);
            const bool use0 = (mk.x & lane_bit) && (d.d2.x > leaf_thr);
            const bool use1 = (mk.y & lane_bit) && (d.d2.y > leaf_thr);
            pair_add<kPot>(A[t], d, zm, use0, use1);
            if (kCount) A[t].n_part += (use0 ? 1u : 0u) + (use1 ? 1u : 0u);
        }
    }
    if (kCount) {
        WC.w_src += (uint32_t)nsrc;
        for (int e0 = 0; e0 < nsrc; e0 += 32) {
            const int e = e0 + lane;
#pragma unroll
            for (int t = 0; t < T; ++t) WC.l_src += warp_popc_sum(e < nsrc, e < nsrc ? W.srcm[t][e] : 0u);
        }
    }
    __syncwarp();
}

__device__ __forceinline__ uint32_t warp_exclusive_scan(uint32_t v, int lane) {
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    return x - v;
}

template <int H, int T, bool kPot, bool kCount>
__global__ void __launch_bounds__(kWalkThreads, (WalkOcc<H, T>::kMinBlocks))
walk_kernel(Layout L, WalkParams wp, const float4* __restrict__ pos,
            const WalkNode* __restrict__ wn, const WalkGroup* __restrict__ groups,
            int n_groups, float4* __restrict__ acc, uint32_t* __restrict__ queue,
            uint32_t* __restrict__ status, unsigned long long* __restrict__ counts,
            typename EntryOf<T>::type* __restrict__ gstack, int gstack_cap, WalkEpilogue ep,
            WalkFrontier fr) {
    using Smem = WarpSmem<H, T>;
    using Entry = typename Smem::Entry;
    extern __shared__ __align__(16) unsigned char walk_smem[];
    const int warp = threadIdx.x >> 5;
    Smem& W = reinterpret_cast<Smem*>(walk_smem)[warp];
    Entry* const gstk = gstack + ((size_t)blockIdx.x * kWalkWarps + warp) * (size_t)gstack_cap;
    const int lane = threadIdx.x & 31;
    const uint32_t lane_bit = 1u << lane;
    const uint32_t lt = lane_bit - 1u;
    const float G = wp.G, eps2 = wp.eps2, theta2 = wp.theta2;
    const float2 e2 = make_float2(eps2, eps2), th2 = make_float2(theta2, theta2);
    const float leaf_thr = __fmul_rn(eps2, 1.01f);
    // box classification thresholds: take iff w^2 < s2min * k_take, open iff
    // w^2 >= s2max * k_open (theta^2 with the 2^-16 relative margin)
    const float k_take = theta2 * kBoxLo, k_open = theta2 * kBoxHi;
    const int batch = wp.batch;

    for (;;) {
        int g = 0;
        if (lane == 0) g = (int)atomicAdd(queue, 1u);
        g = __shfl_sync(kFull, g, 0);
        if (g >= n_groups) break;
        const WalkGroup grp = groups[g];
        bool valid[T];
        uint32_t live[T];
        Targets<T> X;
        // bounding box of the group's targets
        float3 box_lo = make_float3(INFINITY, INFINITY, INFINITY);
        float3 box_hi = make_float3(-INFINITY, -INFINITY, -INFINITY);
        Accum A[T];
#pragma unroll
        for (int t = 0; t < T; ++t) {
            valid[t] = lane + 32 * t < grp.count;
            float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
            if (valid[t]) {
                const int j = grp.start + lane + 32 * t;
                p = __ldg(pos + (fr.perm ? __ldg(fr.perm + j) : j));
            }
            live[t] = __ballot_sync(kFull, valid[t]);
            X.npx[t] = make_float2(-p.x, -p.x);
            X.npy[t] = make_float2(-p.y, -p.y);
            X.npz[t] = make_float2(-p.z, -p.z);
            if (valid[t]) {
                box_lo = make_float3(fminf(box_lo.x, p.x), fminf(box_lo.y, p.y), fminf(box_lo.z, p.z));
                box_hi = make_float3(fmaxf(box_hi.x, p.x), fmaxf(box_hi.y, p.y), fmaxf(box_hi.z, p.z));
            }
            A[t].ax = A[t].ay = A[t].az = A[t].pot = make_float2(0.f, 0.f);
            A[t].n_mono = A[t].n_part = 0u;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            box_lo.x = fminf(box_lo.x, __shfl_xor_sync(kFull, box_lo.x, o));
            box_lo.y = fminf(box_lo.y, __shfl_xor_sync(kFull, box_lo.y, o));
            box_lo.z = fminf(box_lo.z, __shfl_xor_sync(kFull, box_lo.z, o));
            box_hi.x = fmaxf(box_hi.x, __shfl_xor_sync(kFull, box_hi.x, o));
            box_hi.y = fmaxf(box_hi.y, __shfl_xor_sync(kFull, box_hi.y, o));
            box_hi.z = fmaxf(box_hi.z, __shfl_xor_sync(kFull, box_hi.z, o));
        }
        const int s = grp.seg;
        const int off = (int)__ldg(L.seg_off + s);
        const int seg_n = (int)__ldg(L.seg_off + s + 1) - off;
        WarpCount WC;
        WC.w_node = WC.w_src = WC.rounds = WC.spills = WC.all_open = WC.all_take = WC.peak = 0u;
        WC.r_list = WC.r_full = WC.r_part = WC.r_mixed = 0u;
        WC.l_part = WC.l_mixed = WC.l_accept = WC.l_src = 0u;
        int nsrc = 0;

        if (seg_n >= 2) {
            int top = 0, gtop = 0;
            int4 fm = make_int4(0, 0, 0, 0);
            if (fr.meta) fm = fr.meta[grp.super];
            if (fm.w && fm.z - Smem::kSpillAbove <= gstack_cap) {
                // the super-group's shared work: its take list for every
                // target (two records per lane per chunk of 64, staged in the
                // source pairs), its sources, then the frontier as the stack
                const int32_t* tl = fr.list + (size_t)grp.super * kSuperCap;
                for (int base = 0; base < fm.x; base += kSrcCap) {
                    const int cnt = min(kSrcCap, fm.x - base);
                    const int padded = (cnt + 1) & ~1;
                    for (int e = lane; e < padded; e += 32) {
                        float4 q = make_float4(1e30f, 1e30f, 1e30f, 0.0f);
                        if (e < cnt) q = __ldg(&wn[__ldg(tl + base + e)].cm);
                        put_pair(W.sxy, W.szm, e, q);
                    }
                    __syncwarp();
#pragma unroll 4
                    for (int q = 0; q < (padded >> 1); ++q) {
                        const float4 zm = W.szm[q];
                        const float4 xy = W.sxy[q];
#pragma unroll
                        for (int t = 0; t < T; ++t) {
                            const PairD d = pair_d_take(xy, zm, X.npx[t], X.npy[t], X.npz[t], e2);
                            pair_add<kPot>(A[t], d, zm, true, true);
                        }
                    }
                    __syncwarp();
                }
                if (kCount) {
#pragma unroll
                    for (int t = 0; t < T; ++t)
                        if (valid[t]) A[t].n_mono += (uint32_t)fm.x;
                    WC.w_node += (uint32_t)fm.x;
                    WC.all_take += (uint32_t)fm.x;
                    WC.r_list += (uint32_t)fm.x;
                }
                const int32_t* sl = fr.src + (size_t)grp.super * kSuperSrcCap;
                for (int base = 0; base < fm.y; base += kSrcCap) {
                    const int cnt = min(kSrcCap, fm.y - base);
                    for (int e = lane; e < cnt; e += 32) {
                        W.srcp[e] = __ldg(sl + base + e);
#pragma unroll
                        for (int t = 0; t < T; ++t) W.srcm[t][e] = live[t];
                    }
                    flush_sources<H, T, kPot, kCount>(W, cnt, lane, lane_bit, pos, G, X, e2, leaf_thr, A, WC);
                }
                // frontier entries [kSuperCap - n_front, kSuperCap): what the
                // shared stack cannot hold goes to the global bottom
                const int32_t* fl = tl + kSuperCap - fm.z;
                const int to_g = max(0, fm.z - Smem::kSpillAbove);
                for (int j = lane; j < to_g; j += 32) gstk[j] = make_entry(__ldg(fl + j), live);
                for (int j = lane; j < fm.z - to_g; j += 32) W.stk[j] = make_entry(__ldg(fl + to_g + j), live);
                gtop = to_g;
                top = fm.z - to_g;
            } else {
                if (lane == 0) W.stk[0] = make_entry(off - s, live);
                top = 1;
            }
            __syncwarp();
            // Each internal node has one parent, so a walk pops it at most
            // once: more pops than internal nodes means a malformed tree.
            int pop_budget = seg_n - 1;
            while (top > 0 || gtop > 0) {
                // refill the shared top from the global bottom when it runs low
                if (top < batch && gtop > 0) {
                    const int k = gtop < kSpillCount ? gtop : kSpillCount;
                    Entry keep[H];
#pragma unroll
                    for (int h = 0; h < H; ++h) keep[h] = lane + 32 * h < top ? W.stk[lane + 32 * h] : Entry{};
                    __syncwarp();
#pragma unroll
                    for (int h = 0; h < H; ++h)
                        if (lane + 32 * h < top) W.stk[k + lane + 32 * h] = keep[h];
                    for (int j = lane; j < k; j += 32) W.stk[j] = __ldcg(gstk + gtop - k + j);
                    gtop -= k;
                    top += k;
                    __syncwarp();
                }
                const int b = top < batch ? top : batch;
                pop_budget -= b;
                if (pop_budget < 0) {
                    if (lane == 0) atomicOr(status, GCS_DEV_TREE_MALFORMED);
                    break;
                }
                top -= b;
                // 1-2. fetch and classify nodes lane and lane+32
                int code_a[H], code_b[H], cls[H];
                uint32_t my_mask[H][T];
                float4 com[H];
                float w2[H];
#pragma unroll
                for (int h = 0; h < H; ++h) {
                    const int j = lane + 32 * h;
                    code_a[h] = 0;
                    code_b[h] = kWalkSkipTag;
                    cls[h] = kClassNone;
#pragma unroll
                    for (int t = 0; t < T; ++t) my_mask[h][t] = 0u;
                    com[h] = make_float4(0.f, 0.f, 0.f, 0.f);
                    w2[h] = 0.0f;
                    if (j < b) {
                        const Entry e = W.stk[top + j];
                        const float4* np = reinterpret_cast<const float4*>(wn + e.x);
                        const float4 a = __ldg(np);
                        const int4 k = __ldg(reinterpret_cast<const int4*>(np + 1));
                        w2[h] = __int_as_float(k.x);
                        code_a[h] = k.y;
                        code_b[h] = k.z;
                        com[h] = a;
                        entry_masks(e, my_mask[h]);
                        bool full = true;
#pragma unroll
                        for (int t = 0; t < T; ++t) full = full && my_mask[h][t] == live[t];
                        cls[h] = box_class(a, w2[h], box_lo, box_hi, eps2, k_take, k_open);
                        if (cls[h] == kClassTake && full) cls[h] = kClassTakeFull;
                    }
                }
                // compact into three pair-interleaved lists, each starting at
                // an even slot: take nodes with every live target in their
                // masks, other take nodes, mixed nodes; odd lists end with an
                // empty entry
                uint32_t bf[H], bt[H], bm[H];
                int n_full = 0, n_take = 0, n_mixed = 0;
#pragma unroll
                for (int h = 0; h < H; ++h) {
                    bf[h] = __ballot_sync(kFull, cls[h] == kClassTakeFull);
                    bt[h] = __ballot_sync(kFull, cls[h] == kClassTake);
                    bm[h] = __ballot_sync(kFull, cls[h] == kClassMixed);
                    n_full += __popc(bf[h]);
                    n_take += __popc(bt[h]);
                    n_mixed += __popc(bm[h]);
                }
                const int take_base = (n_full + 1) & ~1;
                const int mixed_base = (take_base + n_take + 1) & ~1;
                int slot[H];
                {
                    int full_before = 0, take_before = 0, mixed_before = 0;
#pragma unroll
                    for (int h = 0; h < H; ++h) {
                        slot[h] = cls[h] == kClassTakeFull ? full_before + __popc(bf[h] & lt)
                                : cls[h] == kClassTake ? take_base + take_before + __popc(bt[h] & lt)
                                : cls[h] == kClassMixed ? mixed_base + mixed_before + __popc(bm[h] & lt) : -1;
                        full_before += __popc(bf[h]);
                        take_before += __popc(bt[h]);
                        mixed_before += __popc(bm[h]);
                        if (slot[h] >= 0) {
                            put_pair(W.pxy, W.pzm, slot[h], com[h]);
#pragma unroll
                            for (int t = 0; t < T; ++t) put_mask(W.pmask[t], slot[h], my_mask[h][t]);
                            reinterpret_cast<float*>(W.pw2 + (slot[h] >> 1))[slot[h] & 1] = w2[h];
                        }
                    }
                    const float4 empty = make_float4(1e30f, 1e30f, 1e30f, 0.0f);
                    const int pad = lane == 0 ? ((n_full & 1) ? n_full : -1)
                                  : lane == 1 ? ((n_take & 1) ? take_base + n_take : -1)
                                  : lane == 2 ? ((n_mixed & 1) ? mixed_base + n_mixed : -1) : -1;
                    if (pad >= 0) {
                        put_pair(W.pxy, W.pzm, pad, empty);
#pragma unroll
                        for (int t = 0; t < T; ++t) put_mask(W.pmask[t], pad, 0u);
                        reinterpret_cast<float*>(W.pw2 + (pad >> 1))[1] = 0.0f;
                    }
                }
                __syncwarp();
                if (kCount) {
                    WC.peak = max(WC.peak, (uint32_t)(top + b + gtop));
                    WC.w_node += (uint32_t)b;
                    WC.rounds += 1u;
                    WC.all_open += (uint32_t)(b - n_full - n_take - n_mixed);
                    WC.all_take += (uint32_t)(n_full + n_take);
                    WC.r_full += (uint32_t)n_full;
                    WC.r_part += (uint32_t)n_take;
                    WC.r_mixed += (uint32_t)n_mixed;
#pragma unroll
                    for (int h = 0; h < H; ++h) {
#pragma unroll
                        for (int t = 0; t < T; ++t) {
                            WC.l_part += warp_popc_sum(cls[h] == kClassTake, my_mask[h][t]);
                            WC.l_mixed += warp_popc_sum(cls[h] == kClassMixed, my_mask[h][t]);
                        }
                    }
                }
                // 3a. nodes every live target accepts: monopole terms, two
                // nodes per packed evaluation, no masks
#pragma unroll 4
                for (int q = 0; q < (take_base >> 1); ++q) {
                    const float4 zm = W.pzm[q];
                    const float4 xy = W.pxy[q];
#pragma unroll
                    for (int t = 0; t < T; ++t) {
                        const PairD d = pair_d_take(xy, zm, X.npx[t], X.npy[t], X.npz[t], e2);
                        pair_add<kPot>(A[t], d, zm, true, true);
                    }
                }
                if (kCount) {
#pragma unroll
                    for (int t = 0; t < T; ++t)
                        if (valid[t]) A[t].n_mono += (uint32_t)n_full;
                }
                // 3b. nodes accepted by every target of their masks
#pragma unroll 4
                for (int q = take_base >> 1; q < (mixed_base >> 1); ++q) {
                    const float4 zm = W.pzm[q];
                    const float4 xy = W.pxy[q];
#pragma unroll
                    for (int t = 0; t < T; ++t) {
                        const uint2 mk = W.pmask[t][q];
                        const PairD d = pair_d_take(xy, zm, X.npx[t], X.npy[t], X.npz[t], e2);
                        const bool use0 = (mk.x & lane_bit) != 0u, use1 = (mk.y & lane_bit) != 0u;
                        pair_add<kPot>(A[t], d, zm, use0, use1);
                        if (kCount) A[t].n_mono += (use0 ? 1u : 0u) + (use1 ? 1u : 0u);
                    }
                }
                // 3c. mixed nodes: each target's own test; lane 0 records the
                // ballots of opening lanes for the nodes' owners
#pragma unroll 2
                for (int q = mixed_base >> 1; q < ((mixed_base + n_mixed + 1) >> 1); ++q) {
                    const float4 zm = W.pzm[q];
                    const float4 xy = W.pxy[q];
                    const float2 w2q = W.pw2[q];
#pragma unroll
                    for (int t = 0; t < T; ++t) {
                        const uint2 mk = W.pmask[t][q];
                        const PairD d = pair_d(xy, zm, X.npx[t], X.npy[t], X.npz[t], e2);
                        const float2 lim = __fmul2_rn(d.d2, th2);  // accept_monopole: w^2 < d2 * theta^2
                        const bool act0 = (mk.x & lane_bit) != 0u, act1 = (mk.y & lane_bit) != 0u;
                        const bool take0 = w2q.x < lim.x, take1 = w2q.y < lim.y;
                        pair_add<kPot>(A[t], d, zm, act0 && take0, act1 && take1);
                        if (kCount) {
                            A[t].n_mono += (act0 && take0 ? 1u : 0u) + (act1 && take1 ? 1u : 0u);
                            WC.l_accept += (uint32_t)(__popc(__ballot_sync(kFull, act0 && take0)) +
                                                      __popc(__ballot_sync(kFull, act1 && take1)));
                        }
                        const uint32_t om0 = __ballot_sync(kFull, act0 && !take0);
                        const uint32_t om1 = __ballot_sync(kFull, act1 && !take1);
                        if (lane == 0) W.pnopen[t][q] = make_uint2(om0, om1);
                    }
                }
                __syncwarp();
                // 4. parallel push / append for the opened nodes
                uint32_t my_open[H][T];
                int n_push[H], n_src[H];
                int lane_push = 0, lane_src = 0;
#pragma unroll
                for (int h = 0; h < H; ++h) {
                    uint32_t any = 0u;
#pragma unroll
                    for (int t = 0; t < T; ++t) {
                        my_open[h][t] = cls[h] == kClassOpen ? my_mask[h][t]
                                      : (cls[h] == kClassMixed
                                             ? reinterpret_cast<const uint32_t*>(W.pnopen[t])[slot[h]] : 0u);
                        any |= my_open[h][t];
                    }
                    n_push[h] = 0;
                    n_src[h] = 0;
                    if (any != 0u && code_b[h] != kWalkSkipTag) {
                        if (code_b[h] >= kWalkBucketTag) {
                            n_src[h] = code_b[h] - kWalkBucketTag;
                        } else {
                            n_push[h] = (code_a[h] >= 0) + (code_b[h] >= 0);
                            n_src[h] = (code_a[h] < 0) + (code_b[h] < 0);
                        }
                    }
                    lane_push += n_push[h];
                    lane_src += n_src[h];
                }
                const uint32_t both = ((uint32_t)lane_push << 16) | (uint32_t)lane_src;
                const uint32_t excl = warp_exclusive_scan(both, lane);
                const uint32_t total = __shfl_sync(kFull, excl + both, 31);
                {
                    int at = top + (int)(excl >> 16);
#pragma unroll
                    for (int h = 0; h < H; ++h) {
                        if (n_push[h] > 0) {
                            if (code_a[h] >= 0) W.stk[at++] = make_entry(code_a[h], my_open[h]);
                            if (code_b[h] >= 0) W.stk[at++] = make_entry(code_b[h], my_open[h]);
                        }
                    }
                }
                top += (int)(total >> 16);
                // sources: this lane's [src_at, src_at + lane_src) of this
                // round's `add` new ones, appended in windows that fit the
                // list, flushing between windows
                const int src_at = (int)(excl & 0xFFFFu);
                const int add = (int)(total & 0xFFFFu);
                if (add > 0) {
                    // one descriptor per node with sources, lane-major like
                    // the sources themselves: the lanes before this one hold
                    // descriptors [0, before)
                    int before = 0, n_desc = 0;
#pragma unroll
                    for (int h = 0; h < H; ++h) {
                        const uint32_t bh = __ballot_sync(kFull, n_src[h] > 0);
                        before += __popc(bh & lt);
                        n_desc += __popc(bh);
                    }
                    {
                        int d = before, first = src_at;
#pragma unroll
                        for (int h = 0; h < H; ++h) {
                            if (n_src[h] > 0) {
                                W.sdesc[d] = make_int4(first, code_a[h], code_b[h], 0);
#pragma unroll
                                for (int t = 0; t < T; ++t)
                                    reinterpret_cast<uint32_t*>(W.pmask[t])[d] = my_open[h][t];
                                ++d;
                            }
                            first += n_src[h];
                        }
                    }
                    __syncwarp();
                    // the round's sources [0, add), appended in windows that
                    // fit the list (flushing between windows), one per lane
                    for (int base = 0; base < add;) {
                        if (nsrc == kSrcCap) {
                            flush_sources<H, T, kPot, kCount>(W, nsrc, lane, lane_bit, pos, G, X, e2, leaf_thr, A,
                                                              WC);
                            nsrc = 0;
                        }
                        const int window = min(kSrcCap - nsrc, add - base);
                        for (int j = base + lane; j < base + window; j += 32) {
                            // the last descriptor starting at or before j
                            int lo = 0, hi = n_desc - 1;
                            while (lo < hi) {
                                const int mid = (lo + hi + 1) >> 1;
                                if (W.sdesc[mid].x <= j) lo = mid;
                                else hi = mid - 1;
                            }
                            const int4 e = W.sdesc[lo];
                            const int r = j - e.x;  // r-th source of that node
                            const int particle = e.z >= kWalkBucketTag ? e.y + r
                                               : ((r == 0 && e.y < 0) ? ~e.y : ~e.z);
                            const int at = nsrc + (j - base);
                            W.srcp[at] = particle;
#pragma unroll
                            for (int t = 0; t < T; ++t)
                                W.srcm[t][at] = reinterpret_cast<const uint32_t*>(W.pmask[t])[lo];
                        }
                        nsrc += window;
                        base += window;
                    }
                }
                __syncwarp();
                if (nsrc >= 32) {
                    flush_sources<H, T, kPot, kCount>(W, nsrc, lane, lane_bit, pos, G, X, e2, leaf_thr, A, WC);
                    nsrc = 0;
                }
                // spill the shared stack's bottom before it can overflow
                if (top > Smem::kSpillAbove) {
                    if (gtop + kSpillCount <= gstack_cap) {
                        for (int j = lane; j < kSpillCount; j += 32) gstk[gtop + j] = W.stk[j];
                        gtop += kSpillCount;
                    } else if (lane == 0) {
                        atomicOr(status, GCS_DEV_WALK_STACK_OVERFLOW);
                    }
                    constexpr int kMove = (Smem::kStackCap - kSpillCount + 31) / 32;
                    const int rest = top - kSpillCount;  // <= kStackCap - kSpillCount
                    Entry mv[kMove];
#pragma unroll
                    for (int i = 0; i < kMove; ++i) {
                        const int j = lane + 32 * i;
                        mv[i] = j < rest ? W.stk[kSpillCount + j] : Entry{};
                    }
                    __syncwarp();
#pragma unroll
                    for (int i = 0; i < kMove; ++i) {
                        const int j = lane + 32 * i;
                        if (j < rest) W.stk[j] = mv[i];
                    }
                    top = rest;
                    if (kCount) WC.spills += 1u;
                    __syncwarp();
                }
            }
        }
        if (nsrc > 0) flush_sources<H, T, kPot, kCount>(W, nsrc, lane, lane_bit, pos, G, X, e2, leaf_thr, A, WC);
#pragma unroll
        for (int t = 0; t < T; ++t) {
            if (!valid[t]) continue;
            const int j = grp.start + lane + 32 * t;
            const int64_t i = fr.perm ? __ldg(fr.perm + j) : j;  // the target's particle
            const float4 a = make_float4(__fadd_rn(A[t].ax.x, A[t].ax.y), __fadd_rn(A[t].ay.x, A[t].ay.y),
                                         __fadd_rn(A[t].az.x, A[t].az.y), __fadd_rn(A[t].pot.x, A[t].pot.y));
            acc[i] = a;
            if (ep.vel_in) {
                // the step's kick/drift of this target, out of place, and its Star
                float4 p = __ldg(pos + i);
                float4 v = __ldg(ep.vel_in + i);
                kick_drift(p, v, a, ep.dt, ep.recolor);
                ep.pos_out[i] = p;
                ep.vel_out[i] = v;
                if (ep.stars) store_star(ep.stars, i, p, v);
            }
        }
        if (ep.vel_in && ep.host_flags) {
            // count the group in its chunk; the warp that completes the chunk
            // tells the host (every warp fences before counting, so a chunk
            // seen complete has all of its records written)
            __syncwarp();
            if (lane == 0) {
                __threadfence();
                // the chunk holding group g: the last boundary <= g
                int lo = 0, hi = ep.n_chunks - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (ep.chunk_bound[mid] <= g) lo = mid;
                    else hi = mid - 1;
                }
                const int k = lo;
                const int in_chunk = ep.chunk_bound[k + 1] - ep.chunk_bound[k];
                if (atomicAdd(ep.chunk_done + k, 1u) == (uint32_t)in_chunk - 1u) {
                    __threadfence_system();
                    *reinterpret_cast<volatile uint32_t*>(ep.host_flags + k) = ep.epoch;
                }
            }
        }
        if (kCount) {
            unsigned long long cm = 0ull, cp = 0ull;
#pragma unroll
            for (int t = 0; t < T; ++t) {
                cm += A[t].n_mono;
                cp += A[t].n_part;
            }
            for (int o = 16; o > 0; o >>= 1) {
                cm += __shfl_xor_sync(kFull, cm, o);
                cp += __shfl_xor_sync(kFull, cp, o);
            }
            if (lane == 0) {
                atomicAdd(counts, cm);
                atomicAdd(counts + 1, cp);
                atomicAdd(counts + 2, (unsigned long long)WC.w_node);
                atomicAdd(counts + 3, (unsigned long long)WC.w_src);
                atomicAdd(counts + 4, (unsigned long long)WC.rounds);
                atomicAdd(counts + 5, (unsigned long long)WC.spills);
                atomicAdd(counts + 6, (unsigned long long)WC.all_open);
                atomicAdd(counts + 7, (unsigned long long)WC.all_take);
                atomicMax(counts + 8, (unsigned long long)WC.peak);
                const uint32_t lu[8] = {WC.r_list, WC.r_full, WC.r_part, WC.r_mixed,
                                        WC.l_part, WC.l_mixed, WC.l_accept, WC.l_src};
#pragma unroll
                for (int k = 0; k < 8; ++k) atomicAdd(counts + 9 + k, (unsigned long long)lu[k]);
            }
        }
        __syncwarp();
    }
    // Work queue: queue[0] is the next group, queue[1] counts warps that
    // found it empty.  Every warp fetches past the end exactly once, so the
    // last of them knows no warp will touch the queue again and resets it.
    if (lane == 0) {
        const uint32_t total = gridDim.x * kWalkWarps;
        if (atomicAdd(queue + 1, 1u) == total - 1) {
            queue[0] = 0u;
            queue[1] = 0u;
            __threadfence();
        }
    }
}

// Group partition of full super-groups (WalkFrontier::perm): one warp per
// super-group, its kSuperTargets targets held 8 per lane (element i = lane *
// 8 + r in register r).  Each level halves every part: the part's box comes
// from the lane's 8 elements and a shuffle reduction over the part's lanes,
// and the part is sorted by its coordinate along the box's longest axis with
// a bitonic network (register pairs inside a lane, shuffles across lanes), so
// its lower and upper halves are the two sides of the median.  After `levels`
// levels the parts are the groups.  Keys are the coordinate's order-preserving
// bits with the low 8 replaced by the target's index: unique, so the
// partition is a deterministic function of the positions (targets whose
// coordinates agree to 24 bits split by index, which only moves the median).
constexpr int kPartWarps = 8;
constexpr int kPartPerLane = kSuperTargets / 32;
static_assert(kSuperTargets == 256 && kPartPerLane == 8, "8 targets per lane; keys carry 8-bit target indices");

__global__ void __launch_bounds__(kPartWarps * 32)
partition_kernel(const float4* __restrict__ pos, const SuperGroup* __restrict__ supers, int n_supers, int levels,
                 int32_t* __restrict__ perm) {
    __shared__ float sp[kPartWarps][3][kSuperTargets];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int sgi = blockIdx.x * kPartWarps + warp;
    if (sgi >= n_supers) return;
    const SuperGroup sg = supers[sgi];
    if (sg.count != kSuperTargets) {  // a partial super-group keeps Morton order
        for (int i = lane; i < sg.count; i += 32) perm[sg.start + i] = sg.start + i;
        return;
    }
    float(*P)[kSuperTargets] = sp[warp];
    for (int i = lane; i < kSuperTargets; i += 32) {
        const float4 p = __ldg(pos + sg.start + i);
        P[0][i] = p.x;
        P[1][i] = p.y;
        P[2][i] = p.z;
    }
    __syncwarp();
    int e[kPartPerLane];
#pragma unroll
    for (int r = 0; r < kPartPerLane; ++r) e[r] = lane * kPartPerLane + r;
    for (int level = 0; level < levels; ++level) {
        const int part = kSuperTargets >> level;
        const int part_lanes = part / kPartPerLane;
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
        for (int r = 0; r < kPartPerLane; ++r)
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float v = P[a][e[r]];
                lo[a] = fminf(lo[a], v);
                hi[a] = fmaxf(hi[a], v);
            }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            if (o < part_lanes) {
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    lo[a] = fminf(lo[a], __shfl_xor_sync(kFull, lo[a], o));
                    hi[a] = fmaxf(hi[a], __shfl_xor_sync(kFull, hi[a], o));
                }
            }
        }
        int ax = 0;
        float ext = hi[0] - lo[0];
        if (hi[1] - lo[1] > ext) {
            ax = 1;
            ext = hi[1] - lo[1];
        }
        if (hi[2] - lo[2] > ext) ax = 2;
        uint32_t key[kPartPerLane];
#pragma unroll
        for (int r = 0; r < kPartPerLane; ++r)
            key[r] = (float_to_ordered(P[ax][e[r]]) & 0xFFFFFF00u) | (uint32_t)e[r];
#pragma unroll
        for (int k = 2; k <= kSuperTargets; k <<= 1) {
            if (k > part) continue;  // uniform; the loops stay unrolled, register indices constant
#pragma unroll
            for (int j = k >> 1; j > 0; j >>= 1) {
                if (j >= kPartPerLane) {  // partner in lane ^ (j / 8), same register
                    const int lj = j / kPartPerLane;
                    const bool lower = (lane & lj) == 0;
#pragma unroll
                    for (int r = 0; r < kPartPerLane; ++r) {
                        const uint32_t other = __shfl_xor_sync(kFull, key[r], lj);
                        const bool ascending = ((lane * kPartPerLane + r) & k) == 0;
                        key[r] = (lower == ascending) ? min(key[r], other) : max(key[r], other);
                    }
                } else {  // partner in register r ^ j of this lane
#pragma unroll
                    for (int r = 0; r < kPartPerLane; ++r) {
                        if ((r & j) != 0) continue;
                        const bool ascending = ((lane * kPartPerLane + r) & k) == 0;
                        const uint32_t a = key[r], b = key[r | j];
                        key[r] = ascending ? min(a, b) : max(a, b);
                        key[r | j] = ascending ? max(a, b) : min(a, b);
                    }
                }
            }
        }
#pragma unroll
        for (int r = 0; r < kPartPerLane; ++r) e[r] = (int)(key[r] & 0xFFu);
    }
#pragma unroll
    for (int r = 0; r < kPartPerLane; ++r) perm[sg.start + lane * kPartPerLane + r] = sg.start + e[r];
}

// Frontier pass (WalkFrontier, gcs_internal.h): one warp per super-group
// walks the tree against the super-group's bounding box, up to 64 nodes per
// round (lane k classifies nodes k and k + 32 with box_class).  The pass is a
// chain of dependent rounds, about one per tree level, so wider rounds do not
// shorten it.  Certified
// take nodes are appended to the take list, undecided ones to the frontier,
// and nodes every target opens contribute their internal children to the
// stack and their particles (leaf children, or the whole range of a small
// node) to the source list.  Lists grow at offsets from warp ballots and
// scans; a list or stack that would overflow, or more pops than the segment
// has internal nodes, marks the super-group invalid (its groups then walk
// from the root), so nothing is written out of bounds.
constexpr int kFrontWarps = 4;  // 1,024 blocks for 4,096 super-groups: better spread over the SMs than 8
constexpr int kFrontStack = 1024;
constexpr int kFrontSlots = 2;  // nodes per lane per round

__global__ void __launch_bounds__(kFrontWarps * 32)
frontier_kernel(Layout L, const float4* __restrict__ pos, const WalkNode* __restrict__ wn, WalkFrontier fr,
                float eps2, float theta2, uint32_t* __restrict__ status) {
    __shared__ int32_t stk_all[kFrontWarps][kFrontStack];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int sgi = blockIdx.x * kFrontWarps + warp;
    if (sgi >= fr.n_supers) return;
    int32_t* stk = stk_all[warp];
    const uint32_t lt = (1u << lane) - 1u;
    const SuperGroup sg = fr.supers[sgi];
    float3 lo = make_float3(INFINITY, INFINITY, INFINITY), hi = make_float3(-INFINITY, -INFINITY, -INFINITY);
    for (int i = lane; i < sg.count; i += 32) {
        const float4 p = __ldg(pos + sg.start + i);
        lo = make_float3(fminf(lo.x, p.x), fminf(lo.y, p.y), fminf(lo.z, p.z));
        hi = make_float3(fmaxf(hi.x, p.x), fmaxf(hi.y, p.y), fmaxf(hi.z, p.z));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo.x = fminf(lo.x, __shfl_xor_sync(kFull, lo.x, o));
        lo.y = fminf(lo.y, __shfl_xor_sync(kFull, lo.y, o));
        lo.z = fminf(lo.z, __shfl_xor_sync(kFull, lo.z, o));
        hi.x = fmaxf(hi.x, __shfl_xor_sync(kFull, hi.x, o));
        hi.y = fmaxf(hi.y, __shfl_xor_sync(kFull, hi.y, o));
        hi.z = fmaxf(hi.z, __shfl_xor_sync(kFull, hi.z, o));
    }
    const float k_take = theta2 * kBoxLo, k_open = theta2 * kBoxHi;
    const int s = sg.seg;
    const int off = (int)__ldg(L.seg_off + s);
    const int seg_n = (int)__ldg(L.seg_off + s + 1) - off;
    int32_t* list = fr.list + (size_t)sgi * kSuperCap;
    int32_t* src = fr.src + (size_t)sgi * kSuperSrcCap;
    int n_take = 0, n_src = 0, n_front = 0;
    bool ok = true;
    if (seg_n >= 2) {
        int top = 1;
        if (lane == 0) stk[0] = off - s;
        __syncwarp();
        int budget = seg_n - 1;
        while (top > 0) {
            const int b = top < 32 * kFrontSlots ? top : 32 * kFrontSlots;
            budget -= b;
            if (budget < 0) {
                if (lane == 0) atomicOr(status, GCS_DEV_TREE_MALFORMED);
                ok = false;
                break;
            }
            top -= b;
            int node[kFrontSlots], cls[kFrontSlots], code_a[kFrontSlots], code_b[kFrontSlots];
#pragma unroll
            for (int h = 0; h < kFrontSlots; ++h) {
                node[h] = -1;
                cls[h] = kClassNone;
                code_a[h] = 0;
                code_b[h] = kWalkSkipTag;
                if (lane + 32 * h < b) {
                    node[h] = stk[top + lane + 32 * h];
                    const float4* np = reinterpret_cast<const float4*>(wn + node[h]);
                    const float4 a = __ldg(np);
                    const int4 k = __ldg(reinterpret_cast<const int4*>(np + 1));
                    code_a[h] = k.y;
                    code_b[h] = k.z;
                    cls[h] = box_class(a, __int_as_float(k.x), lo, hi, eps2, k_take, k_open);
                }
            }
            __syncwarp();
            uint32_t bt[kFrontSlots], bm[kFrontSlots];
            int add_take = 0, add_front = 0, lane_push = 0, lane_src = 0;
            int n_push[kFrontSlots], n_s[kFrontSlots];
#pragma unroll
            for (int h = 0; h < kFrontSlots; ++h) {
                bt[h] = __ballot_sync(kFull, cls[h] == kClassTake);
                bm[h] = __ballot_sync(kFull, cls[h] == kClassMixed);
                add_take += __popc(bt[h]);
                add_front += __popc(bm[h]);
                n_push[h] = 0;
                n_s[h] = 0;
                if (cls[h] == kClassOpen && code_b[h] != kWalkSkipTag) {
                    if (code_b[h] >= kWalkBucketTag) {
                        n_s[h] = code_b[h] - kWalkBucketTag;
                    } else {
                        n_push[h] = (code_a[h] >= 0) + (code_b[h] >= 0);
                        n_s[h] = (code_a[h] < 0) + (code_b[h] < 0);
                    }
                }
                lane_push += n_push[h];
                lane_src += n_s[h];
            }
            const uint32_t both = ((uint32_t)lane_push << 16) | (uint32_t)lane_src;
            const uint32_t excl = warp_exclusive_scan(both, lane);
            const uint32_t total = __shfl_sync(kFull, excl + both, 31);
            const int push_total = (int)(total >> 16), src_total = (int)(total & 0xFFFFu);
            if (n_take + n_front + add_take + add_front > kSuperCap || n_src + src_total > kSuperSrcCap ||
                top + push_total > kFrontStack) {
                ok = false;
                break;
            }
            int take_before = 0, front_before = 0;
            int at = top + (int)(excl >> 16), sat = n_src + (int)(excl & 0xFFFFu);
#pragma unroll
            for (int h = 0; h < kFrontSlots; ++h) {
                if (cls[h] == kClassTake) list[n_take + take_before + __popc(bt[h] & lt)] = node[h];
                if (cls[h] == kClassMixed)
                    list[kSuperCap - 1 - (n_front + front_before + __popc(bm[h] & lt))] = node[h];
                take_before += __popc(bt[h]);
                front_before += __popc(bm[h]);
                if (n_push[h] > 0) {
                    if (code_a[h] >= 0) stk[at++] = code_a[h];
                    if (code_b[h] >= 0) stk[at++] = code_b[h];
                }
                if (n_s[h] > 0) {
                    if (code_b[h] >= kWalkBucketTag) {
                        for (int r = 0; r < n_s[h]; ++r) src[sat + r] = code_a[h] + r;
                        sat += n_s[h];
                    } else {
                        if (code_a[h] < 0) src[sat++] = ~code_a[h];
                        if (code_b[h] < 0) src[sat++] = ~code_b[h];
                    }
                }
            }
            n_take += add_take;
            n_front += add_front;
            top += push_total;
            n_src += src_total;
            __syncwarp();
        }
    }
    if (lane == 0) fr.meta[sgi] = make_int4(n_take, n_src, n_front, ok ? 1 : 0);
}

template <int H, int T>
constexpr size_t smem_bytes() {
    return sizeof(WarpSmem<H, T>) * kWalkWarps;
}

// Opt the instantiation in to its dynamic shared memory (above 48 KB), once
// per device.
template <int H, int T, bool kPot, bool kCount>
void configure() {
    static std::once_flag done[kMaxDevices];
    once_per_device(done, [] {
        cudaFuncSetAttribute(walk_kernel<H, T, kPot, kCount>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_bytes<H, T>());
    });
}

template <int H, int T, bool kPot, bool kCount>
int occupancy_of() {
    configure<H, T, kPot, kCount>();
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, walk_kernel<H, T, kPot, kCount>, kWalkThreads,
                                                  smem_bytes<H, T>());
    return nb > 0 ? nb : 1;
}

template <int T>
int max_blocks_of(int batch, int with_potential) {
    // per device (the query needs the device's attribute opt-in first)
    static std::atomic<int> cached[kMaxDevices][2][2] = {};
    const int hi = batch > 32 ? 1 : 0, pot = with_potential ? 1 : 0;
    const int dev = current_device();
    if (dev >= 0 && dev < kMaxDevices) {
        const int v = cached[dev][hi][pot].load(std::memory_order_relaxed);
        if (v > 0) return v;
    }
    int nb;
    if (hi) nb = pot ? occupancy_of<2, T, true, false>() : occupancy_of<2, T, false, false>();
    else nb = pot ? occupancy_of<1, T, true, false>() : occupancy_of<1, T, false, false>();
    if (dev >= 0 && dev < kMaxDevices) cached[dev][hi][pot].store(nb, std::memory_order_relaxed);
    return nb;
}

}  // namespace

int walk_max_blocks_per_sm(int batch, int with_potential, int targets_per_lane) {
    return targets_per_lane > 1 ? max_blocks_of<2>(batch, with_potential) : max_blocks_of<1>(batch, with_potential);
}

int64_t walk_grid_blocks(int n_groups, int blocks_per_sm, int sm_count, int with_potential) {
    int max_b = 0;
    for (int t = 1; t <= 2; ++t)
        max_b = std::max(max_b, std::max(walk_max_blocks_per_sm(32, with_potential, t),
                                         walk_max_blocks_per_sm(64, with_potential, t)));
    const int bps = blocks_per_sm > 0 && blocks_per_sm < max_b ? blocks_per_sm : max_b;
    int64_t grid = (int64_t)sm_count * bps;
    const int64_t need = ((int64_t)n_groups + kWalkWarps - 1) / kWalkWarps;
    if (grid > need) grid = need;
    return grid < 1 ? 1 : grid;
}

size_t walk_stack_entries(int64_t grid_blocks) {
    return (size_t)grid_blocks * kWalkWarps * (size_t)kWalkGlobalStack;
}

template <int H, int T>
static void launch_ht(const Layout& L, const WalkParams& q, const float4* pos, const WalkNode* wn,
                      const WalkGroup* groups, int n_groups, float4* acc, uint32_t* queue, uint32_t* status,
                      unsigned long long* counts, int2* gstack, int cap, unsigned g, cudaStream_t st,
                      const WalkEpilogue& ep, const WalkFrontier& fr) {
    using Entry = typename EntryOf<T>::type;
    Entry* gs = reinterpret_cast<Entry*>(gstack);
    const size_t sm = smem_bytes<H, T>();
    if (counts) {
        if (q.with_potential) {
            configure<H, T, true, true>();
            walk_kernel<H, T, true, true><<<g, kWalkThreads, sm, st>>>(L, q, pos, wn, groups, n_groups, acc, queue,
                                                                       status, counts, gs, cap, ep, fr);
        } else {
            configure<H, T, false, true>();
            walk_kernel<H, T, false, true><<<g, kWalkThreads, sm, st>>>(L, q, pos, wn, groups, n_groups, acc, queue,
                                                                        status, counts, gs, cap, ep, fr);
        }
    } else if (q.with_potential) {
        configure<H, T, true, false>();
        walk_kernel<H, T, true, false><<<g, kWalkThreads, sm, st>>>(L, q, pos, wn, groups, n_groups, acc, queue,
                                                                    status, nullptr, gs, cap, ep, fr);
    } else {
        configure<H, T, false, false>();
        walk_kernel<H, T, false, false><<<g, kWalkThreads, sm, st>>>(L, q, pos, wn, groups, n_groups, acc, queue,
                                                                     status, nullptr, gs, cap, ep, fr);
    }
}

void launch_walk(const Layout& L, const WalkParams& wp, const float4* pos,
                 const WalkNode* wn, const WalkGroup* groups, int n_groups, int targets_per_lane, float4* acc,
                 uint32_t* queue, uint32_t* status, int blocks_per_sm, int sm_count,
                 unsigned long long* counts, int2* gstack, size_t gstack_entries, cudaStream_t st,
                 const WalkEpilogue& ep, const WalkFrontier& fr_in) {
    if (n_groups <= 0) return;
    WalkFrontier fr = fr_in;
    if (fr.supers && fr.n_supers > 0 && fr.list && fr.src && fr.meta) {
        const unsigned fb = (unsigned)((fr.n_supers + kFrontWarps - 1) / kFrontWarps);
        bool joined = false;
        if (fr.perm && fr.split_levels > 0) {
            const unsigned pb = (unsigned)((fr.n_supers + kPartWarps - 1) / kPartWarps);
            if (fr.side && fr.fork && fr.join && cudaEventRecord(fr.fork, st) == cudaSuccess &&
                cudaStreamWaitEvent(fr.side, fr.fork, 0) == cudaSuccess) {
                partition_kernel<<<pb, kPartWarps * 32, 0, fr.side>>>(pos, fr.supers, fr.n_supers, fr.split_levels,
                                                                      fr.perm);
                cudaEventRecord(fr.join, fr.side);
                joined = true;
            } else {
                partition_kernel<<<pb, kPartWarps * 32, 0, st>>>(pos, fr.supers, fr.n_supers, fr.split_levels,
                                                                 fr.perm);
            }
        } else {
            fr.perm = nullptr;
        }
        frontier_kernel<<<fb, kFrontWarps * 32, 0, st>>>(L, pos, wn, fr, wp.eps2, wp.theta2, status);
        if (joined) cudaStreamWaitEvent(st, fr.join, 0);
    } else {
        fr.meta = nullptr;  // every group walks from its root, targets in Morton order
        fr.perm = nullptr;
    }
    WalkParams q = wp;
    if (q.batch < 1) q.batch = 1;
    if (q.batch > kWalkMaxBatch) q.batch = kWalkMaxBatch;
    if (q.leaf_size < 1) q.leaf_size = 1;
    if (q.leaf_size > 32) q.leaf_size = 32;
    const int T = targets_per_lane > 1 ? 2 : 1;
    const int max_b = walk_max_blocks_per_sm(q.batch, q.with_potential, T);
    const int bps = blocks_per_sm > 0 && blocks_per_sm < max_b ? blocks_per_sm : max_b;
    int64_t grid = (int64_t)sm_count * bps;
    const int64_t need = ((int64_t)n_groups + kWalkWarps - 1) / kWalkWarps;
    if (grid > need) grid = need;
    // never more warps than the global stack regions provided: the int2
    // buffer holds kWalkGlobalStack 8-byte units per warp; a T = 2 entry
    // takes two of them
    const int64_t fit = (int64_t)(gstack_entries / ((size_t)kWalkWarps * kWalkGlobalStack));
    if (grid > fit) grid = fit;
    if (grid < 1) return;  // no stack regions: nothing can run (the engine always provides them)
    const unsigned g = (unsigned)grid;
    // entries per warp region: the whole buffer split over this grid's warps
    const size_t units = gstack_entries / ((size_t)grid * kWalkWarps);
    const int cap = (int)(std::min<size_t>(units, (size_t)1 << 24) / (size_t)T);
    if (T == 2) {
        if (q.batch > 32)
            launch_ht<2, 2>(L, q, pos, wn, groups, n_groups, acc, queue, status, counts, gstack, cap, g, st, ep, fr);
        else
            launch_ht<1, 2>(L, q, pos, wn, groups, n_groups, acc, queue, status, counts, gstack, cap, g, st, ep, fr);
    } else if (q.batch > 32) {
        launch_ht<2, 1>(L, q, pos, wn, groups, n_groups, acc, queue, status, counts, gstack, cap, g, st, ep, fr);
    } else {
        launch_ht<1, 1>(L, q, pos, wn, groups, n_groups, acc, queue, status, counts, gstack, cap, g, st, ep, fr);
    }
}

}  // namespace gcs
