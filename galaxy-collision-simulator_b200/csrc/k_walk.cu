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
// Execution: a persistent grid of warps pulls groups of <= 32 consecutive
// (Morton-adjacent) targets of one segment from a global work queue.  The
// warp walks the tree once for its group with one stack; each stack entry
// carries the mask of lanes that still need that subtree, and each lane
// takes its own opening decision, so the group walk is the union of the 32
// per-target walks with no change to any target's terms.  Each round:
//   1. up to `batch` (<= 32*H) entries are popped; lane k fetches nodes k and
//      k+32 (two 16-byte loads each) and digests them: G*mass, width^2, and
//      either the particle range to sum (a node of <= L particles) or its two
//      children coded as node or particle;
//   2. each node is classified against the group's bounding box with a
//      2^-16 relative margin: "take" if every lane of the box must accept
//      it, "open" if every lane must open it, else "mixed" (the margin is far
//      above the few-ulp rounding of any lane's own d2, so a class never
//      contradicts a lane's own test);
//   3. take nodes go through a monopole-only loop, mixed nodes through the
//      per-lane opening test (a predicated monopole and a ballot of opening
//      lanes), open nodes skip evaluation altogether;
//   4. in parallel, each lane pushes its nodes' internal children and
//      appends their particle sources (leaf children, or the whole range of
//      a small node) at offsets from one warp prefix scan;
//   5. particle sources accumulate in a per-warp list; when it fills, the
//      lanes fetch up to 64 source records in parallel into shared memory and
//      every lane sums them.
// The stack's top lives in shared memory; when it passes a threshold its
// bottom is spilled to a per-warp region of global memory (L2) and read back
// when the top runs low, so batches are never throttled and the logical
// stack order is that of an unbounded stack.  A global region that would
// overflow sets GCS_DEV_WALK_STACK_OVERFLOW (entries are dropped, nothing is
// written out of bounds); a walk that pops more nodes than the tree holds
// stops with GCS_DEV_TREE_MALFORMED.  The work queue resets itself: the last
// warp to find it empty zeroes it.
#include <algorithm>

#include "gcs_internal.h"
#include "device_math.cuh"

namespace gcs {

namespace {

constexpr int kWalkWarps = 8;
constexpr int kWalkThreads = kWalkWarps * 32;
constexpr int kSpillCount = 128;  // entries moved per spill / refill
constexpr int kSrcCap = 64;
constexpr uint32_t kFull = 0xFFFFFFFFu;
// Digested node codes (code_a / code_b):
//   code_b >= kBucketTag   the node itself is summed directly: particles
//                          [code_a, code_a + code_b - kBucketTag)
//   code_b == kSkipTag     no node, or malformed children: nothing pushed
//   otherwise              children: >= 0 internal node, < 0 particle ~code
constexpr int kBucketTag = 1 << 30;
constexpr int kSkipTag = 0x7FFFFFFF;

// Classes of a batch node against the group's bounding box.
constexpr int kClassNone = 0;   // lane holds no node
constexpr int kClassTake = 1;   // every lane of the group accepts it
constexpr int kClassOpen = 2;   // every lane of the group opens it
constexpr int kClassMixed = 3;  // lanes decide one by one
constexpr float kBoxLo = 1.0f - 1.0f / 65536.0f;
constexpr float kBoxHi = 1.0f + 1.0f / 65536.0f;

// Per-warp shared memory for H nodes per lane per round.
template <int H>
struct WarpSmem {
    static constexpr int kBatch = 32 * H;
    static constexpr int kStackCap = 256 + 64 * H;                 // stack entries
    static constexpr int kSpillAbove = kStackCap - 2 * kBatch;     // a round pushes <= 2*batch
    int2 stk[kStackCap];          // node, lane mask
    float4 nc[kBatch];            // com x, y, z, G*mass (compacted: take, then mixed)
    uint2 nw[kBatch];             // bits of width^2, lane mask
    uint32_t nopen[kBatch];       // opening lanes of each mixed node
    float4 src[kSrcCap];          // x, y, z, G*mass
    int2 srcm[kSrcCap];           // particle, lane mask
};

// Resident blocks per SM the register budget is set for (H=1: 48 registers
// a thread, 40 warps; H=2: 64 registers, 32 warps).
template <int H>
struct WalkOcc {
    static constexpr int kMinBlocks = H == 1 ? 5 : 4;
};

struct Accum {
    float ax, ay, az, pot;
    uint32_t n_mono, n_part;      // interaction counts (count mode only)
    uint32_t w_node, w_src;       // warp-wide node / source evaluations (count mode only)
    uint32_t rounds, spills;      // pop rounds, stack spills to global memory
    uint32_t all_open, all_take;  // nodes classified open / take by the box test
};

// Sum the listed particle sources into every lane whose bit is in the
// source's mask (leaf rule: skip d2 <= 1.01 eps^2).
template <int H, bool kPot, bool kCount>
__device__ __forceinline__ void flush_sources(WarpSmem<H>& W, int nsrc, int lane, uint32_t lane_bit,
                                              const float4* __restrict__ pos, float G, float4 p,
                                              float eps2, float leaf_thr, Accum& A) {
    __syncwarp();
    for (int e = lane; e < nsrc; e += 32) {
        float4 q = __ldg(pos + W.srcm[e].x);
        q.w = __fmul_rn(G, q.w);
        W.src[e] = q;
    }
    __syncwarp();
#pragma unroll 4
    for (int e = 0; e < nsrc; ++e) {
        const float4 q = W.src[e];
        const uint32_t m = (uint32_t)W.srcm[e].y;
        const float dx = __fsub_rn(q.x, p.x);
        const float dy = __fsub_rn(q.y, p.y);
        const float dz = __fsub_rn(q.z, p.z);
        const float d2 = softened_d2(dx, dy, dz, eps2);
        const bool use = (m & lane_bit) && (d2 > leaf_thr);
        const float inv = rsqrt_approx(d2);
        const float inv3 = __fmul_rn(__fmul_rn(inv, inv), inv);
        const float f = use ? __fmul_rn(q.w, inv3) : 0.0f;
        A.ax = __fmaf_rn(dx, f, A.ax);
        A.ay = __fmaf_rn(dy, f, A.ay);
        A.az = __fmaf_rn(dz, f, A.az);
        if (kPot) A.pot = use ? __fmaf_rn(-q.w, inv, A.pot) : A.pot;
        if (kCount) A.n_part += use ? 1u : 0u;
    }
    if (kCount) A.w_src += (uint32_t)nsrc;
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

template <int H, bool kPot, bool kCount>
__global__ void __launch_bounds__(kWalkThreads, WalkOcc<H>::kMinBlocks)
walk_kernel(Layout L, WalkParams wp, const float4* __restrict__ pos,
            const BvhNodeTraverse* __restrict__ tr, const WalkGroup* __restrict__ groups,
            int n_groups, float4* __restrict__ acc, uint32_t* __restrict__ queue,
            uint32_t* __restrict__ status, unsigned long long* __restrict__ counts,
            int2* __restrict__ gstack, int gstack_cap) {
    using Smem = WarpSmem<H>;
    extern __shared__ __align__(16) unsigned char walk_smem[];
    const int warp = threadIdx.x >> 5;
    Smem& W = reinterpret_cast<Smem*>(walk_smem)[warp];
    int2* const gstk = gstack + ((size_t)blockIdx.x * kWalkWarps + warp) * (size_t)gstack_cap;
    const int lane = threadIdx.x & 31;
    const uint32_t lane_bit = 1u << lane;
    const uint32_t lt = lane_bit - 1u;
    const float G = wp.G, eps2 = wp.eps2, theta2 = wp.theta2;
    const float leaf_thr = __fmul_rn(eps2, 1.01f);
    const int leaf_size = wp.leaf_size;
    const int batch = wp.batch;
    const int n_internal = L.n_internal;
    const int n_total = L.n;

    for (;;) {
        int g = 0;
        if (lane == 0) g = (int)atomicAdd(queue, 1u);
        g = __shfl_sync(kFull, g, 0);
        if (g >= n_groups) break;
        const WalkGroup grp = groups[g];
        const bool valid = lane < grp.count;
        const int t = grp.start + lane;
        const float4 p = valid ? __ldg(pos + t) : make_float4(0.f, 0.f, 0.f, 0.f);
        const uint32_t live = __ballot_sync(kFull, valid);
        // bounding box of the group's targets
        float3 box_lo = valid ? make_float3(p.x, p.y, p.z) : make_float3(INFINITY, INFINITY, INFINITY);
        float3 box_hi = valid ? make_float3(p.x, p.y, p.z) : make_float3(-INFINITY, -INFINITY, -INFINITY);
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
        const int seg_end = off + seg_n;
        Accum A = {0.f, 0.f, 0.f, 0.f, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
        int nsrc = 0;

        if (seg_n >= 2) {
            int top = 1, gtop = 0;
            if (lane == 0) W.stk[0] = make_int2(off - s, (int)live);
            __syncwarp();
            // Each internal node has one parent, so a walk pops it at most
            // once: more pops than internal nodes means a malformed tree.
            int pop_budget = seg_n - 1;
            while (top > 0 || gtop > 0) {
                // refill the shared top from the global bottom when it runs low
                if (top < batch && gtop > 0) {
                    const int k = gtop < kSpillCount ? gtop : kSpillCount;
                    int2 keep[H];
#pragma unroll
                    for (int h = 0; h < H; ++h)
                        keep[h] = lane + 32 * h < top ? W.stk[lane + 32 * h] : make_int2(0, 0);
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
                // 1-2. fetch, digest and classify nodes lane and lane+32
                int code_a[H], code_b[H], cls[H];
                uint32_t my_mask[H];
                float4 com[H];
                float w2[H];
#pragma unroll
                for (int h = 0; h < H; ++h) {
                    const int j = lane + 32 * h;
                    code_a[h] = 0;
                    code_b[h] = kSkipTag;
                    cls[h] = kClassNone;
                    my_mask[h] = 0u;
                    com[h] = make_float4(0.f, 0.f, 0.f, 0.f);
                    w2[h] = 0.0f;
                    if (j < b) {
                        const int2 e = W.stk[top + j];
                        const float4* np = reinterpret_cast<const float4*>(tr + e.x);
                        float4 a = __ldg(np);
                        const float4 c = __ldg(np + 1);
                        a.w = __fmul_rn(G, a.w);
                        const int own = e.x + s;  // particle index at this end of the range
                        const int re = __float_as_int(c.w);
                        const int lo = max(min(own, re), off);
                        const int cnt = min(max(own, re), seg_end - 1) - lo + 1;
                        if (cnt <= leaf_size) {
                            code_a[h] = lo;
                            code_b[h] = kBucketTag + max(cnt, 0);
                        } else {
                            const int cl = __float_as_int(c.y), cr = __float_as_int(c.z);
                            if (cl >= 0 && cl < n_internal + n_total && cr >= 0 && cr < n_internal + n_total) {
                                code_a[h] = cl >= n_internal ? ~(cl - n_internal) : cl;
                                code_b[h] = cr >= n_internal ? ~(cr - n_internal) : cr;
                            } else {
                                atomicOr(status, GCS_DEV_BUILD_RANGE);
                            }
                        }
                        w2[h] = __fmul_rn(c.x, c.x);
                        com[h] = a;
                        my_mask[h] = (uint32_t)e.y;
                        float s2min = 0.0f, s2max = 0.0f;
                        {
                            const float dl[3] = {box_lo.x - a.x, box_lo.y - a.y, box_lo.z - a.z};
                            const float dh[3] = {a.x - box_hi.x, a.y - box_hi.y, a.z - box_hi.z};
#pragma unroll
                            for (int ax = 0; ax < 3; ++ax) {
                                const float near = fmaxf(fmaxf(dl[ax], dh[ax]), 0.0f);
                                const float far = fmaxf(fabsf(dl[ax]), fabsf(dh[ax]));
                                s2min = fmaf(near, near, s2min);
                                s2max = fmaf(far, far, s2max);
                            }
                        }
                        if (w2[h] < theta2 * (s2min + eps2) * kBoxLo) cls[h] = kClassTake;
                        else if (w2[h] >= theta2 * (s2max + eps2) * kBoxHi) cls[h] = kClassOpen;
                        else cls[h] = kClassMixed;
                    }
                }
                // compact: take nodes first, then mixed ones
                uint32_t bt[H], bm[H];
                int n_take = 0, n_mixed = 0;
#pragma unroll
                for (int h = 0; h < H; ++h) {
                    bt[h] = __ballot_sync(kFull, cls[h] == kClassTake);
                    bm[h] = __ballot_sync(kFull, cls[h] == kClassMixed);
                    n_take += __popc(bt[h]);
                    n_mixed += __popc(bm[h]);
                }
                int slot[H];
                {
                    int take_before = 0, mixed_before = 0;
#pragma unroll
                    for (int h = 0; h < H; ++h) {
                        slot[h] = cls[h] == kClassTake ? take_before + __popc(bt[h] & lt)
                                : (cls[h] == kClassMixed ? n_take + mixed_before + __popc(bm[h] & lt) : -1);
                        take_before += __popc(bt[h]);
                        mixed_before += __popc(bm[h]);
                        if (slot[h] >= 0) {
                            W.nc[slot[h]] = com[h];
                            W.nw[slot[h]] = make_uint2(__float_as_uint(w2[h]), my_mask[h]);
                        }
                    }
                }
                __syncwarp();
                if (kCount) {
                    A.w_node += (uint32_t)b;
                    A.rounds += 1u;
                    A.all_open += (uint32_t)(b - n_take - n_mixed);
                    A.all_take += (uint32_t)n_take;
                }
                // 3a. nodes every lane accepts: monopole terms only
#pragma unroll 2
                for (int k = 0; k < n_take; ++k) {
                    const float4 a = W.nc[k];
                    const bool active = (W.nw[k].y & lane_bit) != 0u;
                    const float dx = __fsub_rn(a.x, p.x);
                    const float dy = __fsub_rn(a.y, p.y);
                    const float dz = __fsub_rn(a.z, p.z);
                    const float d2 = softened_d2(dx, dy, dz, eps2);
                    const float inv = rsqrt_approx(d2);
                    const float inv3 = __fmul_rn(__fmul_rn(inv, inv), inv);
                    const float f = active ? __fmul_rn(a.w, inv3) : 0.0f;
                    A.ax = __fmaf_rn(dx, f, A.ax);
                    A.ay = __fmaf_rn(dy, f, A.ay);
                    A.az = __fmaf_rn(dz, f, A.az);
                    if (kPot) A.pot = active ? __fmaf_rn(-a.w, inv, A.pot) : A.pot;
                    if (kCount) A.n_mono += active ? 1u : 0u;
                }
                // 3b. mixed nodes: each lane's own test; lane 0 records the
                // ballot of opening lanes for the node's owner
                for (int k = n_take; k < n_take + n_mixed; ++k) {
                    const float4 a = W.nc[k];
                    const uint2 wm = W.nw[k];
                    const bool active = (wm.y & lane_bit) != 0u;
                    const float dx = __fsub_rn(a.x, p.x);
                    const float dy = __fsub_rn(a.y, p.y);
                    const float dz = __fsub_rn(a.z, p.z);
                    const float d2 = softened_d2(dx, dy, dz, eps2);
                    const bool take = accept_monopole(__uint_as_float(wm.x), d2, theta2);
                    const bool mono = active && take;
                    const float inv = rsqrt_approx(d2);
                    const float inv3 = __fmul_rn(__fmul_rn(inv, inv), inv);
                    const float f = mono ? __fmul_rn(a.w, inv3) : 0.0f;
                    A.ax = __fmaf_rn(dx, f, A.ax);
                    A.ay = __fmaf_rn(dy, f, A.ay);
                    A.az = __fmaf_rn(dz, f, A.az);
                    if (kPot) A.pot = mono ? __fmaf_rn(-a.w, inv, A.pot) : A.pot;
                    if (kCount) A.n_mono += mono ? 1u : 0u;
                    const uint32_t om = __ballot_sync(kFull, active && !take);
                    if (lane == 0) W.nopen[k] = om;
                }
                __syncwarp();
                // 4. parallel push / append for the opened nodes
                uint32_t my_open[H];
                int n_push[H], n_src[H];
                int lane_push = 0, lane_src = 0;
#pragma unroll
                for (int h = 0; h < H; ++h) {
                    my_open[h] = cls[h] == kClassOpen ? my_mask[h]
                               : (cls[h] == kClassMixed ? W.nopen[slot[h]] : 0u);
                    n_push[h] = 0;
                    n_src[h] = 0;
                    if (my_open[h] != 0u && code_b[h] != kSkipTag) {
                        if (code_b[h] >= kBucketTag) {
                            n_src[h] = code_b[h] - kBucketTag;
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
                            if (code_a[h] >= 0) W.stk[at++] = make_int2(code_a[h], (int)my_open[h]);
                            if (code_b[h] >= 0) W.stk[at++] = make_int2(code_b[h], (int)my_open[h]);
                        }
                    }
                }
                top += (int)(total >> 16);
                // sources: this lane's [src_at, src_at + lane_src) of this
                // round's `add` new ones, appended in windows that fit the
                // list, flushing between windows
                const int src_at = (int)(excl & 0xFFFFu);
                const int add = (int)(total & 0xFFFFu);
                for (int base = 0; base < add;) {
                    if (nsrc == kSrcCap) {
                        flush_sources<H, kPot, kCount>(W, nsrc, lane, lane_bit, pos, G, p, eps2, leaf_thr, A);
                        nsrc = 0;
                    }
                    const int window = min(kSrcCap - nsrc, add - base);
                    int first = src_at;  // this lane's first source index in the round
#pragma unroll
                    for (int h = 0; h < H; ++h) {
                        const int j0 = max(first, base), j1 = min(first + n_src[h], base + window);
                        for (int j = j0; j < j1; ++j) {
                            const int r = j - first;  // r-th source of node h
                            int particle;
                            if (code_b[h] >= kBucketTag) particle = code_a[h] + r;
                            else particle = (r == 0 && code_a[h] < 0) ? ~code_a[h] : ~code_b[h];
                            W.srcm[nsrc + (j - base)] = make_int2(particle, (int)my_open[h]);
                        }
                        first += n_src[h];
                    }
                    nsrc += window;
                    base += window;
                }
                __syncwarp();
                if (nsrc >= 32) {
                    flush_sources<H, kPot, kCount>(W, nsrc, lane, lane_bit, pos, G, p, eps2, leaf_thr, A);
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
                    int2 mv[kMove];
#pragma unroll
                    for (int i = 0; i < kMove; ++i) {
                        const int j = lane + 32 * i;
                        mv[i] = j < rest ? W.stk[kSpillCount + j] : make_int2(0, 0);
                    }
                    __syncwarp();
#pragma unroll
                    for (int i = 0; i < kMove; ++i) {
                        const int j = lane + 32 * i;
                        if (j < rest) W.stk[j] = mv[i];
                    }
                    top = rest;
                    if (kCount) A.spills += 1u;
                    __syncwarp();
                }
            }
        }
        if (nsrc > 0) flush_sources<H, kPot, kCount>(W, nsrc, lane, lane_bit, pos, G, p, eps2, leaf_thr, A);
        if (valid) acc[t] = make_float4(A.ax, A.ay, A.az, A.pot);
        if (kCount) {
            unsigned long long cm = A.n_mono, cp = A.n_part;
            for (int o = 16; o > 0; o >>= 1) {
                cm += __shfl_xor_sync(kFull, cm, o);
                cp += __shfl_xor_sync(kFull, cp, o);
            }
            if (lane == 0) {
                atomicAdd(counts, cm);
                atomicAdd(counts + 1, cp);
                atomicAdd(counts + 2, (unsigned long long)A.w_node);
                atomicAdd(counts + 3, (unsigned long long)A.w_src);
                atomicAdd(counts + 4, (unsigned long long)A.rounds);
                atomicAdd(counts + 5, (unsigned long long)A.spills);
                atomicAdd(counts + 6, (unsigned long long)A.all_open);
                atomicAdd(counts + 7, (unsigned long long)A.all_take);
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

template <int H>
constexpr size_t smem_bytes() {
    return sizeof(WarpSmem<H>) * kWalkWarps;
}

// Opt the instantiation in to its dynamic shared memory (above 48 KB for H=2).
template <int H, bool kPot, bool kCount>
void configure() {
    static bool done = false;
    if (!done) {
        cudaFuncSetAttribute(walk_kernel<H, kPot, kCount>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_bytes<H>());
        done = true;
    }
}

template <int H, bool kPot, bool kCount>
int occupancy_of() {
    configure<H, kPot, kCount>();
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, walk_kernel<H, kPot, kCount>, kWalkThreads,
                                                  smem_bytes<H>());
    return nb > 0 ? nb : 1;
}

}  // namespace

int walk_max_blocks_per_sm(int batch, int with_potential) {
    // the same for every device of this build (sm_100a only)
    static int cached[2][2] = {{0, 0}, {0, 0}};
    const int hi = batch > 32 ? 1 : 0, pot = with_potential ? 1 : 0;
    int& nb = cached[hi][pot];
    if (nb == 0) {
        if (hi) nb = pot ? occupancy_of<2, true, false>() : occupancy_of<2, false, false>();
        else nb = pot ? occupancy_of<1, true, false>() : occupancy_of<1, false, false>();
    }
    return nb;
}

int64_t walk_grid_blocks(int n_groups, int blocks_per_sm, int sm_count, int with_potential) {
    const int max_b = std::max(walk_max_blocks_per_sm(32, with_potential), walk_max_blocks_per_sm(64, with_potential));
    const int bps = blocks_per_sm > 0 && blocks_per_sm < max_b ? blocks_per_sm : max_b;
    int64_t grid = (int64_t)sm_count * bps;
    const int64_t need = ((int64_t)n_groups + kWalkWarps - 1) / kWalkWarps;
    if (grid > need) grid = need;
    return grid < 1 ? 1 : grid;
}

size_t walk_stack_entries(int64_t grid_blocks) {
    return (size_t)grid_blocks * kWalkWarps * (size_t)kWalkGlobalStack;
}

template <int H>
static void launch_h(const Layout& L, const WalkParams& q, const float4* pos, const BvhNodeTraverse* tr,
                     const WalkGroup* groups, int n_groups, float4* acc, uint32_t* queue, uint32_t* status,
                     unsigned long long* counts, int2* gstack, unsigned g, cudaStream_t st) {
    const int cap = kWalkGlobalStack;
    const size_t sm = smem_bytes<H>();
    if (counts) {
        if (q.with_potential) {
            configure<H, true, true>();
            walk_kernel<H, true, true><<<g, kWalkThreads, sm, st>>>(L, q, pos, tr, groups, n_groups, acc, queue,
                                                                    status, counts, gstack, cap);
        } else {
            configure<H, false, true>();
            walk_kernel<H, false, true><<<g, kWalkThreads, sm, st>>>(L, q, pos, tr, groups, n_groups, acc,
                                                                     queue, status, counts, gstack, cap);
        }
    } else if (q.with_potential) {
        configure<H, true, false>();
        walk_kernel<H, true, false><<<g, kWalkThreads, sm, st>>>(L, q, pos, tr, groups, n_groups, acc, queue,
                                                                 status, nullptr, gstack, cap);
    } else {
        configure<H, false, false>();
        walk_kernel<H, false, false><<<g, kWalkThreads, sm, st>>>(L, q, pos, tr, groups, n_groups, acc, queue,
                                                                  status, nullptr, gstack, cap);
    }
}

void launch_walk(const Layout& L, const WalkParams& wp, const float4* pos,
                 const BvhNodeTraverse* tr, const WalkGroup* groups, int n_groups, float4* acc,
                 uint32_t* queue, uint32_t* status, int blocks_per_sm, int sm_count,
                 unsigned long long* counts, int2* gstack, size_t gstack_entries, cudaStream_t st) {
    if (n_groups <= 0) return;
    WalkParams q = wp;
    if (q.batch < 1) q.batch = 1;
    if (q.batch > kWalkMaxBatch) q.batch = kWalkMaxBatch;
    if (q.leaf_size < 1) q.leaf_size = 1;
    if (q.leaf_size > 32) q.leaf_size = 32;
    const int max_b = walk_max_blocks_per_sm(q.batch, q.with_potential);
    const int bps = blocks_per_sm > 0 && blocks_per_sm < max_b ? blocks_per_sm : max_b;
    int64_t grid = (int64_t)sm_count * bps;
    const int64_t need = ((int64_t)n_groups + kWalkWarps - 1) / kWalkWarps;
    if (grid > need) grid = need;
    // never more warps than the global stack regions provided
    const int64_t fit = (int64_t)(gstack_entries / ((size_t)kWalkWarps * kWalkGlobalStack));
    if (grid > fit) grid = fit;
    if (grid < 1) return;  // no stack regions: nothing can run (the engine always provides them)
    const unsigned g = (unsigned)grid;
    if (q.batch > 32)
        launch_h<2>(L, q, pos, tr, groups, n_groups, acc, queue, status, counts, gstack, g, st);
    else
        launch_h<1>(L, q, pos, tr, groups, n_groups, acc, queue, status, counts, gstack, g, st);
}

}  // namespace gcs
