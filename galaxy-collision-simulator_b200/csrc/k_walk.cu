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
//   1. up to `batch` entries are popped; lane k fetches node k (two 16-byte
//      loads) and digests it (G*mass, width^2, and either the particle range
//      to sum for a node of <= L particles or its two children coded as node
//      or particle) into shared memory and its own registers;
//   2. a branch-free loop over the batch: every lane tests its own opening
//      criterion, adds the monopole term where it accepts (predicated), and
//      the warp ballots the lanes that open; lane k keeps node k's ballot;
//   3. in parallel, lane k pushes node k's internal children and appends its
//      particle sources (leaf children, or the whole range of a small node)
//      at offsets from one warp prefix scan;
//   4. particle sources accumulate in a per-warp list; when it fills, the
//      lanes fetch up to 64 source records in parallel into shared memory and
//      every lane sums them.
// The stack's top lives in shared memory; when it passes a threshold its
// bottom half is spilled to a per-warp region of global memory (L2) and read
// back when the top runs low, so batches are never throttled and the
// logical stack order is exactly that of an unbounded stack.  A global region
// that would overflow sets GCS_DEV_WALK_STACK_OVERFLOW (entries are dropped,
// nothing is written out of bounds); a walk that pops more nodes than the
// tree holds stops with GCS_DEV_TREE_MALFORMED.  The work queue resets
// itself: the last warp to find it empty zeroes it.
#include "gcs_internal.h"
#include "device_math.cuh"

namespace gcs {

namespace {

constexpr int kWalkWarps = 8;
constexpr int kWalkThreads = kWalkWarps * 32;
// 5 resident blocks (40 warps) per SM: 48 registers a thread.
constexpr int kWalkMinBlocks = 5;
constexpr int kMaxBatch = 32;
constexpr int kStackCap = 256;                       // shared-memory stack entries per warp
constexpr int kSpillAbove = kStackCap - 2 * kMaxBatch;  // a round pushes at most 2*batch
constexpr int kSpillCount = 128;                     // entries moved per spill / refill
constexpr int kSrcCap = 64;
constexpr uint32_t kFull = 0xFFFFFFFFu;
// Digested node codes (NodeRec .y/.z):
//   .z >= kBucketTag    the node itself is summed directly: particles
//                       [.y, .y + .z - kBucketTag)
//   .z == kSkipTag      malformed children, nothing pushed
//   otherwise .y/.z     children: >= 0 internal node, < 0 particle ~code
constexpr int kBucketTag = 1 << 30;
constexpr int kSkipTag = 0x7FFFFFFF;

// Classes of a batch node against the group's bounding box.
constexpr int kClassNone = 0;   // lane holds no node
constexpr int kClassTake = 1;   // every lane of the group accepts it
constexpr int kClassOpen = 2;   // every lane of the group opens it
constexpr int kClassMixed = 3;  // lanes decide one by one
constexpr float kBoxLo = 1.0f - 1.0f / 65536.0f;
constexpr float kBoxHi = 1.0f + 1.0f / 65536.0f;

struct WarpSmem {
    int2 stk[kStackCap];          // node, lane mask
    float4 nc[kMaxBatch];         // com x, y, z, G*mass (compacted: take, then mixed)
    uint2 nw[kMaxBatch];          // bits of width^2, lane mask
    uint32_t nopen[kMaxBatch];    // opening lanes of each mixed node
    float4 src[kSrcCap];          // x, y, z, G*mass
    int2 srcm[kSrcCap];           // particle, lane mask
};

struct Accum {
    float ax, ay, az, pot;
    uint32_t n_mono, n_part;  // interaction counts (count mode only)
    uint32_t w_node, w_src;   // warp-wide node / source evaluations (count mode only)
    uint32_t rounds, spills;  // pop rounds, stack spills to global memory
    uint32_t all_open, all_take;  // node evaluations opened / accepted by every active lane
};

// Sum the listed particle sources into every lane whose bit is in the
// source's mask (leaf rule: skip d2 <= 1.01 eps^2).
template <bool kPot, bool kCount>
__device__ __forceinline__ void flush_sources(WarpSmem& W, int nsrc, int lane, uint32_t lane_bit,
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

template <bool kPot, bool kCount>
__global__ void __launch_bounds__(kWalkThreads, kWalkMinBlocks)
walk_kernel(Layout L, WalkParams wp, const float4* __restrict__ pos,
            const BvhNodeTraverse* __restrict__ tr, const WalkGroup* __restrict__ groups,
            int n_groups, float4* __restrict__ acc, uint32_t* __restrict__ queue,
            uint32_t* __restrict__ status, unsigned long long* __restrict__ counts,
            int2* __restrict__ gstack, int gstack_cap) {
    __shared__ WarpSmem smem[kWalkWarps];
    const int warp = threadIdx.x >> 5;
    WarpSmem& W = smem[warp];
    int2* const gstk = gstack + ((size_t)blockIdx.x * kWalkWarps + warp) * (size_t)gstack_cap;
    const int lane = threadIdx.x & 31;
    const uint32_t lane_bit = 1u << lane;
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
                    const int2 keep = lane < top ? W.stk[lane] : make_int2(0, 0);  // top < batch <= 32
                    __syncwarp();
                    if (lane < top) W.stk[k + lane] = keep;
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
                // 1. fetch, digest and classify node `lane` of the batch
                int code_a = 0, code_b = kSkipTag;
                int cls = kClassNone;
                float w2 = 0.0f;
                float4 com = make_float4(0.f, 0.f, 0.f, 0.f);
                uint32_t my_mask = 0u;
                if (lane < b) {
                    const int2 e = W.stk[top + lane];
                    const float4* np = reinterpret_cast<const float4*>(tr + e.x);
                    float4 a = __ldg(np);
                    const float4 c = __ldg(np + 1);
                    a.w = __fmul_rn(G, a.w);
                    const int own = e.x + s;  // particle index at this end of the range
                    const int re = __float_as_int(c.w);
                    const int lo = max(min(own, re), off);
                    const int cnt = min(max(own, re), seg_end - 1) - lo + 1;
                    if (cnt <= leaf_size) {
                        code_a = lo;
                        code_b = kBucketTag + max(cnt, 0);
                    } else {
                        const int cl = __float_as_int(c.y), cr = __float_as_int(c.z);
                        if (cl >= 0 && cl < n_internal + n_total && cr >= 0 && cr < n_internal + n_total) {
                            code_a = cl >= n_internal ? ~(cl - n_internal) : cl;
                            code_b = cr >= n_internal ? ~(cr - n_internal) : cr;
                        } else {
                            atomicOr(status, GCS_DEV_BUILD_RANGE);
                        }
                    }
                    w2 = __fmul_rn(c.x, c.x);
                    com = a;
                    my_mask = (uint32_t)e.y;
                    // Classify against the group's box.  With a 2^-16 relative
                    // margin (far above the few-ulp rounding of any lane's own
                    // d2 or of these sums) "take" guarantees every lane in the
                    // box accepts, "open" that every lane opens.
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
                    if (w2 < theta2 * (s2min + eps2) * kBoxLo) cls = kClassTake;
                    else if (w2 >= theta2 * (s2max + eps2) * kBoxHi) cls = kClassOpen;
                    else cls = kClassMixed;
                }
                // compact: accepted-by-all nodes first, then mixed ones
                const uint32_t bt = __ballot_sync(kFull, cls == kClassTake);
                const uint32_t bm = __ballot_sync(kFull, cls == kClassMixed);
                const int n_take = __popc(bt), n_mixed = __popc(bm);
                const uint32_t lt = lane_bit - 1u;
                const int slot = cls == kClassTake ? __popc(bt & lt)
                                                   : (cls == kClassMixed ? n_take + __popc(bm & lt) : -1);
                if (slot >= 0) {
                    W.nc[slot] = com;
                    W.nw[slot] = make_uint2(__float_as_uint(w2), my_mask);
                }
                __syncwarp();
                if (kCount) {
                    A.w_node += (uint32_t)b;
                    A.rounds += 1u;
                    A.all_open += (uint32_t)(b - n_take - n_mixed);
                    A.all_take += (uint32_t)n_take;
                }
                // 2a. nodes every lane accepts: monopole terms only
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
                // 2b. mixed nodes: each lane's own test; lane 0 records the
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
                uint32_t my_open = 0u;
                if (cls == kClassOpen) my_open = my_mask;
                else if (cls == kClassMixed) my_open = W.nopen[slot];
                // 3. parallel push / append for the opened nodes
                int n_push = 0, n_src = 0;
                if (my_open != 0u && code_b != kSkipTag) {
                    if (code_b >= kBucketTag) {
                        n_src = code_b - kBucketTag;
                    } else {
                        n_push = (code_a >= 0) + (code_b >= 0);
                        n_src = (code_a < 0) + (code_b < 0);
                    }
                }
                const uint32_t both = ((uint32_t)n_push << 16) | (uint32_t)n_src;
                const uint32_t excl = warp_exclusive_scan(both, lane);
                const uint32_t total = __shfl_sync(kFull, excl + both, 31);
                const int push_at = top + (int)(excl >> 16);
                if (n_push > 0) {
                    int at = push_at;
                    if (code_a >= 0) W.stk[at++] = make_int2(code_a, (int)my_open);
                    if (code_b >= 0) W.stk[at] = make_int2(code_b, (int)my_open);
                }
                top += (int)(total >> 16);
                // sources: [src_at, src_at + n_src) of this round's `add` new ones,
                // appended in windows that fit the list, flushing between windows
                const int src_at = (int)(excl & 0xFFFFu);
                const int add = (int)(total & 0xFFFFu);
                for (int base = 0; base < add;) {
                    if (nsrc == kSrcCap) {
                        flush_sources<kPot, kCount>(W, nsrc, lane, lane_bit, pos, G, p, eps2, leaf_thr, A);
                        nsrc = 0;
                    }
                    const int window = min(kSrcCap - nsrc, add - base);
                    const int j0 = max(src_at, base), j1 = min(src_at + n_src, base + window);
                    for (int j = j0; j < j1; ++j) {
                        const int r = j - src_at;  // r-th source of this lane's node
                        int particle;
                        if (code_b >= kBucketTag) particle = code_a + r;
                        else particle = (r == 0 && code_a < 0) ? ~code_a : ~code_b;
                        W.srcm[nsrc + (j - base)] = make_int2(particle, (int)my_open);
                    }
                    nsrc += window;
                    base += window;
                }
                __syncwarp();
                if (nsrc >= 32) {
                    flush_sources<kPot, kCount>(W, nsrc, lane, lane_bit, pos, G, p, eps2, leaf_thr, A);
                    nsrc = 0;
                }
                // spill the shared stack's bottom half before it can overflow
                if (top > kSpillAbove) {
                    if (gtop + kSpillCount <= gstack_cap) {
                        for (int j = lane; j < kSpillCount; j += 32) gstk[gtop + j] = W.stk[j];
                        gtop += kSpillCount;
                    } else if (lane == 0) {
                        atomicOr(status, GCS_DEV_WALK_STACK_OVERFLOW);
                    }
                    const int rest = top - kSpillCount;  // <= kStackCap - kSpillCount = 128
                    int2 mv[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const int j = lane + 32 * i;
                        mv[i] = j < rest ? W.stk[kSpillCount + j] : make_int2(0, 0);
                    }
                    __syncwarp();
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const int j = lane + 32 * i;
                        if (j < rest) W.stk[j] = mv[i];
                    }
                    top = rest;
                    if (kCount) A.spills += 1u;
                    __syncwarp();
                }
            }
        }
        if (nsrc > 0) flush_sources<kPot, kCount>(W, nsrc, lane, lane_bit, pos, G, p, eps2, leaf_thr, A);
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

}  // namespace

int walk_max_blocks_per_sm(int batch, int with_potential) {
    (void)batch;
    static int cached[2] = {0, 0};  // same for every device of this build (sm_100a only)
    int& nb = cached[with_potential ? 1 : 0];
    if (nb == 0) {
        if (with_potential)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, walk_kernel<true, false>, kWalkThreads, 0);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, walk_kernel<false, false>, kWalkThreads, 0);
        if (nb <= 0) nb = 1;
    }
    return nb;
}

int64_t walk_grid_blocks(int n_groups, int blocks_per_sm, int sm_count, int with_potential) {
    const int max_b = walk_max_blocks_per_sm(0, with_potential);
    const int bps = blocks_per_sm > 0 && blocks_per_sm < max_b ? blocks_per_sm : max_b;
    int64_t grid = (int64_t)sm_count * bps;
    const int64_t need = ((int64_t)n_groups + kWalkWarps - 1) / kWalkWarps;
    if (grid > need) grid = need;
    return grid < 1 ? 1 : grid;
}

size_t walk_stack_entries(int64_t grid_blocks) {
    return (size_t)grid_blocks * kWalkWarps * (size_t)kWalkGlobalStack;
}

void launch_walk(const Layout& L, const WalkParams& wp, const float4* pos,
                 const BvhNodeTraverse* tr, const WalkGroup* groups, int n_groups, float4* acc,
                 uint32_t* queue, uint32_t* status, int blocks_per_sm, int sm_count,
                 unsigned long long* counts, int2* gstack, size_t gstack_entries, cudaStream_t st) {
    if (n_groups <= 0) return;
    WalkParams q = wp;
    if (q.batch < 1) q.batch = 1;
    if (q.batch > kMaxBatch) q.batch = kMaxBatch;
    if (q.leaf_size < 1) q.leaf_size = 1;
    if (q.leaf_size > 32) q.leaf_size = 32;
    int64_t grid = walk_grid_blocks(n_groups, blocks_per_sm, sm_count, q.with_potential);
    // never more warps than the global stack regions provided
    const int64_t fit = (int64_t)(gstack_entries / ((size_t)kWalkWarps * kWalkGlobalStack));
    if (grid > fit) grid = fit;
    if (grid < 1) return;  // no stack regions: nothing can run (the engine always provides them)
    const unsigned g = (unsigned)grid;
    const int cap = kWalkGlobalStack;
    if (counts) {
        if (q.with_potential)
            walk_kernel<true, true><<<g, kWalkThreads, 0, st>>>(L, q, pos, tr, groups, n_groups, acc,
                                                                queue, status, counts, gstack, cap);
        else
            walk_kernel<false, true><<<g, kWalkThreads, 0, st>>>(L, q, pos, tr, groups, n_groups, acc,
                                                                 queue, status, counts, gstack, cap);
    } else if (q.with_potential) {
        walk_kernel<true, false><<<g, kWalkThreads, 0, st>>>(L, q, pos, tr, groups, n_groups, acc,
                                                             queue, status, nullptr, gstack, cap);
    } else {
        walk_kernel<false, false><<<g, kWalkThreads, 0, st>>>(L, q, pos, tr, groups, n_groups, acc,
                                                              queue, status, nullptr, gstack, cap);
    }
}

}  // namespace gcs
