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
//   * a term adds G m d / d2^{3/2}, with 1/sqrt from rsqrtf.
// With theta = 1 and L = 1 every target sees exactly the reference's set of
// terms; only the order of the FP32 sums differs.
//
// Execution: a persistent grid of warps pulls groups of <= 32 consecutive
// (Morton-adjacent) targets of one segment from a global work queue.  The
// warp walks the tree once for its group with one stack in shared memory;
// each stack entry carries the mask of lanes that still need that subtree,
// and each lane takes its own opening decision, so the group walk is the
// union of the 32 per-target walks with no change to any target's terms.
//   * up to `batch` entries are popped at once and their 32-byte nodes are
//     fetched by different lanes in parallel (two 16-byte loads each), then
//     evaluated one after another from shared memory (broadcast reads);
//   * particle sources (opened small nodes, leaf children) go to a
//     per-warp list; when it fills, the lanes fetch up to 64 source records
//     in parallel into shared memory and every lane sums them;
//   * the stack never overflows: batches are popped only while the stack
//     has room for a batch's children plus a depth-first descent of the
//     deepest possible path (96 internal levels: prefix lengths along a path
//     strictly increase and are < 96), so it is bounded by construction; the
//     bounds check that remains sets GCS_DEV_WALK_STACK_OVERFLOW instead of
//     writing out of bounds.
#include "gcs_internal.h"
#include "device_math.cuh"

namespace gcs {

namespace {

constexpr int kWalkWarps = 8;
constexpr int kWalkThreads = kWalkWarps * 32;
constexpr int kStackCap = 224;
constexpr int kMaxDepth = 96;
constexpr int kBatchLimit = kStackCap - kMaxDepth - 1;
constexpr int kMaxBatch = 32;
constexpr int kSrcCap = 64;
constexpr uint32_t kFull = 0xFFFFFFFFu;

struct WarpSmem {
    int2 stk[kStackCap];          // node, lane mask
    float4 nb0[kMaxBatch];        // com x,y,z, G*mass
    float4 nb1[kMaxBatch];        // width^2, child_left, child_right, range_end (bits)
    int2 nbm[kMaxBatch];          // node, lane mask
    float4 src[kSrcCap];          // x, y, z, G*mass
    int2 srcm[kSrcCap];           // particle, lane mask
};

struct Accum {
    float ax, ay, az, pot;
    uint32_t n_mono, n_part;  // interaction counts (count mode only)
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
        const float inv = rsqrtf(d2);
        const float inv3 = __fmul_rn(__fmul_rn(inv, inv), inv);
        const float f = use ? __fmul_rn(q.w, inv3) : 0.0f;
        A.ax = __fmaf_rn(dx, f, A.ax);
        A.ay = __fmaf_rn(dy, f, A.ay);
        A.az = __fmaf_rn(dz, f, A.az);
        if (kPot) A.pot = use ? __fmaf_rn(-q.w, inv, A.pot) : A.pot;
        if (kCount) A.n_part += use ? 1u : 0u;
    }
    __syncwarp();
}

template <bool kPot, bool kCount>
__global__ void __launch_bounds__(kWalkThreads)
walk_kernel(Layout L, WalkParams wp, const float4* __restrict__ pos,
            const BvhNodeTraverse* __restrict__ tr, const WalkGroup* __restrict__ groups,
            int n_groups, float4* __restrict__ acc, uint32_t* __restrict__ work_counter,
            uint32_t* __restrict__ status, unsigned long long* __restrict__ counts) {
    __shared__ WarpSmem smem[kWalkWarps];
    WarpSmem& W = smem[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const uint32_t lane_bit = 1u << lane;
    const float G = wp.G, eps2 = wp.eps2, theta2 = wp.theta2;
    const float leaf_thr = __fmul_rn(eps2, 1.01f);
    const int leaf_size = wp.leaf_size;
    const int batch = wp.batch;
    const int n_internal = L.n_internal;

    for (;;) {
        int g = 0;
        if (lane == 0) g = (int)atomicAdd(work_counter, 1u);
        g = __shfl_sync(kFull, g, 0);
        if (g >= n_groups) break;
        const WalkGroup grp = groups[g];
        const bool valid = lane < grp.count;
        const int t = grp.start + lane;
        const float4 p = valid ? __ldg(pos + t) : make_float4(0.f, 0.f, 0.f, 0.f);
        const uint32_t live = __ballot_sync(kFull, valid);
        const int s = grp.seg;
        const int off = (int)__ldg(L.seg_off + s);
        const int seg_n = (int)__ldg(L.seg_off + s + 1) - off;
        Accum A = {0.f, 0.f, 0.f, 0.f, 0u, 0u};
        int nsrc = 0;

        if (seg_n >= 2) {
            int top = 1;
            if (lane == 0) W.stk[0] = make_int2(off - s, (int)live);
            __syncwarp();
            // Each internal node has one parent, so a walk pops it at most
            // once: more pops than internal nodes means a malformed tree.
            int pop_budget = seg_n - 1;
            while (top > 0) {
                int b = top < batch ? top : batch;
                if (top + b > kBatchLimit) b = 1;
                pop_budget -= b;
                if (pop_budget < 0) {
                    if (lane == 0) atomicOr(status, GCS_DEV_TREE_MALFORMED);
                    break;
                }
                top -= b;
                if (lane < b) {
                    const int2 e = W.stk[top + lane];
                    const float4* np = reinterpret_cast<const float4*>(tr + e.x);
                    float4 a = __ldg(np);
                    float4 c = __ldg(np + 1);
                    a.w = __fmul_rn(G, a.w);
                    c.x = __fmul_rn(c.x, c.x);
                    W.nb0[lane] = a;
                    W.nb1[lane] = c;
                    W.nbm[lane] = e;
                }
                __syncwarp();
                for (int k = b - 1; k >= 0; --k) {
                    const float4 a = W.nb0[k];
                    const float4 c = W.nb1[k];
                    const int2 nm = W.nbm[k];
                    const bool active = ((uint32_t)nm.y & lane_bit) != 0u;
                    const float dx = __fsub_rn(a.x, p.x);
                    const float dy = __fsub_rn(a.y, p.y);
                    const float dz = __fsub_rn(a.z, p.z);
                    const float d2 = softened_d2(dx, dy, dz, eps2);
                    const bool take = accept_monopole(c.x, d2, theta2);
                    const bool mono = active && take;
                    if (__any_sync(kFull, mono)) {
                        const float inv = rsqrtf(d2);
                        const float inv3 = __fmul_rn(__fmul_rn(inv, inv), inv);
                        const float f = mono ? __fmul_rn(a.w, inv3) : 0.0f;
                        A.ax = __fmaf_rn(dx, f, A.ax);
                        A.ay = __fmaf_rn(dy, f, A.ay);
                        A.az = __fmaf_rn(dz, f, A.az);
                        if (kPot) A.pot = mono ? __fmaf_rn(-a.w, inv, A.pot) : A.pot;
                        if (kCount) A.n_mono += mono ? 1u : 0u;
                    }
                    const uint32_t om = __ballot_sync(kFull, active && !take);
                    if (om == 0u) continue;
                    const int own = nm.x + s;                 // particle index of this end
                    const int re = __float_as_int(c.w);
                    // clamp to the segment: a malformed range can never read outside it
                    const int lo = max(own < re ? own : re, off);
                    const int cnt = min((own < re ? re - own : own - re) + 1, off + seg_n - lo);
                    if (cnt <= leaf_size) {
                        if (nsrc + cnt > kSrcCap) {
                            flush_sources<kPot, kCount>(W, nsrc, lane, lane_bit, pos, G, p, eps2, leaf_thr, A);
                            nsrc = 0;
                        }
                        if (lane < cnt) W.srcm[nsrc + lane] = make_int2(lo + lane, (int)om);
                        nsrc += max(cnt, 0);
                    } else {
#pragma unroll
                        for (int side = 0; side < 2; ++side) {
                            const int ch = __float_as_int(side == 0 ? c.y : c.z);
                            if (ch < 0 || ch >= n_internal + L.n) {
                                if (lane == 0) atomicOr(status, GCS_DEV_BUILD_RANGE);
                            } else if (ch >= n_internal) {
                                if (nsrc + 1 > kSrcCap) {
                                    flush_sources<kPot, kCount>(W, nsrc, lane, lane_bit, pos, G, p, eps2,
                                                        leaf_thr, A);
                                    nsrc = 0;
                                }
                                if (lane == 0) W.srcm[nsrc] = make_int2(ch - n_internal, (int)om);
                                nsrc += 1;
                            } else if (top < kStackCap) {
                                if (lane == 0) W.stk[top] = make_int2(ch, (int)om);
                                ++top;
                            } else if (lane == 0) {
                                atomicOr(status, GCS_DEV_WALK_STACK_OVERFLOW);
                            }
                        }
                    }
                }
                __syncwarp();
                if (nsrc >= 32) {
                    flush_sources<kPot, kCount>(W, nsrc, lane, lane_bit, pos, G, p, eps2, leaf_thr, A);
                    nsrc = 0;
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
            }
        }
        __syncwarp();
    }
}

}  // namespace

int walk_max_blocks_per_sm(int batch, int with_potential) {
    (void)batch;
    int nb = 0;
    if (with_potential)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, walk_kernel<true, false>, kWalkThreads, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, walk_kernel<false, false>, kWalkThreads, 0);
    return nb > 0 ? nb : 1;
}

void launch_walk(const Layout& L, const WalkParams& wp, const float4* pos,
                 const BvhNodeTraverse* tr, const WalkGroup* groups, int n_groups, float4* acc,
                 uint32_t* work_counter, uint32_t* status, int blocks_per_sm, int sm_count,
                 unsigned long long* counts, cudaStream_t st) {
    if (n_groups <= 0) return;
    WalkParams q = wp;
    if (q.batch < 1) q.batch = 1;
    if (q.batch > kMaxBatch) q.batch = kMaxBatch;
    if (q.leaf_size < 1) q.leaf_size = 1;
    if (q.leaf_size > 32) q.leaf_size = 32;
    const int max_b = walk_max_blocks_per_sm(q.batch, q.with_potential);
    const int bps = blocks_per_sm > 0 && blocks_per_sm < max_b ? blocks_per_sm : max_b;
    int64_t grid = (int64_t)sm_count * bps;
    const int64_t need = ((int64_t)n_groups + kWalkWarps - 1) / kWalkWarps;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    const unsigned g = (unsigned)grid;
    if (counts) {
        if (q.with_potential)
            walk_kernel<true, true><<<g, kWalkThreads, 0, st>>>(L, q, pos, tr, groups, n_groups, acc,
                                                                work_counter, status, counts);
        else
            walk_kernel<false, true><<<g, kWalkThreads, 0, st>>>(L, q, pos, tr, groups, n_groups, acc,
                                                                 work_counter, status, counts);
    } else if (q.with_potential) {
        walk_kernel<true, false><<<g, kWalkThreads, 0, st>>>(L, q, pos, tr, groups, n_groups, acc,
                                                             work_counter, status, nullptr);
    } else {
        walk_kernel<false, false><<<g, kWalkThreads, 0, st>>>(L, q, pos, tr, groups, n_groups, acc,
                                                              work_counter, status, nullptr);
    }
}

}  // namespace gcs
