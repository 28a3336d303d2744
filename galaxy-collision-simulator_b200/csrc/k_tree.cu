// k_tree.cu - Karras (2012) binary radix tree over each segment's sorted
// Morton keys, and the bottom-up aggregation of bounds, mass and centre of
// mass.
//
// Build: one thread per internal node, as in karras_bvh.cuh:73-131.  The
// steps of the published algorithm (direction from the neighbours' common
// prefixes, exponential then binary search for the far end, binary search
// for the split) decide the topology, so they are the same steps; the
// common-prefix function is the reference's, including its duplicate-key
// rule (equal keys compare their positions, karras_bvh.cuh:23-31).  Indices
// are local to the segment, so a segment's tree is the tree the reference
// builds for that segment alone.  Each node also records the far end of its
// particle range, which gives the walk the node's particle count.
//
// Aggregation: a climb starts at every particle's leaf (a lane runs one climb
// after another over its block's particles); at each node the first arrival
// stops and the second computes the node from both children
// (karras_bvh.cuh:175-225).  Unlike the reference, the arrival counter is a
// release/acquire handshake (__threadfence on both sides and L2-coherent
// loads of the children), so the second arrival always sees the first one's
// writes.  Centres of mass are either the reference's FP32 formula or FP64
// mass-weighted sums carried up the tree (exact for leaf terms, no
// cancellation at the top of the tree), rounded once to FP32.
#include "gcs_internal.h"
#include "device_math.cuh"

namespace gcs {

namespace {

// Arrival counter increment with acquire-release semantics at GPU scope.
__device__ __forceinline__ int arrive_acq_rel(int32_t* flag) {
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(old) : "l"(flag) : "memory");
    return old;
}
__device__ __forceinline__ int arrive_relaxed(int32_t* flag) {
    int old;
    asm volatile("atom.relaxed.gpu.global.add.s32 %0, [%1], 1;" : "=r"(old) : "l"(flag) : "memory");
    return old;
}
// Acquire side of a relaxed arrival (the fence makes the sibling's writes,
// released by its own acq_rel arrival, visible to the loads that follow).
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Common prefix length of sorted keys i and j of one segment (local indices);
// -1 when j falls outside the segment.
__device__ __forceinline__ int lcp(int i, int j, int n, const uint64_t* __restrict__ k,
                                   uint64_t ki) {
    if (j < 0 || j >= n) return -1;
    const uint64_t kj = __ldg(k + j);
    if (ki == kj) return 64 + __clz(i ^ j);
    return __clzll(ki ^ kj);
}

__global__ void build_kernel(Layout L, const uint64_t* __restrict__ keys,
                             BvhNodeTraverse* __restrict__ tr, BvhNodeBuild* __restrict__ bd,
                             int32_t* __restrict__ leaf_parent, uint32_t* __restrict__ status) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < L.n; g += gridDim.x * blockDim.x) {
        const int s = L.nseg > 1 ? __ldg(L.seg_id + g) : 0;
        const int off = (int)__ldg(L.seg_off + s);
        const int n = (int)__ldg(L.seg_off + s + 1) - off;
        const int i = g - off;                  // local index
        const int node_base = off - s;          // first internal node of the segment
        const int leaf_base = L.n_internal + off;
        const uint64_t* k = keys + off;
        if (n == 1) {                           // single particle: its leaf is the root
            leaf_parent[g] = -1;
            continue;
        }
        if (i >= n - 1) continue;
        const uint64_t ki = __ldg(k + i);
        const int d = (lcp(i, i + 1, n, k, ki) - lcp(i, i - 1, n, k, ki)) > 0 ? 1 : -1;
        const int dmin = lcp(i, i - d, n, k, ki);
        int lmax = 2;
        while (lcp(i, i + lmax * d, n, k, ki) > dmin) lmax *= 2;
        int l = 0;
        for (int t = lmax / 2; t >= 1; t /= 2)
            if (lcp(i, i + (l + t) * d, n, k, ki) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = lcp(i, j, n, k, ki);
        int s_ = 0, step = l;
        do {
            step = (step + 1) >> 1;
            if (lcp(i, i + (s_ + step) * d, n, k, ki) > dnode) s_ += step;
        } while (step > 1);
        const int split = i + s_ * d + (d > 0 ? 0 : -1);
        const int lo = min(i, j), hi = max(i, j);
        if (split < lo || split + 1 > hi) {  // cannot happen for sorted keys; never write out of range
            atomicOr(status, GCS_DEV_BUILD_RANGE);
            continue;
        }
        const int node = node_base + i;
        const int cl = (lo == split) ? leaf_base + split : node_base + split;
        const int cr = (hi == split + 1) ? leaf_base + split + 1 : node_base + split + 1;
        BvhNodeTraverse* nt = tr + node;
        nt->child_left = cl;
        nt->child_right = cr;
        nt->range_end = off + j;
        if (lo == split) leaf_parent[off + split] = node;
        else bd[cl].parent = node;
        if (hi == split + 1) leaf_parent[off + split + 1] = node;
        else bd[cr].parent = node;
        bd[node].flag = 0;
        if (i == 0) bd[node].parent = -1;       // segment root
    }
}

struct ChildData {
    float3 lo, hi, com;
    float m;
    double3 mx;   // FP64 mass-weighted position sums
    double md;    // FP64 mass sum
};

// Loads child c; its FP64 sums only when `fp64` (the caller's test that c is
// an internal node of at least kComFp64Min particles under a node that sums
// in FP64; a particle is never one).
__device__ __forceinline__ ChildData load_child(int c, int n_internal, const float4* __restrict__ pos,
                                                const BvhNodeTraverse* tr, const BvhNodeBuild* bd,
                                                const double4* com64, bool fp64) {
    ChildData r;
    if (c >= n_internal) {
        const float4 p = __ldg(pos + (c - n_internal));
        r.lo = r.hi = r.com = make_float3(p.x, p.y, p.z);
        r.m = p.w;
    } else {
        // Written by another thread of this launch: read through L2.
        const float4 a = __ldcg(reinterpret_cast<const float4*>(tr + c));
        const float4 b0 = __ldcg(reinterpret_cast<const float4*>(bd + c));
        const float2 b1 = __ldcg(reinterpret_cast<const float2*>(bd + c) + 2);
        r.com = make_float3(a.x, a.y, a.z);
        r.m = a.w;
        r.lo = make_float3(b0.x, b0.y, b0.z);
        r.hi = make_float3(b0.w, b1.x, b1.y);
        if (fp64) {
            const double2 q0 = __ldcg(reinterpret_cast<const double2*>(com64 + c));
            const double2 q1 = __ldcg(reinterpret_cast<const double2*>(com64 + c) + 1);
            r.mx = make_double3(q0.x, q0.y, q1.x);
            r.md = q1.y;
        }
    }
    return r;
}

constexpr uint32_t kFull = 0xFFFFFFFFu;
constexpr int kAggThreads = 128;     // threads of an aggregation block
constexpr int kAggRange = 512;       // particles a block owns (its lanes take them as they finish)
constexpr int kAggBlocksPerSm = 8;
// FP64 centre-of-mass sums (com_fp64) are kept for the top of the tree:
// nodes of at least this many particles, where the mass-weighted positions
// of many particles are summed.  A child below the size (or a particle)
// enters its parent's sums as the exact double product of its FP32 mass and
// centre of mass (position).  Block-local nodes hold at most kAggRange
// particles, so they are never FP64 nodes.
constexpr int kComFp64Min = 1024;
static_assert(kComFp64Min > kAggRange, "block-local nodes are never FP64 nodes");

// A node finished inside the block, kept in shared memory for its parent.
struct LocalNode {
    float3 lo, hi, com;
    float m;
};

__device__ __forceinline__ ChildData from_local(const LocalNode& q) {
    ChildData r;
    r.lo = q.lo;
    r.hi = q.hi;
    r.com = q.com;
    r.m = q.m;
    return r;
}

// A child's terms in its parent's FP64 sums: its own sums if it is an FP64
// node, else the double product of its FP32 mass and centre of mass.
__device__ __forceinline__ void fp64_terms(const ChildData& c, bool big, double3& mx, double& md) {
    if (big) {
        mx = c.mx;
        md = c.md;
    } else {
        md = (double)c.m;
        mx = make_double3(md * (double)c.com.x, md * (double)c.com.y, md * (double)c.com.z);
    }
}

// Walk record of internal node `node` (links already range-checked): the
// particle range [min(own, re), max(own, re)] clipped to the segment
// [seg_lo, seg_hi]; <= leaf_size particles make a bucket, else the children
// are coded as internal node or ~particle.
__device__ __forceinline__ void write_walk_node(const WalkNodeParams& wnp, int node, float3 com, float m,
                                                float width, int cl, int cr, int own, int re, int seg_lo,
                                                int seg_hi, int n_internal) {
    const int lo = max(min(own, re), seg_lo);
    const int cnt = min(max(own, re), seg_hi) - lo + 1;
    int ca, cb;
    if (cnt <= wnp.leaf_size) {
        ca = lo;
        cb = kWalkBucketTag + max(cnt, 0);
    } else {
        ca = cl >= n_internal ? ~(cl - n_internal) : cl;
        cb = cr >= n_internal ? ~(cr - n_internal) : cr;
    }
    float4* w = reinterpret_cast<float4*>(wnp.wn + node);
    w[0] = make_float4(com.x, com.y, com.z, __fmul_rn(wnp.G, m));
    reinterpret_cast<int4*>(w)[1] = make_int4(__float_as_int(__fmul_rn(width, width)), ca, cb, 0);
}

// Walk records from the traverse records: one thread per particle g; the
// internal node g - s exists for every particle but the last of segment s.
__global__ void walk_nodes_kernel(Layout L, const BvhNodeTraverse* __restrict__ tr, WalkNodeParams wnp,
                                  uint32_t* __restrict__ status) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= L.n) return;
    const int s = L.nseg > 1 ? __ldg(L.seg_id + g) : 0;
    const int seg_lo = (int)__ldg(L.seg_off + s), seg_hi = (int)__ldg(L.seg_off + s + 1) - 1;
    if (g >= seg_hi) return;
    const int node = g - s;
    const float4* np = reinterpret_cast<const float4*>(tr + node);
    const float4 a = __ldg(np);
    const float4 c = __ldg(np + 1);
    const int cl = __float_as_int(c.y), cr = __float_as_int(c.z);
    const int lim = L.n_internal + L.n;
    if (cl >= 0 && cl < lim && cr >= 0 && cr < lim) {
        write_walk_node(wnp, node, make_float3(a.x, a.y, a.z), a.w, c.x, cl, cr, node + s, __float_as_int(c.w),
                        seg_lo, seg_hi, L.n_internal);
    } else {
        atomicOr(status, GCS_DEV_BUILD_RANGE);
        float4* w = reinterpret_cast<float4*>(wnp.wn + node);
        w[0] = make_float4(a.x, a.y, a.z, __fmul_rn(wnp.G, a.w));
        reinterpret_cast<int4*>(w)[1] = make_int4(__float_as_int(__fmul_rn(c.x, c.x)), 0, kWalkSkipTag, 0);
    }
}

// Block b owns particles [kAggRange b, kAggRange (b + 1)).  A node whose
// particle range lies inside its block's range has both children finished by
// threads of that block: its arrival counter and the finished children live
// in shared memory and the handshake is block-scoped.  Every other node uses
// the GPU-scope counter in its build record.  The side a node uses depends
// only on the node, so both arrivals always meet.
//
// Each lane climbs from one particle at a time: it arrives at the parent of
// what it has just finished; the first arrival stops, the second computes the
// parent and climbs on.  A lane whose climb has stopped takes the block's
// next particle at once (the warp claims particles for all its idle lanes
// with one shared-memory atomic), so a warp keeps its lanes busy instead of
// running as long as its longest-climbing lane.  Which lane computes a node
// does not change its value.
__global__ void __launch_bounds__(kAggThreads, kAggBlocksPerSm)
aggregate_kernel(Layout L, const float4* __restrict__ pos, BvhNodeTraverse* __restrict__ tr,
                 BvhNodeBuild* __restrict__ bd, double4* __restrict__ com64,
                 const int32_t* __restrict__ leaf_parent, int com_fp64, WalkNodeParams wnp,
                 uint32_t* __restrict__ status) {
    __shared__ int sflag[kAggRange];
    __shared__ LocalNode snode[kAggRange];
    __shared__ int s_next;  // the block's next unclaimed particle
    const bool fp64 = com_fp64 != 0;
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const int ni = L.n_internal;
    const int b0 = blockIdx.x * kAggRange;
    const int b_end = min(b0 + kAggRange, L.n);
    for (int i = threadIdx.x; i < kAggRange; i += kAggThreads) sflag[i] = 0;
    if (threadIdx.x == 0) s_next = b0;
    __syncthreads();
    bool have = false;  // this lane is climbing
    int s = 0, seg_lo = 0, seg_hi = 0, from = 0, node = -1, cl = -1, cr = -1, up = -1, re = 0, levels = 0;
    ChildData mine;
    for (;;) {
        // idle lanes take the block's next particles
        const uint32_t idle = __ballot_sync(kFull, !have);
        if (idle) {
            const int leader = __ffs(idle) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(&s_next, __popc(idle));
            base = __shfl_sync(kFull, base, leader);
            if (!have) {
                const int g = base + __popc(idle & lt);
                if (g < b_end) {
                    s = L.nseg > 1 ? __ldg(L.seg_id + g) : 0;
                    seg_lo = (int)__ldg(L.seg_off + s);
                    seg_hi = (int)__ldg(L.seg_off + s + 1) - 1;
                    from = ni + g;
                    mine = load_child(from, ni, pos, tr, bd, com64, false);
                    node = __ldg(leaf_parent + g);
                    levels = 0;
                    if (node >= 0 && node < ni) {
                        cl = __ldg(&tr[node].child_left);
                        cr = __ldg(&tr[node].child_right);
                        up = __ldg(&bd[node].parent);
                        re = __ldg(&tr[node].range_end);
                    }
                    have = node >= 0;  // a one-particle segment has no parent
                }
            }
        }
        if (!__any_sync(kFull, have)) break;
        if (!have) continue;
        // one step of this lane's climb: arrive at `node`, the parent of `from`
        // (a valid tree has at most 96 internal levels: strictly increasing
        // prefix lengths below 96; more means malformed parent links)
        if (++levels > 96 || node >= ni) {
            atomicOr(status, GCS_DEV_TREE_MALFORMED);
            have = false;
            continue;
        }
        const int own = node + s;  // particle index at this end of the node's range
        const bool local = min(own, re) >= b0 && max(own, re) < b0 + kAggRange;
        int old;
        if (local) {
            // block scope: this lane's writes (shared and global) before the
            // arrival, the sibling's after it
            __threadfence_block();
            old = atomicAdd(&sflag[own - b0], 1);
            if (old != 0) __threadfence_block();
        } else if (levels == 1) {
            // at the leaf level this lane has written nothing for `from`, so
            // its arrival needs no release; it acquires only if it arrives second
            old = arrive_relaxed(&bd[node].flag);
            if (old != 0) fence_acq_rel();
        } else {
            // release: the child this lane just finished is visible to whoever
            // acquires the counter next; acquire: the second arrival sees the
            // sibling's writes
            old = arrive_acq_rel(&bd[node].flag);
        }
        if (old == 0) {  // first arrival: the sibling's climb finishes the node
            have = false;
            continue;
        }
        if (cl < 0 || cr < 0 || cl >= ni + L.n || cr >= ni + L.n || (cl != from && cr != from)) {
            atomicOr(status, GCS_DEV_TREE_MALFORMED);
            have = false;
            continue;
        }
        int ncl = -1, ncr = -1, nup = -1, nre = 0;
        if (up >= 0 && up < ni) {
            ncl = __ldg(&tr[up].child_left);
            ncr = __ldg(&tr[up].child_right);
            nup = __ldg(&bd[up].parent);
            nre = __ldg(&tr[up].range_end);
        }
        const bool left = cl == from;
        const int sib = left ? cr : cl;
        // particles of the node and of its two children (the split is the
        // left child's end of the range)
        const int lo_p = min(own, re), hi_p = max(own, re);
        const int split = cl >= ni ? cl - ni : cl + s;
        const bool big = fp64 && hi_p - lo_p + 1 >= kComFp64Min;
        const bool big_l = big && split - lo_p + 1 >= kComFp64Min;
        const bool big_r = big && hi_p - split >= kComFp64Min;
        // a local node's internal children are local too: read them from
        // shared memory (their own range end is inside the block)
        ChildData other;
        if (local && sib < ni) {
            const int so = sib + s - b0;
            if (so < 0 || so >= kAggRange) {
                atomicOr(status, GCS_DEV_TREE_MALFORMED);
                have = false;
                continue;
            }
            other = from_local(snode[so]);
        } else {
            other = load_child(sib, ni, pos, tr, bd, com64, left ? big_r : big_l);
        }
        const ChildData& A = left ? mine : other;   // left child
        const ChildData& B = left ? other : mine;   // right child
        const float3 lo = make_float3(fminf(A.lo.x, B.lo.x), fminf(A.lo.y, B.lo.y), fminf(A.lo.z, B.lo.z));
        const float3 hi = make_float3(fmaxf(A.hi.x, B.hi.x), fmaxf(A.hi.y, B.hi.y), fmaxf(A.hi.z, B.hi.z));
        const float width = fmaxf(__fsub_rn(hi.x, lo.x), fmaxf(__fsub_rn(hi.y, lo.y), __fsub_rn(hi.z, lo.z)));
        const float m = __fadd_rn(A.m, B.m);
        float3 com;
        ChildData next;
        next.md = 0.0;
        next.mx = make_double3(0.0, 0.0, 0.0);
        if (m > 0.0f) {
            if (big) {
                double3 amx, bmx;
                double amd, bmd;
                fp64_terms(A, big_l, amx, amd);
                fp64_terms(B, big_r, bmx, bmd);
                next.md = amd + bmd;
                next.mx = make_double3(amx.x + bmx.x, amx.y + bmx.y, amx.z + bmx.z);
                com = make_float3((float)(next.mx.x / next.md), (float)(next.mx.y / next.md),
                                  (float)(next.mx.z / next.md));
            } else {
                com = make_float3(com_fp32(A.com.x, A.m, B.com.x, B.m, m), com_fp32(A.com.y, A.m, B.com.y, B.m, m),
                                  com_fp32(A.com.z, A.m, B.com.z, B.m, m));
            }
        } else {
            com = make_float3(__fmul_rn(__fadd_rn(lo.x, hi.x), 0.5f), __fmul_rn(__fadd_rn(lo.y, hi.y), 0.5f),
                              __fmul_rn(__fadd_rn(lo.z, hi.z), 0.5f));
        }
        if (big) com64[node] = make_double4(next.mx.x, next.mx.y, next.mx.z, next.md);
        float4* t4 = reinterpret_cast<float4*>(tr + node);
        t4[0] = make_float4(com.x, com.y, com.z, m);
        tr[node].width = width;
        if (wnp.wn) write_walk_node(wnp, node, com, m, width, cl, cr, own, re, seg_lo, seg_hi, ni);
        float4* b4 = reinterpret_cast<float4*>(bd + node);
        b4[0] = make_float4(lo.x, lo.y, lo.z, hi.x);
        reinterpret_cast<float2*>(b4 + 1)[0] = make_float2(hi.y, hi.z);
        next.lo = lo;
        next.hi = hi;
        next.com = com;
        next.m = m;
        if (local) {
            LocalNode& q = snode[own - b0];
            q.lo = lo;
            q.hi = hi;
            q.com = com;
            q.m = m;
        }
        mine = next;
        from = node;
        node = up;
        cl = ncl;
        cr = ncr;
        up = nup;
        re = nre;
        have = node >= 0;  // the root ends the climb
    }
}

int tree_grid(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

void launch_build(const Layout& L, const uint64_t* keys, BvhNodeTraverse* tr, BvhNodeBuild* bd,
                  int32_t* leaf_parent, uint32_t* status, cudaStream_t st) {
    if (L.n <= 0) return;
    build_kernel<<<tree_grid(L.n), 256, 0, st>>>(L, keys, tr, bd, leaf_parent, status);
}

void launch_aggregate(const Layout& L, const float4* pos, BvhNodeTraverse* tr, BvhNodeBuild* bd,
                      double4* com64, const int32_t* leaf_parent, int com_fp64, const WalkNodeParams& wnp,
                      uint32_t* status, cudaStream_t st) {
    if (L.n <= 0) return;
    const unsigned blocks = (unsigned)((L.n + kAggRange - 1) / kAggRange);
    aggregate_kernel<<<blocks, kAggThreads, 0, st>>>(L, pos, tr, bd, com64, leaf_parent, com_fp64,
                                                             wnp, status);
}

void launch_walk_nodes(const Layout& L, const BvhNodeTraverse* tr, WalkNodeParams wnp, uint32_t* status,
                       cudaStream_t st) {
    if (L.n <= 0 || !wnp.wn) return;
    walk_nodes_kernel<<<tree_grid(L.n), 256, 0, st>>>(L, tr, wnp, status);
}

}  // namespace gcs
