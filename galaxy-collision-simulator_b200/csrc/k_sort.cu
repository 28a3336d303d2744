// k_sort.cu - stable LSD radix sort of (u64 Morton key, u32 position) pairs,
// one "onesweep" launch per 8-bit digit.
//
// Replaces cub::DeviceRadixSort::SortPairs (cuda_engine.cu:272,397).  The
// method is the single-pass LSD sort of Adinets & Merrill (2022): per pass,
// every tile of 4096 keys ranks its keys locally, publishes its per-digit
// counts, and learns the counts of all earlier tiles by decoupled look-back,
// so each key moves exactly once per pass.  This implementation:
//
//  * global digit histograms of all passes come from the encode kernel
//    (k_stream.cu), so no counting pass over the keys is needed;
//  * tiles are taken in launch order from an atomic ticket, so a tile only
//    ever waits on tiles that are already resident (forward progress);
//  * ranking is warp-local with 8 ballots per key (lanes with equal digits
//    are found by intersecting per-bit ballots) and a per-warp shared-memory
//    histogram; keys of warp w precede those of warp w+1 and items are
//    ranked in input order, so equal digits keep their input order (the sort
//    is stable, which makes position the tie-break, karras_bvh.cuh:40);
//  * a tile's keys and values are loaded right after its ticket, and the
//    global digit starts are scanned while those loads are in flight;
//  * look-back waits are bounded: a wait that runs out sets
//    GCS_DEV_SORT_LOOKBACK_TIMEOUT, the tile still publishes (so later tiles
//    finish) and skips its scatter, so nothing is written out of bounds;
//  * keys are scattered through shared memory so global writes come out as
//    runs of equal digits.
//
// With more than one segment, one or two further stable passes order by the
// segment id of each element's source position; the result is every segment
// sorted by key with position as the tie-break, as if sorted alone.
#include "gcs_internal.h"

namespace gcs {

namespace {

constexpr int kWarps = kSortThreads / 32;
constexpr uint32_t kFlagAggregate = 1u << 30;
constexpr uint32_t kFlagInclusive = 2u << 30;
constexpr uint32_t kCountMask = (1u << 30) - 1;
constexpr uint32_t kSpinLimit = 1u << 22;
constexpr int kLookWindow = 8;

struct SortSmem {
    uint64_t keys[kSortTile];
    uint32_t vals[kSortTile];
    uint8_t dig[kSortTile];
    uint32_t whist[kWarps][kRadix];
    uint32_t gbase[kRadix];
    uint32_t tstart[kRadix];
    int64_t final_base[kRadix];
    uint32_t warp_sums[kWarps];
    uint32_t tile;
    int bad;
};

// Exclusive scan of one value per thread over the 256-thread block.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_sums) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    uint32_t off = 0;
    for (int w = 0; w < warp; ++w) off += warp_sums[w];
    __syncthreads();
    return off + x - v;
}

template <bool kSegPass>
__global__ void __launch_bounds__(kSortThreads, 2)
onesweep_kernel(Layout L, int shift, const uint64_t* __restrict__ keys_in,
                const uint32_t* __restrict__ vals_in, uint64_t* __restrict__ keys_out,
                uint32_t* __restrict__ vals_out, const uint32_t* __restrict__ hist,
                uint32_t* __restrict__ tile_counter, uint32_t* __restrict__ lookback,
                uint32_t* __restrict__ status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem& S = *reinterpret_cast<SortSmem*>(smem_raw);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int64_t n = L.n;

    if (t == 0) {
        S.tile = atomicAdd(tile_counter, 1u);
        S.bad = 0;
    }
    for (int i = t; i < kWarps * kRadix; i += kSortThreads) (&S.whist[0][0])[i] = 0;
    const uint32_t h = hist[t];  // t == digit
    __syncthreads();
    const uint32_t tile = S.tile;
    const int64_t tile_base = (int64_t)tile * kSortTile;
    const int64_t warp_base = tile_base + (int64_t)warp * (kSortItems * 32);

    // ---- load (warp-striped: item j of lane l is warp_base + 32j + l); the
    // values come with the keys and the global digit starts are scanned while
    // the loads are in flight, so no later phase waits on global memory
    // except the look-back
    uint64_t key[kSortItems];
    uint32_t val[kSortItems];
    uint32_t rank[kSortItems];  // digit << 16 | rank within the warp's items
    const uint32_t lt_mask = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const int64_t i = warp_base + 32 * j + lane;
        const bool valid = i < n;
        key[j] = valid ? keys_in[i] : 0ull;
        val[j] = valid ? vals_in[i] : 0u;
    }
    S.gbase[t] = block_exclusive_scan(h, S.warp_sums);

    // ---- rank
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const int64_t i = warp_base + 32 * j + lane;
        const bool valid = i < n;
        uint32_t d;
        if (kSegPass) {
            d = valid ? (((uint32_t)__ldg(L.seg_id + val[j]) >> shift) & (kRadix - 1)) : 0u;
        } else {
            d = (uint32_t)(key[j] >> shift) & (kRadix - 1);
        }
        uint32_t peers = __ballot_sync(0xFFFFFFFFu, valid);
#pragma unroll
        for (int b = 0; b < kRadixBits; ++b) {
            const bool bit = (d >> b) & 1u;
            const uint32_t bb = __ballot_sync(0xFFFFFFFFu, bit);
            peers &= bit ? bb : ~bb;
        }
        const int leader = valid ? (__ffs(peers) - 1) : lane;
        uint32_t prev = 0;
        if (valid && lane == leader) prev = atomicAdd(&S.whist[warp][d], (uint32_t)__popc(peers));
        prev = __shfl_sync(0xFFFFFFFFu, prev, leader);
        rank[j] = (d << 16) | (prev + (uint32_t)__popc(peers & lt_mask));
    }
    __syncthreads();

    // ---- per-digit tile totals and warp prefixes (thread t owns digit t)
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        const uint32_t c = S.whist[w][t];
        S.whist[w][t] = total;
        total += c;
    }
    // Publish early so later tiles can proceed.
    volatile uint32_t* lb = lookback;
    lb[(int64_t)tile * kRadix + t] = (tile == 0 ? kFlagInclusive : kFlagAggregate) | total;
    const uint32_t tstart = block_exclusive_scan(total, S.warp_sums);
    S.tstart[t] = tstart;

    // ---- decoupled look-back for digit t
    // Predecessors are read kLookWindow at a time (independent loads in
    // flight together), nearest first, until an inclusive prefix is found;
    // an empty slot (a tile that has not published yet) restarts the window
    // there after a short sleep.
    uint32_t excl = 0;
    if (tile > 0) {
        int64_t prev = (int64_t)tile - 1;
        uint32_t spins = 0;
        while (prev >= 0) {
            uint32_t v[kLookWindow];
#pragma unroll
            for (int k = 0; k < kLookWindow; ++k) v[k] = prev - k >= 0 ? lb[(prev - k) * kRadix + t] : 0u;
            int k = 0;
            bool done = false;
            for (; k < kLookWindow && prev - k >= 0; ++k) {
                const uint32_t flag = v[k] & ~kCountMask;
                if (flag == 0u) break;
                excl += v[k] & kCountMask;
                if (flag == kFlagInclusive) {
                    done = true;
                    break;
                }
            }
            if (done) break;
            if (k < kLookWindow && prev - k >= 0) {  // stopped at an empty slot
                prev -= k;
                if (++spins > kSpinLimit) {
                    S.bad = 1;
                    atomicOr(status, GCS_DEV_SORT_LOOKBACK_TIMEOUT);
                    break;
                }
                __nanosleep(32);
                continue;
            }
            prev -= k;
        }
        lb[(int64_t)tile * kRadix + t] = kFlagInclusive | ((excl + total) & kCountMask);
    }
    S.final_base[t] = (int64_t)S.gbase[t] + excl - tstart;
    __syncthreads();

    // ---- scatter into shared memory in digit order
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const int64_t i = warp_base + 32 * j + lane;
        if (i < n) {
            const uint32_t d = rank[j] >> 16;
            const uint32_t lp = S.tstart[d] + S.whist[warp][d] + (rank[j] & 0xFFFFu);
            S.keys[lp] = key[j];
            S.vals[lp] = val[j];
            S.dig[lp] = (uint8_t)d;
        }
    }
    __syncthreads();

    // ---- write out: runs of equal digits land contiguously
    if (!S.bad) {
        const int64_t valid = (n - tile_base) < kSortTile ? (n - tile_base) : kSortTile;
        for (int q = t; q < valid; q += kSortThreads) {
            const int64_t g = S.final_base[S.dig[q]] + q;
            if (g >= 0 && g < n) {
                keys_out[g] = S.keys[q];
                vals_out[g] = S.vals[q];
            }
        }
    }
}

}  // namespace

size_t sort_lookback_words(int64_t n, int passes) {
    const int64_t tiles = (n + kSortTile - 1) / kSortTile;
    return (size_t)(tiles > 0 ? tiles : 1) * kRadix * passes;
}

void launch_sort_pass(const Layout& L, int pass, const uint64_t* keys_in, const uint32_t* vals_in,
                      uint64_t* keys_out, uint32_t* vals_out, const uint32_t* hist,
                      uint32_t* tile_counter, uint32_t* lookback, uint32_t* status,
                      cudaStream_t st) {
    if (L.n <= 0) return;
    const int64_t tiles = (L.n + kSortTile - 1) / kSortTile;
    const size_t smem = sizeof(SortSmem);
    static std::once_flag configured[kMaxDevices];
    once_per_device(configured, [smem] {
        cudaFuncSetAttribute(onesweep_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(onesweep_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    });
    uint32_t* lb = lookback + (size_t)pass * tiles * kRadix;
    if (pass < kKeyPasses) {
        onesweep_kernel<false><<<(unsigned)tiles, kSortThreads, smem, st>>>(
            L, kRadixBits * pass, keys_in, vals_in, keys_out, vals_out, hist + pass * kRadix,
            tile_counter + pass, lb, status);
    } else {
        onesweep_kernel<true><<<(unsigned)tiles, kSortThreads, smem, st>>>(
            L, kRadixBits * (pass - kKeyPasses), keys_in, vals_in, keys_out, vals_out,
            hist + pass * kRadix, tile_counter + pass, lb, status);
    }
}

}  // namespace gcs
