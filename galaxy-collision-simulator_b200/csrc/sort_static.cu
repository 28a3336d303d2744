// sort_static.cu - a stable (u64 key, u32 value) radix sort that allocates
// nothing: the sort's working state lives in one file-scope device array.
//
// Who needs it: code that cannot call cudaMalloc at the point where it has to
// sort - a step running inside a real-time loop or a host callback where the
// implicit device synchronisation of an allocation is not allowed, or a
// plug-in inside a host application that owns the device memory budget and
// forbids allocations of its own.  The reference's own sort asks the caller
// for temporary storage (cub::DeviceRadixSort::SortPairs with d_temp_storage,
// cuda_engine.cu:272-273); this entry point needs none: the caller passes the
// pairs and a second pair of arrays of the same length for the passes, and
// the histograms, tile tickets and look-back state come from g_sort_scratch.
//
// Costs and limits of the shared array:
//   * at most kStaticSortMax (1,048,576) pairs per call; larger sizes are
//     rejected with GCS_ERR_CAPACITY;
//   * the array (about 2.1 MB) is held by every GPU that loads this library
//     until the process exits;
//   * every call uses the same array and leaves its contents behind; each
//     call clears what must start at zero (histograms, tickets, look-back)
//     on its own stream before its kernels run, so calls queued one after
//     another are independent, but two calls whose work overlaps on the GPU
//     (different streams, or different host threads without ordering) race
//     on the array and corrupt each other;
//   * the first call on a device looks up that device's address of the array
//     (cudaGetSymbolAddress, with the device current) and keeps it; make that
//     first call before any stream capture on the device;
//   * with a caller status word the call only queues work on its stream; with
//     status == NULL it waits for its stream to finish and reads the array's
//     own status word, so that a look-back that gave up (a tile whose scatter
//     was skipped) is returned as GCS_ERR_DEVICE instead of going unseen.
#include <cstdio>
#include <mutex>

#include "gcs_internal.h"

namespace gcs {
namespace {

constexpr int64_t kStaticSortMax = int64_t(1) << 20;
constexpr size_t kStaticTiles = (size_t)((kStaticSortMax + kSortTile - 1) / kSortTile);
// word offsets inside the array
constexpr size_t kHistWords = (size_t)kKeyPasses * kRadix;      // digit histograms of all passes
constexpr size_t kTicketWords = 64;                             // one tile ticket per pass (padded)
constexpr size_t kStatusWords = 64;                             // fallback status word (padded)
constexpr size_t kLookbackWords = kStaticTiles * kRadix * kKeyPasses;
constexpr size_t kScratchWords = kHistWords + kTicketWords + kStatusWords + kLookbackWords;

}  // namespace

// The sort's working state.  In host code this name is only a handle for
// cudaGetSymbolAddress: its device address differs per device and is looked
// up once per device below; device code may name it directly.
static __device__ __align__(256) uint32_t g_sort_scratch[kScratchWords];

namespace {

std::mutex g_mu;
uint32_t* g_scratch_addr[kMaxDevices] = {};

// Digit histograms of all 8 key digits (what the engine's encode kernel
// accumulates for its own sort).
__global__ void key_histograms_kernel(const uint64_t* __restrict__ keys, int64_t n, uint32_t* __restrict__ hist) {
    __shared__ uint32_t s[kKeyPasses][kRadix];
    for (int t = threadIdx.x; t < kKeyPasses * kRadix; t += blockDim.x) (&s[0][0])[t] = 0u;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = __ldg(keys + i);
#pragma unroll
        for (int d = 0; d < kKeyPasses; ++d) atomicAdd(&s[d][(uint32_t)(k >> (kRadixBits * d)) & (kRadix - 1)], 1u);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < kKeyPasses * kRadix; t += blockDim.x) {
        const uint32_t c = (&s[0][0])[t];
        if (c) atomicAdd(hist + t, c);
    }
}

// Device address of g_sort_scratch on the current device (looked up once).
int scratch_address(uint32_t** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return GCS_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "gcs_sort_pairs_static: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return GCS_ERR_CUDA;
        }
        g_scratch_addr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_scratch_addr[dev];
    return GCS_OK;
}

}  // namespace
}  // namespace gcs

extern "C" int gcs_sort_pairs_static(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt,
                                     int64_t n, uint32_t* status, void* stream) {
    using namespace gcs;
    if (n < 0) return GCS_ERR_ARG;
    if (n > kStaticSortMax) {
        fprintf(stderr, "gcs_sort_pairs_static: %lld pairs exceed the static scratch limit of %lld\n",
                (long long)n, (long long)kStaticSortMax);
        return GCS_ERR_CAPACITY;
    }
    if (n == 0) return GCS_OK;
    if (!keys || !vals || !keys_alt || !vals_alt) return GCS_ERR_ARG;
    uint32_t* base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    uint32_t* hist = base;
    uint32_t* tickets = base + kHistWords;
    uint32_t* own_status = tickets + kTicketWords;
    uint32_t* lookback = own_status + kStatusWords;
    const int64_t tiles = (n + kSortTile - 1) / kSortTile;
    const size_t clear_words = kHistWords + kTicketWords + kStatusWords + (size_t)tiles * kRadix * kKeyPasses;
    if (cudaMemsetAsync(base, 0, clear_words * sizeof(uint32_t), st) != cudaSuccess) return GCS_ERR_CUDA;
    int64_t grid = (n + 255) / 256;
    const int64_t cap = (int64_t)current_sm_count() * 8;  // 8 resident 256-thread blocks per SM
    if (grid > cap) grid = cap;
    key_histograms_kernel<<<(unsigned)grid, 256, 0, st>>>(keys, n, hist);
    Layout L;
    L.n = (int32_t)n;
    L.nseg = 1;
    L.n_internal = (int32_t)(n - 1);
    L.seg_off = nullptr;
    L.seg_id = nullptr;
    uint32_t* stat = status ? status : own_status;
    uint64_t* kb[2] = {keys, keys_alt};
    uint32_t* vb[2] = {vals, vals_alt};
    for (int pass = 0; pass < kKeyPasses; ++pass) {  // even count: the result lands back in keys/vals
        const int in = pass & 1;
        launch_sort_pass(L, pass, kb[in], vb[in], kb[in ^ 1], vb[in ^ 1], hist, tickets, lookback, stat, st);
    }
    if (cudaGetLastError() != cudaSuccess) return GCS_ERR_CUDA;
    if (status) return GCS_OK;
    // no caller status word: wait and read the array's own, so that a pass
    // that gave up is reported (pageable destination: no allocation)
    uint32_t seen = 0;
    if (cudaMemcpyAsync(&seen, own_status, sizeof seen, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return GCS_ERR_CUDA;
    return seen ? GCS_ERR_DEVICE : GCS_OK;
}
