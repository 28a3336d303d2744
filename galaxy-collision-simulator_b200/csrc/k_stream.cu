// k_stream.cu - the HBM-streaming stages: Star <-> SoA transposes, per-segment
// bounds, Morton encode (+ sort histograms), gather, kick+drift+colour,
// FP64 diagnostics and the FP64 direct sum.
//
// All particle records are float4 (16-byte) loads/stores; grids are sized
// as a multiple of the SM count with grid-stride loops.
#include <atomic>

#include "gcs_internal.h"
#include "device_math.cuh"

namespace gcs {

int current_device() {
    int dev = -1;
    return cudaGetDevice(&dev) == cudaSuccess ? dev : -1;
}

int current_sm_count() {
    static std::atomic<int> cached[kMaxDevices] = {};
    const int dev = current_device();
    if (dev >= 0 && dev < kMaxDevices) {
        const int v = cached[dev].load(std::memory_order_relaxed);
        if (v > 0) return v;
    }
    int sms = 0;
    if (dev < 0 || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        sms = 148;
    if (dev >= 0 && dev < kMaxDevices) cached[dev].store(sms, std::memory_order_relaxed);
    return sms;
}

namespace {

constexpr int kStreamThreads = 256;

int stream_grid(int64_t n) {
    const int sms = current_sm_count();
    int64_t want = (n + kStreamThreads - 1) / kStreamThreads;
    int64_t cap = (int64_t)sms * 8;
    if (want > cap) want = cap;
    if (want < 1) want = 1;
    return (int)want;
}

// seg_id[i] = the segment s with seg_off[s] <= i < seg_off[s+1] (binary
// search over the nseg+1 offsets, which stay in L1).
__global__ void fill_segment_ids_kernel(const int64_t* __restrict__ seg_off, int nseg,
                                        int32_t* __restrict__ seg_id, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = nseg - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(seg_off + mid) <= i) lo = mid;
            else hi = mid - 1;
        }
        seg_id[i] = lo;
    }
}

// Star (x,y,z,vx | vy,vz,m,tcol) <-> pos (x,y,z,m), vel (vx,vy,vz,tcol).
__global__ void unpack_stars_kernel(const float4* __restrict__ stars, float4* __restrict__ pos,
                                    float4* __restrict__ vel, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float4 a = __ldg(stars + 2 * i);
        const float4 b = __ldg(stars + 2 * i + 1);
        pos[i] = make_float4(a.x, a.y, a.z, b.z);
        vel[i] = make_float4(a.w, b.x, b.y, b.w);
    }
}

__global__ void pack_stars_kernel(const float4* __restrict__ pos, const float4* __restrict__ vel,
                                  float4* __restrict__ stars, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        store_star(stars, i, pos[i], vel[i]);
    }
}

// PlaybackStar = x, y, z, r, g, b, type (main.cpp:266 writes type into the
// padding byte).
__global__ void pack_playback_kernel(const float4* __restrict__ pos, const float4* __restrict__ vel,
                                     float4* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float4 p = pos[i];
        const uint32_t tcol = __float_as_uint(vel[i].w);
        const uint32_t rgbt = (tcol >> 8) | ((tcol & 0xFFu) << 24);
        out[i] = make_float4(p.x, p.y, p.z, __uint_as_float(rgbt));
    }
}

// Per-segment min/max over x, y and z of every particle (main.cpp:152-166
// reduces one scalar min and max over all three axes).  min/max is exact in
// any precision, so the reduction runs in FP32.  Each block takes chunks
// that never straddle a segment, reduces in registers and warp shuffles, and
// publishes with one atomicMax per chunk on order-preserving encodings
// (min stored as the max of ~enc), so a zeroed buffer is a valid start.
__global__ void bounds_kernel(const float4* __restrict__ pos, const Chunk* __restrict__ chunks,
                              int n_chunks, uint32_t* __restrict__ bounds_enc,
                              uint32_t* __restrict__ status) {
    constexpr int kInFlight = 8;  // independent loads per thread per sweep
    __shared__ float s_lo[kStreamThreads / 32], s_hi[kStreamThreads / 32];
    for (int c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        const Chunk ch = chunks[c];
        float lo = INFINITY, hi = -INFINITY;
        bool bad = false;
        for (int i0 = threadIdx.x; i0 < ch.count; i0 += kInFlight * blockDim.x) {
            float4 p[kInFlight];
#pragma unroll
            for (int k = 0; k < kInFlight; ++k) {
                const int i = i0 + k * blockDim.x;
                p[k] = i < ch.count ? __ldg(pos + ch.start + i) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int k = 0; k < kInFlight; ++k) {
                if (i0 + k * (int)blockDim.x < ch.count) {
                    bad |= !(isfinite(p[k].x) && isfinite(p[k].y) && isfinite(p[k].z));
                    lo = fminf(lo, fminf(p[k].x, fminf(p[k].y, p[k].z)));
                    hi = fmaxf(hi, fmaxf(p[k].x, fmaxf(p[k].y, p[k].z)));
                }
            }
        }
        if (__any_sync(0xFFFFFFFFu, bad) && (threadIdx.x & 31) == 0)
            atomicOr(status, GCS_DEV_NONFINITE_POSITION);
        for (int o = 16; o > 0; o >>= 1) {
            lo = fminf(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
            hi = fmaxf(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, o));
        }
        const int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) {
            s_lo[w] = lo;
            s_hi[w] = hi;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
                lo = fminf(lo, s_lo[k]);
                hi = fmaxf(hi, s_hi[k]);
            }
            atomicMax(bounds_enc + 2 * ch.seg, ~float_to_ordered(lo));
            atomicMax(bounds_enc + 2 * ch.seg + 1, float_to_ordered(hi));
        }
        __syncthreads();
    }
}

__global__ void bounds_decode_kernel(const uint32_t* __restrict__ enc, float2* __restrict__ out,
                                     int nseg) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x)
        out[s] = make_float2(ordered_to_float(~enc[2 * s]), ordered_to_float(enc[2 * s + 1]));
}

// keys[i] = 63-bit Morton code of particle i in its segment's cube; idx[i] = i
// (karras_bvh.cuh:34-41).  The radix sort's global digit histograms (8 key
// digits, plus the segment-id digits when there is more than one segment)
// are accumulated here in shared memory, so the sort needs no separate
// counting pass over the keys.
__global__ void encode_kernel(Layout L, const float4* __restrict__ pos, int bounds_mode,
                              float gmin, float gmax, const float2* __restrict__ seg_bounds,
                              uint64_t* __restrict__ keys, uint32_t* __restrict__ idx,
                              uint32_t* __restrict__ hist, int n_seg_passes) {
    __shared__ uint32_t s_hist[kMaxPasses][kRadix];
    const int passes = kKeyPasses + n_seg_passes;
    for (int t = threadIdx.x; t < passes * kRadix; t += blockDim.x) (&s_hist[0][0])[t] = 0;
    __syncthreads();
    float lo = gmin, scale = 0.0f;
    int cur_seg = -1;
    if (bounds_mode == GCS_BOUNDS_CALLER) scale = morton_scale(gmin, gmax);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float4 p = __ldg(pos + i);
        const int seg = (L.nseg > 1) ? __ldg(L.seg_id + i) : 0;
        if (bounds_mode != GCS_BOUNDS_CALLER && seg != cur_seg) {
            const float2 b = __ldg(seg_bounds + seg);
            lo = b.x;
            scale = morton_scale(b.x, b.y);
            cur_seg = seg;
        }
        const uint64_t k = morton63(p.x, p.y, p.z, lo, scale);
        keys[i] = k;
        idx[i] = (uint32_t)i;
#pragma unroll
        for (int d = 0; d < kKeyPasses; ++d)
            atomicAdd(&s_hist[d][(uint32_t)(k >> (kRadixBits * d)) & (kRadix - 1)], 1u);
        for (int d = 0; d < n_seg_passes; ++d)
            atomicAdd(&s_hist[kKeyPasses + d][((uint32_t)seg >> (kRadixBits * d)) & (kRadix - 1)], 1u);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < passes * kRadix; t += blockDim.x) {
        const uint32_t c = (&s_hist[0][0])[t];
        if (c) atomicAdd(hist + t, c);
    }
}

// Permute the particle state into sorted order (karras_bvh.cuh:44-70):
// out[k] = in[idx[k]] for the two 16-byte records.
__global__ void gather_kernel(const uint32_t* __restrict__ idx, const float4* __restrict__ pos_in,
                              const float4* __restrict__ vel_in, float4* __restrict__ pos_out,
                              float4* __restrict__ vel_out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t s = __ldg(idx + i);
        if ((int64_t)s >= n) continue;  // only after a sort that timed out (in the status word)
        pos_out[i] = __ldg(pos_in + s);
        vel_out[i] = __ldg(vel_in + s);
    }
}

// v += a dt; x += v dt; recolour types 0/2 by speed (kick_drift,
// cuda_engine.cu:164-216), in place.
__global__ void integrate_kernel(float4* __restrict__ pos, float4* __restrict__ vel,
                                 const float4* __restrict__ acc, float dt, int recolor, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float4 a = __ldg(acc + i);
        float4 v = vel[i];
        float4 p = pos[i];
        kick_drift(p, v, a, dt, recolor);
        vel[i] = v;
        pos[i] = p;
    }
}

__global__ void kick_kernel(float4* __restrict__ vel, const float4* __restrict__ acc, float dt,
                            int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float4 a = __ldg(acc + i);
        float4 v = vel[i];
        v.x = __fmaf_rn(a.x, dt, v.x);
        v.y = __fmaf_rn(a.y, dt, v.y);
        v.z = __fmaf_rn(a.z, dt, v.z);
        vel[i] = v;
    }
}

// FP64 kinetic energy, momentum, mass and potential energy of particles
// [first, first+n).  out = {KE, px, py, pz, M, PE}; PE = 0.5 sum m phi with
// phi from the walk's potential lane (acc.w).  Blocks reduce in shared
// memory and add with FP64 atomics.
// Velocities enter as v + a * kick (in FP64): kick = dt/2 turns the stored
// half-step velocities of the leapfrog into synchronised ones.
__global__ void diag_kernel(const float4* __restrict__ pos, const float4* __restrict__ vel,
                            const float4* __restrict__ accp, int64_t first, int64_t n, double kick,
                            double* __restrict__ out) {
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float4 p = __ldg(pos + first + i);
        const float4 v = __ldg(vel + first + i);
        const float4 a = __ldg(accp + first + i);
        const double m = p.w;
        const double vx = (double)v.x + (double)a.x * kick;
        const double vy = (double)v.y + (double)a.y * kick;
        const double vz = (double)v.z + (double)a.z * kick;
        acc[0] += 0.5 * m * (vx * vx + vy * vy + vz * vz);
        acc[1] += m * vx;
        acc[2] += m * vy;
        acc[3] += m * vz;
        acc[4] += m;
        acc[5] += 0.5 * m * (double)a.w;
    }
    __shared__ double s[6][kStreamThreads / 32];
    for (int k = 0; k < 6; ++k) {
        double x = acc[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, o);
        if ((threadIdx.x & 31) == 0) s[k][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double x = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += s[threadIdx.x][w];
        atomicAdd(out + threadIdx.x, x);
    }
}

// FP64 direct sum: one block per target, sources of the segment streamed by
// the block's threads, excluding only the target itself.
__global__ void direct_fp64_kernel(const float4* __restrict__ pos, int64_t seg_first, int64_t seg_n,
                                   const int64_t* __restrict__ targets, int64_t n_targets, double G,
                                   double eps2, double* __restrict__ out) {
    for (int64_t t = blockIdx.x; t < n_targets; t += gridDim.x) {
        const int64_t ti = targets[t];
        const float4 pt = __ldg(pos + seg_first + ti);
        double ax = 0, ay = 0, az = 0;
        for (int64_t j = threadIdx.x; j < seg_n; j += blockDim.x) {
            if (j == ti) continue;
            const float4 ps = __ldg(pos + seg_first + j);
            const double dx = (double)ps.x - pt.x, dy = (double)ps.y - pt.y, dz = (double)ps.z - pt.z;
            const double r2 = dx * dx + dy * dy + dz * dz + eps2;
            const double inv = 1.0 / sqrt(r2);
            const double f = G * (double)ps.w * inv * inv * inv;
            ax += f * dx;
            ay += f * dy;
            az += f * dz;
        }
        __shared__ double s[3][kStreamThreads / 32];
        for (int o = 16; o > 0; o >>= 1) {
            ax += __shfl_xor_sync(0xFFFFFFFFu, ax, o);
            ay += __shfl_xor_sync(0xFFFFFFFFu, ay, o);
            az += __shfl_xor_sync(0xFFFFFFFFu, az, o);
        }
        if ((threadIdx.x & 31) == 0) {
            s[0][threadIdx.x >> 5] = ax;
            s[1][threadIdx.x >> 5] = ay;
            s[2][threadIdx.x >> 5] = az;
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            double x = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += s[threadIdx.x][w];
            out[3 * t + threadIdx.x] = x;
        }
        __syncthreads();
    }
}

}  // namespace

void launch_fill_segment_ids(const int64_t* seg_off, int nseg, int32_t* seg_id, int64_t n,
                             cudaStream_t st) {
    if (n <= 0) return;
    fill_segment_ids_kernel<<<stream_grid(n), kStreamThreads, 0, st>>>(seg_off, nseg, seg_id, n);
}

void launch_unpack_stars(const Star* stars, float4* pos, float4* vel, int64_t n, cudaStream_t st) {
    if (n <= 0) return;
    unpack_stars_kernel<<<stream_grid(n), kStreamThreads, 0, st>>>(
        reinterpret_cast<const float4*>(stars), pos, vel, n);
}

void launch_pack_stars(const float4* pos, const float4* vel, Star* out, int64_t n, cudaStream_t st) {
    if (n <= 0) return;
    pack_stars_kernel<<<stream_grid(n), kStreamThreads, 0, st>>>(pos, vel,
                                                                 reinterpret_cast<float4*>(out), n);
}

void launch_pack_playback(const float4* pos, const float4* vel, PlaybackStar* out, int64_t n,
                          cudaStream_t st) {
    if (n <= 0) return;
    pack_playback_kernel<<<stream_grid(n), kStreamThreads, 0, st>>>(
        pos, vel, reinterpret_cast<float4*>(out), n);
}

void launch_bounds(const Layout& L, const float4* pos, const Chunk* chunks, int n_chunks,
                   uint32_t* bounds_enc, uint32_t* status, cudaStream_t st) {
    if (n_chunks <= 0) return;
    int grid = stream_grid(L.n);
    if (grid > n_chunks) grid = n_chunks;
    bounds_kernel<<<grid, kStreamThreads, 0, st>>>(pos, chunks, n_chunks, bounds_enc, status);
}

void launch_bounds_decode(const uint32_t* bounds_enc, float2* bounds, int nseg, cudaStream_t st) {
    bounds_decode_kernel<<<(nseg + 255) / 256, 256, 0, st>>>(bounds_enc, bounds, nseg);
}

void launch_encode(const Layout& L, const float4* pos, int bounds_mode, float gmin, float gmax,
                   const float2* seg_bounds, uint64_t* keys, uint32_t* idx, uint32_t* hist,
                   int n_seg_passes, cudaStream_t st) {
    if (L.n <= 0) return;
    encode_kernel<<<stream_grid(L.n), kStreamThreads, 0, st>>>(L, pos, bounds_mode, gmin, gmax,
                                                                seg_bounds, keys, idx, hist,
                                                                n_seg_passes);
}

void launch_gather(const uint32_t* idx, const float4* pos_in, const float4* vel_in, float4* pos_out,
                   float4* vel_out, int64_t n, cudaStream_t st) {
    if (n <= 0) return;
    gather_kernel<<<stream_grid(n), kStreamThreads, 0, st>>>(idx, pos_in, vel_in, pos_out, vel_out,
                                                             n);
}

void launch_integrate(float4* pos, float4* vel, const float4* acc, float dt, int recolor,
                      int64_t n, cudaStream_t st) {
    if (n <= 0) return;
    integrate_kernel<<<stream_grid(n), kStreamThreads, 0, st>>>(pos, vel, acc, dt, recolor, n);
}

void launch_kick(float4* vel, const float4* acc, float dt, int64_t n, cudaStream_t st) {
    if (n <= 0) return;
    kick_kernel<<<stream_grid(n), kStreamThreads, 0, st>>>(vel, acc, dt, n);
}

void launch_diag(const float4* pos, const float4* vel, const float4* acc, int64_t first, int64_t n,
                 double kick, double* out6, cudaStream_t st) {
    if (n <= 0) return;
    diag_kernel<<<stream_grid(n), kStreamThreads, 0, st>>>(pos, vel, acc, first, n, kick, out6);
}

void launch_direct_fp64(const float4* pos, int64_t seg_first, int64_t seg_n, const int64_t* targets,
                        int64_t n_targets, double G, double eps2, double* out, cudaStream_t st) {
    if (n_targets <= 0) return;
    int grid = (int)(n_targets < 148 * 16 ? n_targets : 148 * 16);
    direct_fp64_kernel<<<grid, kStreamThreads, 0, st>>>(pos, seg_first, seg_n, targets, n_targets, G,
                                                        eps2, out);
}

}  // namespace gcs
