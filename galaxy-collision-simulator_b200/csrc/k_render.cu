// k_render.cu - headless point-splat renderer: the reference's GL point
// pipeline as CUDA kernels (no graphics stack exists on the target machines).
//
// Per particle (renderer.cpp:97-122, vertex attributes 226-233):
//   view-space position v = View * (x, y, z, 1)   (model = identity)
//   d = |v|, point size S = clamp(2500/d, 1, 6) for dark matter (type 1),
//   clamp(1000/d, 1, 3) otherwise; clip = Proj * v; points whose centre lies
//   outside the clip volume are culled; window position
//   (xw, yw) = ((ndc + 1) / 2) * (width, height).
// Per fragment (renderer.cpp:125-148): every pixel whose centre c lies in
//   [xw - S/2, xw + S/2) x [yw - S/2, yw + S/2); r^2 = |2 (c - w) / S|^2
//   (gl_PointCoord * 2 - 1); r^2 > 1 is discarded; alpha = exp(-3 r^2);
//   dark matter: colour (0.4, 0, 0.8), a = 0.03 alpha; stars: colour
//   rgb / 255, a = 0.15 alpha.
// Blending (renderer.cpp:202-204): glBlendFunc(GL_SRC_ALPHA, GL_ONE) adds
//   colour * a to the framebuffer, whose clear colour is (0.01, 0.01, 0.02, 1)
//   (renderer.cpp:248); its alpha starts at 1 and only grows, so it resolves
//   to 255.
// Each fragment's colour * a is rounded to 2^-24 units and summed with 64-bit
// atomics, so a frame is the same whatever order fragments arrive in; the
// resolve adds the clear colour, clamps to [0, 1] and rounds to 8 bits once.
#include <algorithm>

#include "gcs_internal.h"

namespace gcs {

namespace {

constexpr float kFixScale = 16777216.0f;  // 2^24 units per colour unit

struct RenderMats {
    float view[16];  // row-major, column vectors
    float proj[16];
    int32_t width, height;
};

// Position and packed type|r|g|b of particle i, from the engine's arrays or
// from Star records (Star bytes 28..31 are the same packed word).
struct PosVelSource {
    const float4* pos;
    const float4* vel;
    __device__ __forceinline__ void get(int64_t i, float& x, float& y, float& z, uint32_t& tcol) const {
        const float4 p = __ldg(pos + i);
        x = p.x;
        y = p.y;
        z = p.z;
        tcol = __float_as_uint(__ldg(vel + i).w);
    }
};
struct StarSource {
    const Star* stars;
    __device__ __forceinline__ void get(int64_t i, float& x, float& y, float& z, uint32_t& tcol) const {
        const float4* s = reinterpret_cast<const float4*>(stars + i);
        const float4 a = __ldg(s);
        x = a.x;
        y = a.y;
        z = a.z;
        tcol = __float_as_uint(__ldg(s + 1).w);
    }
};

// Position and packed type|r|g|b from PlaybackStar records (bytes 12..15 are
// r, g, b, type: the same word rotated by one byte).
struct PlaybackSource {
    const PlaybackStar* recs;
    __device__ __forceinline__ void get(int64_t i, float& x, float& y, float& z, uint32_t& tcol) const {
        const float4 a = __ldg(reinterpret_cast<const float4*>(recs + i));
        x = a.x;
        y = a.y;
        z = a.z;
        const uint32_t w = __float_as_uint(a.w);
        tcol = (w << 8) | (w >> 24);
    }
};

// Row r of a 4x4 row-major matrix times (x, y, z, 1).
__device__ __forceinline__ float row_dot(const float* m, int r, float x, float y, float z) {
    return __fmaf_rn(m[4 * r + 0], x, __fmaf_rn(m[4 * r + 1], y, __fmaf_rn(m[4 * r + 2], z, m[4 * r + 3])));
}
__device__ __forceinline__ float row_dot4(const float* m, int r, float x, float y, float z, float w) {
    return __fmaf_rn(m[4 * r + 0], x,
                     __fmaf_rn(m[4 * r + 1], y, __fmaf_rn(m[4 * r + 2], z, __fmul_rn(m[4 * r + 3], w))));
}

// One thread per particle (grid-stride); each fragment is one 64-bit atomic
// add per non-zero channel.  (Summing a warp's fragments on the same pixel
// first, with __match_any_sync and __reduce_add_sync over fragments walked in
// step, was measured 2.8x slower: the walk runs to the warp's largest point.)
template <class Src>
__global__ void __launch_bounds__(256) splat_kernel(Src src, int64_t n, RenderMats M,
                                                    unsigned long long* __restrict__ acc) {
    const int W = M.width, H = M.height;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float x, y, z;
        uint32_t tcol;
        src.get(i, x, y, z, tcol);
        const float vx = row_dot(M.view, 0, x, y, z);
        const float vy = row_dot(M.view, 1, x, y, z);
        const float vz = row_dot(M.view, 2, x, y, z);
        const float vw = row_dot(M.view, 3, x, y, z);
        const float dist = __fsqrt_rn(__fmaf_rn(vz, vz, __fmaf_rn(vy, vy, __fmul_rn(vx, vx))));
        const bool dm = (tcol & 0xFFu) == 1u;
        const float size = dm ? fminf(fmaxf(__fdiv_rn(2500.0f, dist), 1.0f), 6.0f)
                              : fminf(fmaxf(__fdiv_rn(1000.0f, dist), 1.0f), 3.0f);
        const float cx = row_dot4(M.proj, 0, vx, vy, vz, vw);
        const float cy = row_dot4(M.proj, 1, vx, vy, vz, vw);
        const float cz = row_dot4(M.proj, 2, vx, vy, vz, vw);
        const float cw = row_dot4(M.proj, 3, vx, vy, vz, vw);
        // the point is clipped by its centre (also drops NaN positions)
        if (!(cw > 0.0f && fabsf(cx) <= cw && fabsf(cy) <= cw && fabsf(cz) <= cw)) continue;
        const float xw = __fmaf_rn(__fdiv_rn(cx, cw), 0.5f * W, 0.5f * W);
        const float yw = __fmaf_rn(__fdiv_rn(cy, cw), 0.5f * H, 0.5f * H);
        const float half = __fmul_rn(size, 0.5f);
        // pixels i with xw - half <= i + 0.5 < xw + half
        const int i0 = max((int)ceilf(__fsub_rn(__fsub_rn(xw, half), 0.5f)), 0);
        const int i1 = min((int)ceilf(__fsub_rn(__fadd_rn(xw, half), 0.5f)) - 1, W - 1);
        const int j0 = max((int)ceilf(__fsub_rn(__fsub_rn(yw, half), 0.5f)), 0);
        const int j1 = min((int)ceilf(__fsub_rn(__fadd_rn(yw, half), 0.5f)) - 1, H - 1);
        float cr, cg, cb, amul;
        if (dm) {
            cr = 0.4f;
            cg = 0.0f;
            cb = 0.8f;
            amul = 0.03f;
        } else {
            cr = __fdiv_rn((float)((tcol >> 8) & 0xFFu), 255.0f);
            cg = __fdiv_rn((float)((tcol >> 16) & 0xFFu), 255.0f);
            cb = __fdiv_rn((float)(tcol >> 24), 255.0f);
            amul = 0.15f;
        }
        for (int pj = j0; pj <= j1; ++pj) {
            const float py = __fdiv_rn(__fmul_rn(2.0f, __fsub_rn(__fadd_rn((float)pj, 0.5f), yw)), size);
            for (int pi = i0; pi <= i1; ++pi) {
                const float px = __fdiv_rn(__fmul_rn(2.0f, __fsub_rn(__fadd_rn((float)pi, 0.5f), xw)), size);
                const float r2 = __fmaf_rn(py, py, __fmul_rn(px, px));
                if (r2 > 1.0f) continue;
                const float a = __fmul_rn(expf(__fmul_rn(-r2, 3.0f)), amul);
                unsigned long long* px_acc = acc + 3 * ((size_t)pj * W + pi);
                const unsigned long long ur = __float2ull_rn(__fmul_rn(__fmul_rn(cr, a), kFixScale));
                const unsigned long long ug = __float2ull_rn(__fmul_rn(__fmul_rn(cg, a), kFixScale));
                const unsigned long long ub = __float2ull_rn(__fmul_rn(__fmul_rn(cb, a), kFixScale));
                if (ur) atomicAdd(px_acc + 0, ur);
                if (ug) atomicAdd(px_acc + 1, ug);
                if (ub) atomicAdd(px_acc + 2, ub);
            }
        }
    }
}

// Clear colour + sums, clamped and rounded to 8 bits; alpha is 255.
__global__ void resolve_kernel(const unsigned long long* __restrict__ acc, int64_t pixels,
                               uchar4* __restrict__ rgba) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= pixels) return;
    const double clear[3] = {(double)0.01f, (double)0.01f, (double)0.02f};
    unsigned char c[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double v = fmin(clear[k] + (double)acc[3 * p + k] * (1.0 / 16777216.0), 1.0);
        c[k] = (unsigned char)__double2int_rn(v * 255.0);
    }
    rgba[p] = make_uchar4(c[0], c[1], c[2], 255);
}

int splat_grid(int64_t n) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t blocks = (n + 255) / 256;
    return (int)std::max<int64_t>(1, std::min<int64_t>(blocks, (int64_t)sms * 16));
}

RenderMats mats_of(const float* view, const float* proj, int width, int height) {
    RenderMats M;
    for (int k = 0; k < 16; ++k) {
        M.view[k] = view[k];
        M.proj[k] = proj[k];
    }
    M.width = width;
    M.height = height;
    return M;
}

}  // namespace

void launch_splat_posvel(const float4* pos, const float4* vel, int64_t n, const float* view, const float* proj,
                         int width, int height, unsigned long long* acc, cudaStream_t st) {
    if (n <= 0) return;
    splat_kernel<<<splat_grid(n), 256, 0, st>>>(PosVelSource{pos, vel}, n, mats_of(view, proj, width, height), acc);
}

void launch_splat_stars(const Star* stars, int64_t n, const float* view, const float* proj, int width, int height,
                        unsigned long long* acc, cudaStream_t st) {
    if (n <= 0) return;
    splat_kernel<<<splat_grid(n), 256, 0, st>>>(StarSource{stars}, n, mats_of(view, proj, width, height), acc);
}

void launch_splat_playback(const PlaybackStar* recs, int64_t n, const float* view, const float* proj, int width,
                           int height, unsigned long long* acc, cudaStream_t st) {
    if (n <= 0) return;
    splat_kernel<<<splat_grid(n), 256, 0, st>>>(PlaybackSource{recs}, n, mats_of(view, proj, width, height), acc);
}

void launch_resolve(const unsigned long long* acc, int64_t pixels, uint8_t* rgba, cudaStream_t st) {
    if (pixels <= 0) return;
    resolve_kernel<<<(unsigned)((pixels + 255) / 256), 256, 0, st>>>(acc, pixels, reinterpret_cast<uchar4*>(rgba));
}

}  // namespace gcs
