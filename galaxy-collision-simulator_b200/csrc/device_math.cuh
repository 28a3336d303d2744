// device_math.cuh - the arithmetic the engine must share bit for bit with the
// reference's GPU path and with the oracle's C restatement.
//
// Every expression whose rounding decides a result (a Morton code, a node
// opening decision, a colour byte) is written here once, with explicit
// round-to-nearest intrinsics, so the compiler cannot contract it
// differently in different kernels.  The oracle (oracle/gcs_oracle.c)
// restates each of these with fmaf() in the same order.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gcs {

// ---- Morton code (morton.h:11-28) ---------------------------------------
// Spread the low 21 bits of v so that bit k lands on bit 3k.  Five
// mask-and-shift rounds, each halving the distance between bit groups.
__host__ __device__ __forceinline__ uint64_t spread21(uint32_t v) {
    uint64_t x = v & 0x1FFFFFu;
    x = (x | (x << 32)) & 0x001F00000000FFFFull;
    x = (x | (x << 16)) & 0x001F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

// Quantise one coordinate to the 21-bit grid of the [lo, lo + 2097151/scale]
// cube: (c - lo) * scale, truncated toward zero.  The reference's
// static_cast<uint32_t>(float) compiles on the GPU to a saturating
// round-toward-zero conversion (negatives and NaN -> 0, >= 2^32 -> 2^32-1);
// __float2uint_rz is that conversion.  Values >= 2^21 keep only their low 21
// bits after spread21 (the reference's wrap at c == max).
__device__ __forceinline__ uint32_t quantise21(float c, float lo, float scale) {
    return __float2uint_rz(__fmul_rn(__fsub_rn(c, lo), scale));
}

// scale = 2097151 / (max - min), IEEE single-precision division as in
// morton.h:22 (nvcc's default -prec-div=true).
__device__ __forceinline__ float morton_scale(float lo, float hi) {
    return __fdiv_rn(2097151.0f, __fsub_rn(hi, lo));
}

__device__ __forceinline__ uint64_t morton63(float x, float y, float z, float lo, float scale) {
    return (spread21(quantise21(x, lo, scale)) << 2) | (spread21(quantise21(y, lo, scale)) << 1) |
           spread21(quantise21(z, lo, scale));
}

// ---- softened distance (cuda_engine.cu:128-131) ---------------------------
// d2 = dx*dx + dy*dy + dz*dz + eps^2, evaluated as
// fma(dz, dz, fma(dy, dy, dx*dx)) + eps^2.
__device__ __forceinline__ float softened_d2(float dx, float dy, float dz, float eps2) {
    return __fadd_rn(__fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx))), eps2);
}

// ---- 1/sqrt of a softened distance ------------------------------------------
// The reference's rsqrtf (cuda_engine.cu:135,144) is the hardware reciprocal
// square root; for normal inputs the flush-to-zero form below returns the
// same value without the subnormal-input fix-up, and d2 >= eps^2 > 0 here.
__device__ __forceinline__ float rsqrt_approx(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Two softened distances at once (sm_100 packed FP32): each element is
// rounded exactly as softened_d2 rounds it.
__device__ __forceinline__ float2 softened_d2_x2(float2 dx, float2 dy, float2 dz, float2 eps2) {
    return __fadd2_rn(__ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx))), eps2);
}

// ---- opening criterion (cuda_engine.cu:143 with theta) ---------------------
// A node is used as a monopole iff width^2 < theta^2 * d2 (d2 softened).
// width^2 is formed once per node when it is staged.
__device__ __forceinline__ bool accept_monopole(float width_sq, float d2, float theta2) {
    return width_sq < __fmul_rn(d2, theta2);
}

// ---- node centre of mass, reference FP32 formula (karras_bvh.cuh:213-216) --
// (c_l * m_l + c_r * m_r) / m as fma(c_l, m_l, c_r * m_r) / m.
__device__ __forceinline__ float com_fp32(float cl, float ml, float cr, float mr, float m) {
    return __fdiv_rn(__fmaf_rn(cl, ml, __fmul_rn(cr, mr)), m);
}

// ---- speed colour map (cuda_engine.cu:184-215) ------------------------------
__device__ __forceinline__ float speed_of(float vx, float vy, float vz) {
    return __fsqrt_rn(__fmaf_rn(vz, vz, __fmaf_rn(vy, vy, __fmul_rn(vx, vx))));
}

// Returns the new packed type|r|g|b word for a particle of type 0 or 2.
__device__ __forceinline__ uint32_t recolour(uint32_t tcol, float vx, float vy, float vz) {
    const uint32_t type = tcol & 0xFFu;
    if (type != 0u && type != 2u) return tcol;
    const float speed = speed_of(vx, vy, vz);
    const float t = fminf(__fdiv_rn(speed, 150.0f), 1.0f);
    uint32_t r, g, b;
    if (type == 0u) {  // fire: red -> orange -> yellow
        if (t < 0.5f) {
            const float nt = __fmul_rn(t, 2.0f);
            r = 255u;
            g = (uint32_t)(uint8_t)__float2uint_rz(__fmaf_rn(150.0f, nt, 50.0f));
            b = 0u;
        } else {
            const float nt = __fmul_rn(__fsub_rn(t, 0.5f), 2.0f);
            r = 255u;
            g = (uint32_t)(uint8_t)__float2uint_rz(__fmaf_rn(55.0f, nt, 200.0f));
            b = (uint32_t)(uint8_t)__float2uint_rz(__fmul_rn(150.0f, nt));
        }
    } else {  // ice: dark blue -> cyan -> white
        if (t < 0.5f) {
            const float nt = __fmul_rn(t, 2.0f);
            r = 0u;
            g = (uint32_t)(uint8_t)__float2uint_rz(__fmaf_rn(100.0f, nt, 100.0f));
            b = 255u;
        } else {
            const float nt = __fmul_rn(__fsub_rn(t, 0.5f), 2.0f);
            r = (uint32_t)(uint8_t)__float2uint_rz(__fmul_rn(200.0f, nt));
            g = (uint32_t)(uint8_t)__float2uint_rz(__fmaf_rn(55.0f, nt, 200.0f));
            b = 255u;
        }
    }
    return type | (r << 8) | (g << 16) | (b << 24);
}

// ---- kick/drift of one particle (cuda_engine.cu:164-216) --------------------
// v += a dt; x += v dt; recolour types 0/2 by speed.  The reference's two
// statements per axis contract to fma(a, dt, v) and fma(v, dt, x).  The
// separate integrate kernel and the walk's fused epilogue both call this, so
// their results are the same bits.
__device__ __forceinline__ void kick_drift(float4& p, float4& v, float4 a, float dt, int recolor) {
    v.x = __fmaf_rn(a.x, dt, v.x);
    v.y = __fmaf_rn(a.y, dt, v.y);
    v.z = __fmaf_rn(a.z, dt, v.z);
    p.x = __fmaf_rn(v.x, dt, p.x);
    p.y = __fmaf_rn(v.y, dt, p.y);
    p.z = __fmaf_rn(v.z, dt, p.z);
    if (recolor) v.w = __uint_as_float(recolour(__float_as_uint(v.w), v.x, v.y, v.z));
}

// ---- Star record (types.h:5-11) as two float4 ------------------------------
// Star (x,y,z,vx | vy,vz,m,tcol) from pos (x,y,z,m) and vel (vx,vy,vz,tcol).
__device__ __forceinline__ void store_star(float4* __restrict__ stars, int64_t i, float4 p, float4 v) {
    stars[2 * i] = make_float4(p.x, p.y, p.z, v.x);
    stars[2 * i + 1] = make_float4(v.y, v.z, p.w, v.w);
}

// ---- order-preserving float <-> u32 (for atomicMax-based min/max) ----------
__device__ __forceinline__ uint32_t float_to_ordered(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ordered_to_float(uint32_t o) {
    const uint32_t u = (o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o;
    return __uint_as_float(u);
}

}  // namespace gcs
