// Device helpers shared by the f64 and FP32 kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_types.h"

namespace tpt {

// ---- PCG32 stream of src/rng.rs:9-37 -------------------------------------
// LCG step with XSH-RR output; the state is the reference's u64 `state`.
__device__ __forceinline__ uint32_t pcg_next(uint64_t& s) {
    const uint64_t old = s;
    s = old * 6364136223846793005ull + 1442695040888963407ull;
    const uint32_t xs = (uint32_t)(((old >> 18) ^ old) >> 27);
    const uint32_t rot = (uint32_t)(old >> 59);
    return __funnelshift_r(xs, xs, rot);  // rotate right by rot
}
// next_f64 (src/rng.rs:30-36): 53 bits from two draws.
__device__ __forceinline__ double pcg_f64(uint64_t& s) {
    const uint64_t hi = (uint64_t)pcg_next(s) << 21;
    const uint64_t lo = (uint64_t)pcg_next(s) & ((1ull << 21) - 1);
    return (double)(hi | lo) * (1.0 / 9007199254740992.0);
}
// The same two draws as next_f64, kept to 24 bits: the FP32 kernels consume
// the reference stream draw for draw, with each value truncated to the
// float grid (|error| < 2^-24).
__device__ __forceinline__ float pcg_f32(uint64_t& s) {
    const uint32_t hi = pcg_next(s);
    (void)pcg_next(s);
    return (float)(hi >> 8) * (1.0f / 16777216.0f);
}
// Rng::new (src/rng.rs:12-15) over seed_for(x, y, s) ^ seed (src/render.rs:142,
// src/rng.rs:41-47); s is the task's first sample index.
__host__ __device__ __forceinline__ uint64_t task_seed(uint32_t px, uint32_t py, uint32_t s, uint64_t seed) {
    uint64_t h = 0xD1B54A32D192ED03ull;
    h ^= (uint64_t)px * 0x9E3779B185EBCA87ull;
    h ^= (uint64_t)py * 0xC2B2AE3D27D4EB4Full;
    h ^= (uint64_t)s * 0x165667B19E3779F9ull;
    h = h ^ (h >> 32);
    h ^= seed;
    return h == 0 ? 0x9E3779B97F4A7C15ull : h;
}
// Rng::new (src/rng.rs:12-15) over seed_for(x, y, 0) ^ seed (src/render.rs:142).
__host__ __device__ __forceinline__ uint64_t pixel_seed(uint32_t px, uint32_t py, uint64_t seed) {
    uint64_t h = 0xD1B54A32D192ED03ull;
    h ^= (uint64_t)px * 0x9E3779B185EBCA87ull;
    h ^= (uint64_t)py * 0xC2B2AE3D27D4EB4Full;
    h = h ^ (h >> 32);
    h ^= seed;
    return h == 0 ? 0x9E3779B97F4A7C15ull : h;
}

// ---- float3 helpers --------------------------------------------------------
__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return a * s; }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
// FP32 dot and cross products with their FMAs written out: the FP32 units
// are compiled without automatic contraction, so every kernel rounds them
// the same way.
__device__ __forceinline__ float dot(float3 a, float3 b) {
    return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, a.x * b.x));
}
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return f3(__fmaf_rn(a.y, b.z, -(a.z * b.y)), __fmaf_rn(a.z, b.x, -(a.x * b.z)), __fmaf_rn(a.x, b.y, -(a.y * b.x)));
}
__device__ __forceinline__ float length(float3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float3 normalize(float3 a) { return a * (1.0f / fmaxf(length(a), 1e-30f)); }
__device__ __forceinline__ float luminance(float3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
__device__ __forceinline__ float max3(float3 c) { return fmaxf(fmaxf(c.x, c.y), c.z); }

__device__ __forceinline__ int fbits(float f) { return __float_as_int(f); }
__device__ __forceinline__ float ifloat(int i) { return __int_as_float(i); }

// Device-side error flags (TPT_FLAG_* in tinypt_cuda.h).
__device__ __forceinline__ void raise_flag(int* flags, int bit) { atomicOr(flags, bit); }

}  // namespace tpt
