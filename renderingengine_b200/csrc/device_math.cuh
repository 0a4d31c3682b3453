// Small float3 toolkit and the counter-based RNG used by every kernel.
//
// Arithmetic that must be bit-reproducible against the CPU oracle is written
// with explicit round-to-nearest intrinsics (__fmul_rn / __fadd_rn /
// __fsub_rn), which the compiler never contracts into FMAs.  The library is
// additionally built with --fmad=false, so plain expressions follow the same
// IEEE single-precision sequence as the oracle compiled with
// -ffp-contract=off.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace re {

struct f3 {
    float x, y, z;
};

__host__ __device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__host__ __device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ __forceinline__ f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__host__ __device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ f3 operator*(float s, f3 a) { return {s * a.x, s * a.y, s * a.z}; }
__host__ __device__ __forceinline__ f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__host__ __device__ __forceinline__ f3 operator/(f3 a, f3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
__host__ __device__ __forceinline__ f3& operator+=(f3& a, f3 b) { a = a + b; return a; }
__host__ __device__ __forceinline__ f3& operator*=(f3& a, f3 b) { a = a * b; return a; }
__host__ __device__ __forceinline__ f3& operator*=(f3& a, float s) { a = a * s; return a; }
__host__ __device__ __forceinline__ f3& operator/=(f3& a, float s) { a = a / s; return a; }
// Left-to-right dot: ((a.x*b.x + a.y*b.y) + a.z*b.z).
__host__ __device__ __forceinline__ float dot(f3 a, f3 b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }
__host__ __device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return {(a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x)};
}
__host__ __device__ __forceinline__ f3 f3s(float s) { return {s, s, s}; }
__device__ __forceinline__ f3 from4(float4 v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ float4 to4(f3 v, float w) { return make_float4(v.x, v.y, v.z, w); }
__device__ __forceinline__ bool finite1(float v) { return isfinite(v); }
__device__ __forceinline__ bool finite3(f3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }
__device__ __forceinline__ bool finite_nonneg3(f3 v) {
    return finite3(v) && v.x >= 0.0f && v.y >= 0.0f && v.z >= 0.0f;
}
__device__ __forceinline__ bool any_negative(f3 v) { return v.x < 0.0f || v.y < 0.0f || v.z < 0.0f; }
__device__ __forceinline__ float maxc(f3 v) { return fmaxf(v.x, fmaxf(v.y, v.z)); }
__device__ __forceinline__ f3 fabs3(f3 v) { return {fabsf(v.x), fabsf(v.y), fabsf(v.z)}; }
__device__ __forceinline__ f3 normalize3(f3 v) {
    // HLSL normalize(v) = v * rsqrt(dot(v, v)); computed with an IEEE sqrt and
    // division so host and device agree.
    const float len = sqrtf(dot(v, v));
    return v / len;
}
__device__ __forceinline__ float luminance(f3 v) { return dot(v, mk(0.2126f, 0.7152f, 0.0722f)); }

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11).  Counter = (pixel, sample, dimension, stream tag), key
// = (seed low, seed high); the first output word's top 24 bits map to
// [0, 1).  Same mapping as PbrCounterRandomL6 (pbr_l6_types.hlsli:352-420)
// and CounterRandomFloat (MegakernelBridge.cpp:552-589).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t philox_x(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                             uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xd2511f53u, c0);
        const uint32_t lo0 = 0xd2511f53u * c0;
        const uint32_t hi1 = __umulhi(0xcd9e8d57u, c2);
        const uint32_t lo1 = 0xcd9e8d57u * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9e3779b9u;
        k1 += 0xbb67ae85u;
    }
    return c0;
}

__device__ __forceinline__ float counter_random(uint32_t pixel, uint32_t sample, uint32_t dim,
                                                uint32_t stream, uint32_t seed_lo, uint32_t seed_hi) {
    const uint32_t bits = philox_x(pixel, sample, dim, stream, seed_lo, seed_hi);
    return float(bits >> 8) * (1.0f / 16777216.0f);
}

// RNG dimension map (WavefrontRngDimensions.hpp:7-37).
constexpr uint32_t kDimCameraJitterX = 0;
constexpr uint32_t kDimCameraJitterY = 1;
constexpr uint32_t kDimCameraCount = 4;
constexpr uint32_t kDimPerBounce = 16;
constexpr uint32_t kDimLightSelection = 0;
constexpr uint32_t kDimLightShape0 = 1;
constexpr uint32_t kDimLightShape1 = 2;
constexpr uint32_t kDimLightShape2 = 3;
constexpr uint32_t kDimLightShape3 = 4;
constexpr uint32_t kDimBsdfLobe = 5;
constexpr uint32_t kDimBsdfU = 6;
constexpr uint32_t kDimBsdfV = 7;
constexpr uint32_t kDimRussianRoulette = 9;

__host__ __device__ __forceinline__ uint32_t bounce_dim(uint32_t bounce, uint32_t local) {
    return kDimCameraCount + bounce * kDimPerBounce + local;
}

}  // namespace re
