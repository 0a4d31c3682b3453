// TEST INFRASTRUCTURE ONLY -- shared declarations of the CPU oracle.
#pragma once

#include <cmath>
#include <cstdint>

namespace oracle {

struct V3 {
    float x, y, z;
};
inline V3 v3(float x, float y, float z) { return {x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float dot(V3 a, V3 b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }
inline V3 cross(V3 a, V3 b) { return {(a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x)}; }
inline bool finite3(V3 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }
inline bool nonneg3(V3 v) { return v.x >= 0.f && v.y >= 0.f && v.z >= 0.f; }
inline bool any_neg(V3 v) { return v.x < 0.f || v.y < 0.f || v.z < 0.f; }
inline float maxc(V3 v) { return std::fmax(v.x, std::fmax(v.y, v.z)); }
inline V3 normalize(V3 v) { return v / std::sqrt(dot(v, v)); }
inline V3 splat(float s) { return {s, s, s}; }

// Alpha-mask data (the layout the device reads): per leaf-ordered triangle
// 8 floats (tc0.xy, tc1.xy, tc2.xy, material bits, 0); per material 4 floats
// (alpha factor, cutoff, layer bits, sampler bits); atlas layers x h x w.
struct AlphaData {
    const float* tc;
    const float* materials;
    const float* atlas;
    uint32_t material_count, width, height, layers, sampler_id;
};

// Flattened-SAH closest / any-hit traversal (oracle_trace.cpp).
struct TraceResult {
    uint32_t tri;
    float t, u, v;
    uint32_t front, status;
    uint64_t node_tests, tri_tests;
};
TraceResult trace_flat(const void* nodes, uint32_t node_count, const float* tri_v, const uint32_t* tri_key,
                       V3 o, float tmin, V3 d, float tmax, bool any, bool shadow, uint32_t ign_inst,
                       uint32_t ign_prim, const AlphaData* alpha = nullptr);

}  // namespace oracle
