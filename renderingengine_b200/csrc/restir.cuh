// ReSTIR DI on the primary surface: the ABI-v3 records
// (include/contracts/RestirAbiV3.hpp:109-201) and the production reservoir
// arithmetic of resources/shaders/restir/RestirProductionV3.hlsli, in float
// with the shader's operand order.  Records stay in their ABI layout in HBM:
//   GpuPrimarySurfaceV2   96 B  (ReconstructionAbiV2.hpp:44-52)
//   GpuRestirReservoirV3 256 B  (RestirAbiV3.hpp:149-157)
#pragma once

#include "bsdf.cuh"
#include "lights.cuh"

namespace re {

// Primary-surface flags (ReconstructionAbiV2.hpp:15-22).
constexpr uint32_t kSurfValid = 1u, kSurfFrontFace = 2u, kSurfHasDiffuse = 4u, kSurfHasSpecular = 8u;
// RestirSampleFlags / RestirReservoirFlags / RestirHistoryFlags (RestirAbiV3.hpp:49-80).
constexpr uint32_t kRsSampleValid = 1u, kRsSampleDelta = 2u, kRsSampleArea = 4u, kRsSampleSolidAngle = 8u;
constexpr uint32_t kRsValid = 1u, kRsMClamped = 2u, kRsTemporalAccepted = 4u, kRsSpatialAccepted = 8u,
                   kRsReferenceMode = 16u, kRsFinalVisibility = 32u, kRsVisibilityValid = 64u;
constexpr uint32_t kRsHistoryValid = 1u, kRsHistoryReset = 2u;
// RestirRejectionReason (RestirAbiV3.hpp:82-98).
constexpr uint32_t kRejNone = 0u, kRejInvalidCandidate = 1u, kRejReprojectionOutside = 2u, kRejMotionInvalid = 3u,
                   kRejCameraCut = 4u, kRejResize = 5u, kRejDepth = 6u, kRejNormal = 7u, kRejInstance = 8u,
                   kRejThinGeometry = 9u, kRejSceneGeneration = 10u, kRejLightGeneration = 11u, kRejAge = 12u,
                   kRejMaterial = 13u;
// RestirCandidateSource / RestirReuseSource.
constexpr uint32_t kReuseNone = 0u, kReuseTemporal = 1u, kReuseSpatial = 2u;
constexpr uint32_t kRsInvalidIndex = 0xffffffffu;

struct PrimarySurface {
    float4 pos_depth;  // world position, linear depth
    float4 gn_rough;   // geometric normal, roughness
    float4 sn_metal;   // shading normal, metallic
    float4 dalb;       // diffuse albedo
    float4 salb;       // specular albedo
    uint4 identity;    // material, instance, primitive, flags
};

struct LightSampleV3 {  // GpuPersistentLightSampleV3
    float4 pos_dist;
    float4 dir_pdf;
    float4 rad_pmf;
    float4 cond;
    uint4 identity;
    uint4 generation;
    uint4 metadata;
    uint4 source;
};

struct Reservoir {  // GpuRestirReservoirV3
    LightSampleV3 sel;
    float4 weight;  // weightSum, W, selected target, selected proposal pdf
    float4 terms;   // support, correction, candidate weight, final weight
    uint4 state;    // M, age, flags, rejection
    uint4 prov;     // source, reuse source, source surface, candidate flags
    uint4 h_surface, h_scene, h_frame, h_reproj;
};
static_assert(sizeof(PrimarySurface) == 96, "GpuPrimarySurfaceV2");
static_assert(sizeof(LightSampleV3) == 128, "GpuPersistentLightSampleV3");
static_assert(sizeof(Reservoir) == 256, "GpuRestirReservoirV3");

struct Candidate {
    LightSampleV3 s;
    float4 t;  // target, proposal pdf, support, correction
    uint4 prov;
};

// Per-frame ReSTIR parameters (GpuRestirParametersV3, RestirAbiV3.hpp:184-195,
// plus the previous camera for the reprojection).
struct RestirParams {
    uint32_t enabled, candidates, neighbors, max_m;
    uint32_t max_age, history_enabled, neighbor_mode, parity;
    uint32_t scene_gen, light_gen, camera_gen, resolution_gen;
    uint32_t history_gen, frame_lo, frame_hi, prev_valid;
    uint32_t candidate_source, light_count, prev_light_count;
    uint32_t estimator;  // 0 biased, 1 reference correction (GpuRestirParametersV3 modeAndFlags.x)
    float normal_cos, rel_depth, position_dist, disk_radius;
    f3 prev_pos;
    float prev_tan;
    f3 prev_fwd;
    float prev_aspect;
    f3 prev_right;
    float pad1;
    f3 prev_up;
    float pad2;
};

__device__ __forceinline__ uint32_t restir_hash(uint32_t v) {  // RestirHashV3
    v ^= v >> 16u;
    v *= 0x7feb352du;
    v ^= v >> 15u;
    v *= 0x846ca68bu;
    v ^= v >> 16u;
    return v;
}
__device__ __forceinline__ float restir_random(uint32_t& s) {  // RestirRandomV3
    s = restir_hash(s + 0x9e3779b9u);
    return float(s >> 8u) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ bool fin4(float4 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && isfinite(v.w); }
__device__ __forceinline__ f3 xyz(float4 v) { return mk(v.x, v.y, v.z); }
__device__ __forceinline__ float saturate1(float v) { return fminf(fmaxf(v, 0.f), 1.f); }
__device__ __forceinline__ float length3(f3 v) { return sqrtf(dot(v, v)); }
__device__ __forceinline__ bool finite_nonneg1(float v) { return isfinite(v) && v >= 0.f; }

__device__ __forceinline__ PrimarySurface load_surface(const float4* base, uint32_t p) {
    const float4* q = base + size_t(p) * 6u;
    PrimarySurface s;
    s.pos_depth = q[0];
    s.gn_rough = q[1];
    s.sn_metal = q[2];
    s.dalb = q[3];
    s.salb = q[4];
    const float4 id = q[5];
    s.identity = make_uint4(__float_as_uint(id.x), __float_as_uint(id.y), __float_as_uint(id.z), __float_as_uint(id.w));
    return s;
}

// RestirSurfaceValidV3 (RestirProductionV3.hlsli:233-255).
__device__ __forceinline__ bool surface_valid(const PrimarySurface& s) {
    const f3 da = xyz(s.dalb), sa = xyz(s.salb), gn = xyz(s.gn_rough), sn = xyz(s.sn_metal);
    return (s.identity.w & kSurfValid) != 0u && fin4(s.pos_depth) && fin4(s.gn_rough) && fin4(s.sn_metal) &&
           fin4(s.dalb) && fin4(s.salb) && da.x >= 0.f && da.y >= 0.f && da.z >= 0.f && da.x <= 1.f &&
           da.y <= 1.f && da.z <= 1.f && sa.x >= 0.f && sa.y >= 0.f && sa.z >= 0.f && sa.x <= 1.f && sa.y <= 1.f &&
           sa.z <= 1.f && s.sn_metal.w >= 0.f && s.sn_metal.w <= 1.f && roughness_finite_model(s.gn_rough.w) &&
           dot(gn, gn) > 1.0e-12f && dot(sn, sn) > 1.0e-12f;
}

// RestirSampleValidV3 (RestirProductionV3.hlsli:257-267).
__device__ __forceinline__ bool sample_valid(const LightSampleV3& s, uint32_t scene_gen) {
    return (s.metadata.y & kRsSampleValid) != 0u && s.identity.x != kRsInvalidIndex && s.generation.x != 0u &&
           s.generation.y == scene_gen && finite_nonneg1(s.dir_pdf.w) && finite_nonneg1(s.rad_pmf.w) &&
           finite3(xyz(s.dir_pdf)) && finite3(xyz(s.rad_pmf));
}

__device__ __forceinline__ float luminance_pos(f3 v) {  // RestirLuminanceV3
    return fmaxf(v.x, 0.f) * 0.2126f + fmaxf(v.y, 0.f) * 0.7152f + fmaxf(v.z, 0.f) * 0.0722f;
}

// RestirEvaluateUnshadowedV3 (RestirProductionV3.hlsli:269-315): Lambert on
// the published diffuse albedo plus GGX with Schlick Fresnel on the
// published specular albedo.
__device__ __forceinline__ float evaluate_unshadowed(const LightSampleV3& s, const PrimarySurface& surf, f3 cam_pos,
                                                     uint32_t scene_gen, f3& diffuse, f3& specular) {
    diffuse = f3s(0.f);
    specular = f3s(0.f);
    if (!sample_valid(s, scene_gen) || !surface_valid(surf)) return 0.f;
    const f3 n = normalize3(xyz(surf.sn_metal));
    const f3 l = normalize3(xyz(s.dir_pdf));
    const f3 v = normalize3(cam_pos - xyz(surf.pos_depth));
    const float nol = saturate1(dot(n, l));
    const float nov = saturate1(dot(n, v));
    if (!(nol > 0.f) || !(nov > 0.f)) return 0.f;
    const f3 h = normalize3(l + v);
    const float noh = saturate1(dot(n, h));
    const float voh = saturate1(dot(v, h));
    const float roughness = surf.gn_rough.w;
    const f3 da = mk(fmaxf(surf.dalb.x, 0.f), fmaxf(surf.dalb.y, 0.f), fmaxf(surf.dalb.z, 0.f));
    const f3 f0 = mk(fmaxf(surf.salb.x, 0.f), fmaxf(surf.salb.y, 0.f), fmaxf(surf.salb.z, 0.f));
    const f3 f = fresnel_schlick(voh, f0);
    const float alpha = roughness * roughness;
    const float d = ggx_d(mk(0.f, 0.f, noh), alpha);
    const float g = ggx_g2(mk(sqrtf(fmaxf(0.f, 1.f - nov * nov)), 0.f, nov),
                           mk(sqrtf(fmaxf(0.f, 1.f - nol * nol)), 0.f, nol), alpha);
    const f3 rad = mk(fmaxf(s.rad_pmf.x, 0.f), fmaxf(s.rad_pmf.y, 0.f), fmaxf(s.rad_pmf.z, 0.f));
    diffuse = rad * da * (f3s(1.f) - f) * (nol * kInvPi);
    specular = rad * f * (d * g / fmaxf(4.f * nov, 1.0e-6f));
    if (!finite3(diffuse) || !finite3(specular)) {
        diffuse = f3s(0.f);
        specular = f3s(0.f);
        return 0.f;
    }
    return luminance_pos(diffuse + specular);
}

// RestirEvaluateCandidateV3 (RestirProductionV3.hlsli:317-340).
__device__ __forceinline__ Candidate evaluate_candidate(const LightSampleV3& s, const PrimarySurface& surf, f3 cam_pos,
                                                        uint32_t scene_gen, uint32_t cand_source, uint32_t reuse_source,
                                                        uint32_t source_surface) {
    Candidate c;
    c.s = s;
    f3 dif, spec;
    const float target = evaluate_unshadowed(s, surf, cam_pos, scene_gen, dif, spec);
    const float proposal = s.dir_pdf.w;
    const bool sv = surface_valid(surf);
    const float support = sample_valid(s, scene_gen) && sv && target > 0.f && proposal > 0.f ? 1.f : 0.f;
    c.t = make_float4(target, proposal, support, sv ? 1.f : 0.f);
    c.prov = make_uint4(cand_source, reuse_source, source_surface, s.metadata.y);
    return c;
}

// RestirCandidateValidV3 / RestirCandidateWeightV3 (:342-361).
__device__ __forceinline__ bool candidate_valid(const Candidate& c, uint32_t scene_gen) {
    const float4 t = c.t;
    const bool consistent = t.x > 0.f ? t.z == 1.f : t.z == 0.f;
    return sample_valid(c.s, scene_gen) && finite_nonneg1(t.x) && isfinite(t.y) && t.y > 0.f &&
           (t.z == 0.f || t.z == 1.f) && finite_nonneg1(t.w) && t.w > 0.f && consistent;
}
__device__ __forceinline__ float candidate_weight(const Candidate& c, uint32_t scene_gen) {
    if (!candidate_valid(c, scene_gen)) return 0.f;
    return c.t.x * c.t.z * c.t.w / c.t.y;
}

__device__ __forceinline__ Reservoir empty_reservoir() {
    Reservoir r;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const uint4 u = make_uint4(0u, 0u, 0u, 0u);
    r.sel.pos_dist = z; r.sel.dir_pdf = z; r.sel.rad_pmf = z; r.sel.cond = z;
    r.sel.identity = make_uint4(kRsInvalidIndex, kRsInvalidIndex, 0u, 0u);
    r.sel.generation = u; r.sel.metadata = u; r.sel.source = u;
    r.weight = z; r.terms = z; r.state = u; r.prov = u;
    r.h_surface = u; r.h_scene = u; r.h_frame = u; r.h_reproj = u;
    return r;
}

// RestirUpdateReservoirV3 (:372-405).
__device__ __forceinline__ void update_reservoir(Reservoir& r, const Candidate& c, float weight, uint32_t mult,
                                                 float u, uint32_t scene_gen) {
    if (!candidate_valid(c, scene_gen) || !isfinite(weight) || weight < 0.f || mult == 0u) return;
    const uint32_t old_m = r.state.x;
    const uint32_t new_m = old_m > 0xffffffffu - mult ? 0xffffffffu : old_m + mult;
    if (weight == 0.f) {
        r.state.x = new_m;
        return;
    }
    const float new_sum = r.weight.x + weight;
    if (!(new_sum > 0.f) || !isfinite(new_sum)) return;
    r.weight.x = new_sum;
    r.state.x = new_m;
    if (u * new_sum < weight) {
        r.sel = c.s;
        r.weight.z = c.t.x;
        r.weight.w = c.t.y;
        r.terms = make_float4(c.t.z, c.t.w, weight, 0.f);
        r.prov = c.prov;
    }
}

// update_reservoir split in two for loops that keep the selected
// candidate's index instead of a copy of it: fold_update applies a
// candidate's effect on the weight sum and M (the same checks, additions
// and saturation) and returns whether it is selected; select_candidate
// then writes the selected candidate's fields, as update_reservoir does
// when it selects.
__device__ __forceinline__ bool fold_update(float& wsum, uint32_t& m, bool valid, float weight, uint32_t mult,
                                            float u) {
    if (!valid || !isfinite(weight) || weight < 0.f || mult == 0u) return false;
    const uint32_t new_m = m > 0xffffffffu - mult ? 0xffffffffu : m + mult;
    if (weight == 0.f) {
        m = new_m;
        return false;
    }
    const float new_sum = wsum + weight;
    if (!(new_sum > 0.f) || !isfinite(new_sum)) return false;
    wsum = new_sum;
    m = new_m;
    return u * new_sum < weight;
}
__device__ __forceinline__ void select_candidate(Reservoir& r, const Candidate& c, float weight) {
    r.sel = c.s;
    r.weight.z = c.t.x;
    r.weight.w = c.t.y;
    r.terms = make_float4(c.t.z, c.t.w, weight, 0.f);
    r.prov = c.prov;
}

// RestirFinalizeReservoirV3 (:407-435).
__device__ __forceinline__ void finalize_reservoir(Reservoir& r) {
    if (r.state.x == 0u || !(r.weight.z > 0.f) || !(r.weight.x > 0.f) || !isfinite(r.weight.z) ||
        !isfinite(r.weight.x)) {
        r.state.z &= ~kRsValid;
        r.weight.y = 0.f;
        return;
    }
    const float den = float(r.state.x) * r.weight.z;
    if (!(den > 0.f) || !isfinite(den)) {
        r.state.z &= ~kRsValid;
        r.weight.y = 0.f;
        return;
    }
    r.weight.y = r.weight.x / den;
    if (!(r.weight.y > 0.f) || !isfinite(r.weight.y)) {
        r.state.z &= ~kRsValid;
        r.weight.y = 0.f;
        return;
    }
    r.terms.w = r.weight.y;
    r.state.z |= kRsValid;
}

// RestirClampMV3 (:437-447).
__device__ __forceinline__ void clamp_m(Reservoir& r, uint32_t max_m) {
    if (r.state.x > max_m) {
        const float scale = float(max_m) / float(r.state.x);
        r.weight.x *= scale;
        r.state.x = max_m;
        r.state.z |= kRsMClamped;
    }
}

// RestirValidateSurfacePairV3 (:449-481).
__device__ __forceinline__ uint32_t validate_surface_pair(const PrimarySurface& cur, const PrimarySurface& src,
                                                          const RestirParams& rp) {
    if (!surface_valid(cur) || !surface_valid(src)) return kRejInvalidCandidate;
    if (cur.identity.x != src.identity.x) return kRejMaterial;
    if (cur.identity.y != src.identity.y) return kRejInstance;
    const float scale = fmaxf(1.f, fmaxf(fabsf(cur.pos_depth.w), fabsf(src.pos_depth.w)));
    if (fabsf(cur.pos_depth.w - src.pos_depth.w) / scale > rp.rel_depth) return kRejDepth;
    if (dot(normalize3(xyz(cur.sn_metal)), normalize3(xyz(src.sn_metal))) < rp.normal_cos) return kRejNormal;
    if (length3(xyz(cur.pos_depth) - xyz(src.pos_depth)) > rp.position_dist) return kRejThinGeometry;
    return kRejNone;
}

// WfPublishPrimarySurfaceV2 / PbrPublishPrimarySurfaceV2
// (pbr_reconstruction_export_v2.hlsli:42-92), the ReSTIR copy: Valid only
// where ReSTIR owns the primary direct lighting.
__device__ __forceinline__ void write_primary_surface(float4* base, uint32_t p, f3 pos, float depth, f3 gn, f3 sn,
                                                      uint32_t material, uint32_t instance, uint32_t primitive,
                                                      uint32_t front, f3 base_color, float metallic, float roughness,
                                                      float transmission, f3 f0, bool restir_supported) {
    const float m = saturate1(metallic);
    const f3 bc = mk(fmaxf(base_color.x, 0.f), fmaxf(base_color.y, 0.f), fmaxf(base_color.z, 0.f));
    const f3 da = bc * (1.f - m) * (1.f - saturate1(transmission));
    const f3 sl = f0 + (base_color - f0) * m;
    const f3 sa = mk(fmaxf(sl.x, 0.f), fmaxf(sl.y, 0.f), fmaxf(sl.z, 0.f));
    uint32_t flags = restir_supported ? kSurfValid : 0u;
    if (da.x > 0.f || da.y > 0.f || da.z > 0.f) flags |= kSurfHasDiffuse;
    if (sa.x > 0.f || sa.y > 0.f || sa.z > 0.f) flags |= kSurfHasSpecular;
    if (front != 0u) flags |= kSurfFrontFace;
    float4* q = base + size_t(p) * 6u;
    q[0] = to4(pos, fmaxf(depth, 0.f));
    q[1] = to4(normalize3(gn), saturate1(roughness));
    q[2] = to4(normalize3(sn), m);
    q[3] = to4(da, 0.f);
    q[4] = to4(sa, 0.f);
    q[5] = make_float4(__uint_as_float(material), __uint_as_float(instance), __uint_as_float(primitive),
                       __uint_as_float(flags));
}

}  // namespace re
