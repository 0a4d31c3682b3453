// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// extern "C" shim over the reference's CPU reservoir code, compiled from the
// unmodified reference sources by oracle/Makefile into oracle/_ref/:
//   - CandidateWeight / UpdateReservoir / ClampReservoirM / FinalizeReservoir
//                                  src/restir/Reservoir.cpp:56-173
//   - ValidateTemporalHistory / ValidateSpatialNeighbor
//                                  src/restir/RestirDi.cpp:181-293
#include <cstdint>

#include "restir/Reservoir.hpp"
#include "restir/RestirDi.hpp"

namespace rs = RenderingEngine::Restir;

extern "C" {

// Initial RIS over explicit candidate terms (target, proposal pdf, support,
// correction) with explicit random numbers, the reference's way (double
// weight sum).  Writes (weightSum, normalizationWeight) and M; returns the
// selected candidate or -1.
int ref_restir_ris(const float* terms, const float* u, uint32_t n, uint32_t max_m, double* out, uint32_t* out_m) {
    rs::Reservoir r{};
    for (uint32_t i = 0; i < n; ++i) {
        rs::Candidate c{};
        c.identity.source = rs::CandidateSource::EmissiveTriangle;
        c.identity.lightId = i;
        c.identity.primitiveId = i;
        c.directionToLight = {0.0f, 0.0f, 1.0f};
        c.distance = 1.0f;
        c.unshadowedContribution = {1.0f, 1.0f, 1.0f};
        c.target = terms[4 * i];
        c.proposalPdf = terms[4 * i + 1];
        c.support = terms[4 * i + 2];
        c.correction = terms[4 * i + 3];
        static_cast<void>(rs::UpdateReservoir(r, c, rs::CandidateWeight(c), 1u, u[i]));
    }
    rs::ClampReservoirM(r, max_m);
    rs::FinalizeReservoir(r);
    out[0] = r.weightSum;
    out[1] = r.normalizationWeight;
    *out_m = r.M;
    return (r.flags & rs::ReservoirFlagValid) != 0u ? static_cast<int>(r.selected.identity.lightId) : -1;
}

namespace {

// Surface from 7 floats (position, normal, linear depth) and 5 words
// (instance, primitive, material, scene generation, thin geometry).
rs::SurfaceRecord surface(const float* g, const uint32_t* w) {
    rs::SurfaceRecord s{};
    s.position = {g[0], g[1], g[2]};
    s.normal = {g[3], g[4], g[5]};
    s.linearDepth = g[6];
    s.instanceId = w[0];
    s.primitiveId = w[1];
    s.materialId = w[2];
    s.sceneGeneration = w[3];
    s.thinGeometry = w[4] != 0u;
    return s;
}

// A reservoir that IsReservoirValid accepts when `valid` is set (flag, M,
// normalization weight and a finite candidate), with the given age and the
// selected light's generation.
rs::Reservoir reservoir(uint32_t valid, uint32_t age, uint32_t light_generation) {
    rs::Reservoir r{};
    r.selected.identity.source = rs::CandidateSource::EmissiveTriangle;
    r.selected.identity.lightId = 0u;
    r.selected.identity.generation = light_generation;
    r.selected.directionToLight = {0.0f, 0.0f, 1.0f};
    r.selected.distance = 1.0f;
    r.selected.unshadowedContribution = {1.0f, 1.0f, 1.0f};
    r.selected.target = 1.0f;
    r.selected.proposalPdf = 1.0f;
    r.selected.support = 1.0f;
    r.M = valid ? 1u : 0u;
    r.age = age;
    r.normalizationWeight = valid ? 1.0f : 0.0f;
    r.flags = valid ? rs::ReservoirFlagValid : rs::ReservoirFlagNone;
    return r;
}

rs::ReuseConfig config(const float* thresholds, uint32_t max_age) {
    rs::ReuseConfig c{};
    c.normalCosThreshold = thresholds[0];
    c.relativeDepthThreshold = thresholds[1];
    c.positionDistanceThreshold = thresholds[2];
    c.maxHistoryAge = max_age;
    return c;
}

}  // namespace

// ValidateSpatialNeighbor per case: geo = 14 floats (centre then neighbour
// surface), ids = 14 words (centre surface 5, neighbour surface 5, neighbour
// reservoir valid, age, selected light generation, light exists flag), the
// neighbour's current light generation in gen[i].  Writes the reason bitmask.
void ref_restir_validate_spatial(const float* geo, const uint32_t* ids, const uint32_t* gen, uint32_t n,
                                 const float* thresholds, uint32_t max_age, uint32_t* out) {
    const rs::ReuseConfig cfg = config(thresholds, max_age);
    for (uint32_t i = 0; i < n; ++i) {
        const float* g = geo + 14 * i;
        const uint32_t* w = ids + 14 * i;
        rs::SpatialNeighbor nb{};
        nb.surface = surface(g + 7, w + 5);
        nb.reservoir = reservoir(w[10], w[11], w[12]);
        nb.selectedLightExists = w[13] != 0u;
        nb.currentLightGeneration = gen[i];
        out[i] = static_cast<uint32_t>(rs::ValidateSpatialNeighbor(surface(g, w), nb, cfg));
    }
}

// ValidateTemporalHistory per case: geo / ids as above (current, then history
// surface and history reservoir), flags[i] = reprojectedInside | motionValid
// << 1 | cameraCut << 2 | resized << 3, gen[i] = current light generation.
void ref_restir_validate_temporal(const float* geo, const uint32_t* ids, const uint32_t* flags, const uint32_t* gen,
                                  uint32_t n, const float* thresholds, uint32_t max_age, uint32_t* out) {
    const rs::ReuseConfig cfg = config(thresholds, max_age);
    for (uint32_t i = 0; i < n; ++i) {
        const float* g = geo + 14 * i;
        const uint32_t* w = ids + 14 * i;
        rs::TemporalValidationInput in{};
        in.currentSurface = surface(g, w);
        in.historySurface = surface(g + 7, w + 5);
        in.reprojectedInside = (flags[i] & 1u) != 0u;
        in.motionValid = (flags[i] & 2u) != 0u;
        in.cameraCut = (flags[i] & 4u) != 0u;
        in.resized = (flags[i] & 8u) != 0u;
        in.selectedLightExists = w[13] != 0u;
        in.currentLightGeneration = gen[i];
        out[i] = static_cast<uint32_t>(rs::ValidateTemporalHistory(reservoir(w[10], w[11], w[12]), in, cfg));
    }
}

}  // extern "C"
