// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// extern "C" shim over the reference's CPU reservoir code, compiled from the
// unmodified reference sources by oracle/Makefile into oracle/_ref/:
//   - CandidateWeight / UpdateReservoir / ClampReservoirM / FinalizeReservoir
//                                  src/restir/Reservoir.cpp:56-173
#include <cstdint>

#include "restir/Reservoir.hpp"

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

}  // extern "C"
