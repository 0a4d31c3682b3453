// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// extern "C" shim over the reference's double-precision BSDF
// (integrators/megakernel/include/ReferenceBsdf.hpp, header only, compiled
// unmodified into oracle/_ref): EvaluateBsdfL6 (:922), PdfBsdfL6 (:980),
// SampleBsdfL6 (:1242) and SampleGgxVisibleNormalL6 (:492).  Queries use the
// 160-byte layout of re_bsdf_query (float inputs, widened to double); results
// are the fields of re_bsdf_probe_result as 32 doubles.
#include <cstdint>
#include <cstring>

#include "ReferenceBsdf.hpp"

namespace bsdf = RenderingEngine::Integrators::Megakernel::ReferenceBsdfL6;

namespace {

bsdf::Vec3 v3(const float* p) { return {double(p[0]), double(p[1]), double(p[2])}; }
uint32_t u32(const float* p) {
    uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}

void put(double* o, const bsdf::Vec3& v, double w) {
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = w;
}

}  // namespace

extern "C" {

void ref_bsdf_probe(const float* queries, uint32_t n, double* results) {
    for (uint32_t i = 0; i < n; ++i) {
        const float* q = queries + size_t(i) * 40u;
        bsdf::BsdfContextL6 c{};
        c.geometricNormal = v3(q + 0);
        c.etaIncident = q[3];
        c.shadingNormal = v3(q + 4);
        c.etaTransmitted = q[7];
        c.tangent = v3(q + 8);
        c.transportMode = u32(q + 11);
        bsdf::BsdfParamsL6 p{};
        p.baseColor = v3(q + 12);
        p.metallic = q[15];
        p.f0 = v3(q + 16);
        p.perceptualRoughness = q[19];
        p.conductorEta = v3(q + 20);
        p.transmission = q[23];
        p.conductorK = v3(q + 24);
        p.model = u32(q + 27);
        p.allowedLobes = u32(q + 31);
        p.useComplexConductorFresnel = u32(q + 35);
        const bsdf::Vec3 wo = v3(q + 28), wi = v3(q + 32), u = v3(q + 36);
        const bsdf::BsdfEvalL6 e = bsdf::EvaluateBsdfL6(c, p, wo, wi);
        const bsdf::BsdfSampleL6 s = bsdf::SampleBsdfL6(c, p, wo, u);
        double pdf_at = 0.0;
        if (s.isValid != 0u && s.isDelta == 0u) pdf_at = bsdf::PdfBsdfL6(c, p, wo, s.direction);
        double* o = results + size_t(i) * 32u;
        put(o + 0, e.value, e.pdf);
        put(o + 4, e.diffuseValue, double(e.measure));
        put(o + 8, e.specularValue, double(e.lobeFlags));
        put(o + 12, s.direction, s.pdf);
        put(o + 16, s.value, s.eta);
        put(o + 20, s.diffuseValue, double(s.measure));
        put(o + 24, s.specularValue, double(s.lobeFlags));
        o[28] = double(e.isValid);
        o[29] = double(s.isDelta);
        o[30] = double(s.isValid);
        o[31] = pdf_at;
    }
}

// SampleGgxVisibleNormalL6: visible microfacet normal for a local outgoing
// direction.  wo: 3 doubles per query; u: 2 doubles; out: 4 doubles
// (normal xyz, 1 when valid else 0).
void ref_ggx_vndf(const double* wo, const double* alpha, const double* u, uint32_t n, double* out) {
    for (uint32_t i = 0; i < n; ++i) {
        bsdf::Vec3 m{};
        const bool ok = bsdf::SampleGgxVisibleNormalL6({wo[i * 3], wo[i * 3 + 1], wo[i * 3 + 2]}, alpha[i],
                                                        u[i * 2], u[i * 2 + 1], m);
        out[i * 4 + 0] = m.x;
        out[i * 4 + 1] = m.y;
        out[i * 4 + 2] = m.z;
        out[i * 4 + 3] = ok ? 1.0 : 0.0;
    }
}

}  // extern "C"
