// PBR BSDF evaluation and sampling on the device: Lambert, GGX conductor,
// GGX dielectric reflection, smooth glass, rough dielectric and the glTF
// metallic-roughness mixture, with Heitz visible-normal sampling, exact
// dielectric / conductor Fresnel, Smith height-correlated masking and the
// shading-normal correction.  Semantics follow
// resources/shaders/include/bsdf/PbrBsdf.hlsli:82-1679 (FP64 twin:
// integrators/megakernel/include/ReferenceBsdf.hpp).
#pragma once

#include "device_math.cuh"

namespace re {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTwoPi = 6.28318530717958647692f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kDirEps = 1.0e-7f;
constexpr float kMinAlpha = 1.0e-4f;

constexpr uint32_t kLobeDiffuse = 1u, kLobeGlossy = 2u, kLobeSpecular = 4u, kLobeReflection = 8u,
                   kLobeTransmission = 16u;
constexpr uint32_t kLobeDiffuseReflection = kLobeDiffuse | kLobeReflection;
constexpr uint32_t kLobeGlossyReflection = kLobeGlossy | kLobeReflection;
constexpr uint32_t kLobeGlossyTransmission = kLobeGlossy | kLobeTransmission;
constexpr uint32_t kLobeSpecularReflection = kLobeSpecular | kLobeReflection;
constexpr uint32_t kLobeSpecularTransmission = kLobeSpecular | kLobeTransmission;

constexpr uint32_t kModelLambert = 0, kModelGgxConductor = 1, kModelGgxDielectricReflection = 2,
                   kModelSmoothGlass = 3, kModelRoughDielectric = 4, kModelMetallicRoughness = 5;
constexpr uint32_t kMeasureInvalid = 0, kMeasureSolidAngle = 1, kMeasureDiscrete = 2;

struct BsdfContext {
    f3 ng;
    float eta_i;
    f3 ns;
    float eta_t;
    f3 tangent;
    uint32_t transport;  // 0 radiance, 1 importance
};

struct BsdfParams {
    f3 base_color;
    float metallic;
    f3 f0;
    float roughness;
    f3 cond_eta;
    float transmission;
    f3 cond_k;
    uint32_t model;
    uint32_t lobes;
    uint32_t complex_fresnel;
};

struct BsdfEval {
    f3 value;
    float pdf;
    f3 diffuse;
    f3 specular;
    uint32_t measure;
    uint32_t lobe;
    bool valid;
};

struct BsdfSample {
    f3 dir;
    float pdf;
    f3 value;
    float eta;
    f3 diffuse;
    f3 specular;
    uint32_t measure;
    uint32_t lobe;
    bool delta;
    bool valid;
};

__device__ __forceinline__ BsdfEval bsdf_eval_invalid() {
    BsdfEval r;
    r.value = f3s(0.f); r.pdf = 0.f; r.diffuse = f3s(0.f); r.specular = f3s(0.f);
    r.measure = kMeasureInvalid; r.lobe = 0; r.valid = false;
    return r;
}

__device__ __forceinline__ BsdfSample bsdf_sample_invalid() {
    BsdfSample r;
    r.dir = f3s(0.f); r.pdf = 0.f; r.value = f3s(0.f); r.eta = 1.f; r.diffuse = f3s(0.f); r.specular = f3s(0.f);
    r.measure = kMeasureInvalid; r.lobe = 0; r.delta = false; r.valid = false;
    return r;
}

__device__ __forceinline__ bool has_flags(uint32_t mask, uint32_t req) { return (mask & req) == req; }

__device__ __forceinline__ bool safe_normalize(f3 v, f3& out) {
    out = f3s(0.f);
    const float l2 = dot(v, v);
    if (!isfinite(l2) || l2 <= kDirEps * kDirEps) return false;
    out = v / sqrtf(l2);
    return finite3(out);
}

__device__ __forceinline__ bool unit_color(f3 v) {
    return finite3(v) && v.x >= 0.f && v.y >= 0.f && v.z >= 0.f && v.x <= 1.f && v.y <= 1.f && v.z <= 1.f;
}

__device__ __forceinline__ bool positive_eta(const BsdfContext& c) {
    return isfinite(c.eta_i) && isfinite(c.eta_t) && c.eta_i > 0.f && c.eta_t > 0.f;
}

__device__ __forceinline__ bool roughness_finite_model(float r) {
    if (!isfinite(r) || r <= 0.f || r > 1.f) return false;
    return r * r >= kMinAlpha;
}

// ValidateBsdfParamsL6 (PbrBsdf.hlsli:239-352), general branch.
__device__ __forceinline__ bool validate_params(const BsdfContext& c, const BsdfParams& p) {
    if (p.lobes == 0u || c.transport > 1u) return false;
    const bool trans_ok = isfinite(p.transmission) && p.transmission >= 0.f && p.transmission <= 1.f;
    switch (p.model) {
        case kModelLambert:
            return unit_color(p.base_color);
        case kModelGgxConductor:
            if (!roughness_finite_model(p.roughness)) return false;
            if (p.complex_fresnel != 0u)
                return finite3(p.cond_eta) && finite3(p.cond_k) && p.cond_eta.x > 0.f && p.cond_eta.y > 0.f &&
                       p.cond_eta.z > 0.f && p.cond_k.x >= 0.f && p.cond_k.y >= 0.f && p.cond_k.z >= 0.f;
            return unit_color(p.f0);
        case kModelGgxDielectricReflection:
            return roughness_finite_model(p.roughness) && positive_eta(c);
        case kModelSmoothGlass:
            return positive_eta(c) && trans_ok;
        case kModelRoughDielectric:
            return roughness_finite_model(p.roughness) && positive_eta(c) && trans_ok;
        case kModelMetallicRoughness:
            return unit_color(p.base_color) && unit_color(p.f0) && roughness_finite_model(p.roughness) &&
                   isfinite(p.metallic) && p.metallic >= 0.f && p.metallic <= 1.f && trans_ok;
        default:
            return false;
    }
}

// BsdfSupportsRestirPrimaryDirectL6 (PbrBsdf.hlsli:354-367).
__device__ __forceinline__ bool supports_restir_primary(const BsdfParams& p) {
    const uint32_t required = kLobeDiffuseReflection | kLobeGlossyReflection;
    const uint32_t unsupported = kLobeTransmission | kLobeSpecular;
    return p.model == kModelMetallicRoughness && p.complex_fresnel == 0u && roughness_finite_model(p.roughness) &&
           isfinite(p.transmission) && p.transmission == 0.f && (p.lobes & required) == required &&
           (p.lobes & unsupported) == 0u;
}

struct Frame {
    f3 ng, ns, t, b, wo, wo_local;
};

// BsdfBuildFrameL6 (PbrBsdf.hlsli:369-432).
__device__ __forceinline__ bool build_frame(const BsdfContext& c, f3 wo_in, Frame& f) {
    if (!safe_normalize(c.ng, f.ng) || !safe_normalize(c.ns, f.ns) || !safe_normalize(wo_in, f.wo)) return false;
    if (dot(f.ns, f.ng) < 0.f) f.ns = -f.ns;
    if (dot(f.wo, f.ng) < 0.f) {
        f.ng = -f.ng;
        f.ns = -f.ns;
    }
    if (dot(f.wo, f.ng) <= kDirEps || dot(f.wo, f.ns) <= kDirEps) return false;
    const f3 tc = c.tangent - f.ns * dot(c.tangent, f.ns);
    if (!safe_normalize(tc, f.t)) {
        const f3 helper = fabsf(f.ns.z) < 0.999f ? mk(0.f, 0.f, 1.f) : mk(0.f, 1.f, 0.f);
        if (!safe_normalize(cross(helper, f.ns), f.t)) return false;
    }
    if (!safe_normalize(cross(f.ns, f.t), f.b)) return false;
    f.wo_local = mk(dot(f.wo, f.t), dot(f.wo, f.b), dot(f.wo, f.ns));
    return finite3(f.wo_local) && f.wo_local.z > kDirEps;
}

__device__ __forceinline__ f3 to_local(f3 d, const Frame& f) { return mk(dot(d, f.t), dot(d, f.b), dot(d, f.ns)); }
__device__ __forceinline__ f3 to_world(f3 d, const Frame& f) { return f.t * d.x + f.b * d.y + f.ns * d.z; }

__device__ __forceinline__ bool validate_world_event(f3 wo, f3 wi, f3 ng, uint32_t lobe) {
    const float side = dot(wo, ng) * dot(wi, ng);
    const bool refl = has_flags(lobe, kLobeReflection);
    const bool trans = has_flags(lobe, kLobeTransmission);
    if (refl == trans) return false;
    return refl ? side > 0.f : side < 0.f;
}

__device__ __forceinline__ bool shading_correction(const BsdfContext& c, const Frame& f, f3 wi, float& corr) {
    corr = 0.f;
    const float num = c.transport == 0u ? fabsf(dot(wi, f.ns)) : fabsf(dot(f.wo, f.ns));
    const float den = c.transport == 0u ? fabsf(dot(wi, f.ng)) : fabsf(dot(f.wo, f.ng));
    if (!isfinite(num) || !isfinite(den) || den <= kDirEps) return false;
    corr = num / den;
    return isfinite(corr) && corr >= 0.f;
}

// BsdfFresnelDielectricL6 (PbrBsdf.hlsli:498-541).
__device__ __forceinline__ bool fresnel_dielectric(float cos_in, float eta_i, float eta_t, float& fr) {
    fr = 0.f;
    if (!isfinite(cos_in) || !isfinite(eta_i) || !isfinite(eta_t) || eta_i <= 0.f || eta_t <= 0.f) return false;
    const float ci = fminf(fabsf(cos_in), 1.f);
    const float ratio = eta_i / eta_t;
    const float st2 = ratio * ratio * fmaxf(0.f, 1.f - ci * ci);
    if (st2 >= 1.f) {
        fr = 1.f;
        return true;
    }
    const float ct = sqrtf(fmaxf(0.f, 1.f - st2));
    const float par_den = eta_t * ci + eta_i * ct;
    const float per_den = eta_i * ci + eta_t * ct;
    if (fabsf(par_den) <= kDirEps || fabsf(per_den) <= kDirEps) return false;
    const float par = (eta_t * ci - eta_i * ct) / par_den;
    const float per = (eta_i * ci - eta_t * ct) / per_den;
    fr = 0.5f * (par * par + per * per);
    return isfinite(fr) && fr >= 0.f && fr <= 1.f;
}

__device__ __forceinline__ f3 fresnel_schlick(float cosine, f3 f0) {
    const float m = 1.f - fminf(fabsf(cosine), 1.f);
    const float k = m * m * m * m * m;
    return f0 + (f3s(1.f) - f0) * k;
}

// BsdfFresnelConductorL6 (PbrBsdf.hlsli:551-592), per channel.
__device__ __forceinline__ bool fresnel_conductor1(float ci, float eta, float k, float& out) {
    const float c2 = ci * ci;
    const float s2 = fmaxf(0.f, 1.f - c2);
    const float e2 = eta * eta, k2 = k * k;
    const float t0 = e2 - k2 - s2;
    const float a2b2 = sqrtf(fmaxf(t0 * t0 + 4.f * e2 * k2, 0.f));
    const float t1 = a2b2 + c2;
    const float a = sqrtf(fmaxf(0.5f * (a2b2 + t0), 0.f));
    const float t2 = 2.f * ci * a;
    const float rs_den = t1 + t2;
    const float t3 = c2 * a2b2 + s2 * s2;
    const float t4 = t2 * s2;
    const float rp_den = t3 + t4;
    if (fabsf(rs_den) <= kDirEps || fabsf(rp_den) <= kDirEps) return false;
    const float rs = (t1 - t2) / rs_den;
    const float rp = rs * (t3 - t4) / rp_den;
    out = 0.5f * (rs + rp);
    return true;
}

__device__ __forceinline__ bool fresnel_conductor(float cos_in, f3 eta, f3 k, f3& fr) {
    fr = f3s(0.f);
    if (!isfinite(cos_in) || !finite3(eta) || !finite3(k) || eta.x <= 0.f || eta.y <= 0.f || eta.z <= 0.f ||
        k.x < 0.f || k.y < 0.f || k.z < 0.f)
        return false;
    const float ci = fminf(fabsf(cos_in), 1.f);
    if (!fresnel_conductor1(ci, eta.x, k.x, fr.x) || !fresnel_conductor1(ci, eta.y, k.y, fr.y) ||
        !fresnel_conductor1(ci, eta.z, k.z, fr.z))
        return false;
    return finite3(fr) && fr.x >= 0.f && fr.y >= 0.f && fr.z >= 0.f && fr.x <= 1.f && fr.y <= 1.f && fr.z <= 1.f;
}

__device__ __forceinline__ float ggx_d(f3 m, float alpha) {
    if (m.z <= 0.f || alpha < kMinAlpha) return 0.f;
    const float a2 = alpha * alpha;
    const float c2 = m.z * m.z;
    const float den = c2 * (a2 - 1.f) + 1.f;
    if (den <= 0.f) return 0.f;
    return a2 / (kPi * den * den);
}

__device__ __forceinline__ float ggx_lambda(f3 w, float alpha) {
    const float ac = fabsf(w.z);
    if (ac <= kDirEps) return 1.0e30f;
    const float s2 = fmaxf(0.f, 1.f - ac * ac);
    const float t2 = s2 / (ac * ac);
    return 0.5f * (sqrtf(1.f + alpha * alpha * t2) - 1.f);
}

__device__ __forceinline__ float ggx_g1(f3 w, float alpha) { return 1.f / (1.f + ggx_lambda(w, alpha)); }
__device__ __forceinline__ float ggx_g2(f3 wo, f3 wi, float alpha) {
    return 1.f / (1.f + ggx_lambda(wo, alpha) + ggx_lambda(wi, alpha));
}

__device__ __forceinline__ float ggx_vndf_pdf(f3 wo, f3 m, float alpha) {
    if (wo.z <= kDirEps || m.z <= 0.f || dot(wo, m) <= 0.f) return 0.f;
    return ggx_d(m, alpha) * ggx_g1(wo, alpha) * fabsf(dot(wo, m)) / fabsf(wo.z);
}

// Heitz visible-normal sampling (BsdfSampleGgxVisibleNormalL6, :646-708).
__device__ __forceinline__ bool ggx_sample_vndf(f3 wo, float alpha, float u1, float u2, f3& m) {
    m = f3s(0.f);
    if (wo.z <= kDirEps || alpha < kMinAlpha || !finite3(wo) || !isfinite(u1) || !isfinite(u2) || u1 < 0.f ||
        u2 < 0.f || u1 >= 1.f || u2 >= 1.f)
        return false;
    f3 v;
    if (!safe_normalize(mk(alpha * wo.x, alpha * wo.y, wo.z), v)) return false;
    if (v.z < 0.f) v = -v;
    f3 t1;
    const float lens2 = v.x * v.x + v.y * v.y;
    if (lens2 > kDirEps * kDirEps) {
        t1 = mk(-v.y, v.x, 0.f) / sqrtf(lens2);
    } else {
        t1 = mk(1.f, 0.f, 0.f);
    }
    const f3 t2 = cross(v, t1);
    const float r = sqrtf(u1);
    const float phi = 2.f * kPi * u2;
    const float dx = r * cosf(phi);
    float dy = r * sinf(phi);
    const float blend = 0.5f * (1.f + v.z);
    const float base = sqrtf(fmaxf(0.f, 1.f - dx * dx));
    dy = base + (dy - base) * blend;  // lerp(base, dy, blend)
    const float pz = sqrtf(fmaxf(0.f, 1.f - dx * dx - dy * dy));
    const f3 h = t1 * dx + t2 * dy + v * pz;
    if (!safe_normalize(mk(alpha * h.x, alpha * h.y, h.z), m)) return false;
    return m.z > 0.f && dot(wo, m) > 0.f;
}

__device__ __forceinline__ bool ggx_reflection_terms(f3 wo, f3 wi, float alpha, f3& m, float& d, float& g,
                                                     float& pdf) {
    m = f3s(0.f); d = 0.f; g = 0.f; pdf = 0.f;
    if (wo.z <= kDirEps || wi.z <= kDirEps || !safe_normalize(wo + wi, m)) return false;
    if (m.z < 0.f) m = -m;
    const float wom = fabsf(dot(wo, m));
    if (wom <= kDirEps) return false;
    d = ggx_d(m, alpha);
    g = ggx_g2(wo, wi, alpha);
    pdf = ggx_vndf_pdf(wo, m, alpha) / (4.f * wom);
    return d > 0.f && g >= 0.f && pdf > 0.f && isfinite(pdf);
}

__device__ __forceinline__ bool reflection_fresnel(const BsdfContext& c, const BsdfParams& p, float cosine, f3& fr) {
    fr = f3s(0.f);
    if (p.model == kModelGgxConductor) {
        if (p.complex_fresnel != 0u) return fresnel_conductor(cosine, p.cond_eta, p.cond_k, fr);
        fr = fresnel_schlick(cosine, p.f0);
        return finite3(fr);
    }
    if (p.model == kModelGgxDielectricReflection) {
        float s;
        if (!fresnel_dielectric(cosine, c.eta_i, c.eta_t, s)) return false;
        fr = f3s(s);
        return true;
    }
    fr = fresnel_schlick(cosine, p.f0);
    return finite3(fr);
}

__device__ __forceinline__ BsdfEval eval_lambert(const BsdfParams& p, f3 wo, f3 wi) {
    BsdfEval r = bsdf_eval_invalid();
    if (!has_flags(p.lobes, kLobeDiffuseReflection) || wo.z <= kDirEps || wi.z <= kDirEps) return r;
    r.diffuse = p.base_color * kInvPi;
    r.value = r.diffuse;
    r.pdf = wi.z * kInvPi;
    r.measure = kMeasureSolidAngle;
    r.lobe = kLobeDiffuseReflection;
    r.valid = finite3(r.value) && isfinite(r.pdf) && r.pdf > 0.f;
    return r.valid ? r : bsdf_eval_invalid();
}

__device__ __forceinline__ BsdfEval eval_ggx_reflection(const BsdfContext& c, const BsdfParams& p, f3 wo, f3 wi) {
    BsdfEval r = bsdf_eval_invalid();
    if (!has_flags(p.lobes, kLobeGlossyReflection)) return r;
    const float alpha = p.roughness * p.roughness;
    f3 m;
    float d, g, pdf;
    if (!ggx_reflection_terms(wo, wi, alpha, m, d, g, pdf)) return r;
    f3 fr;
    if (!reflection_fresnel(c, p, fabsf(dot(wo, m)), fr)) return r;
    const float den = 4.f * fabsf(wo.z * wi.z);
    if (den <= kDirEps) return r;
    r.specular = fr * (d * g / den);
    r.value = r.specular;
    r.pdf = pdf;
    r.measure = kMeasureSolidAngle;
    r.lobe = kLobeGlossyReflection;
    r.valid = finite3(r.value) && isfinite(r.pdf) && r.pdf > 0.f;
    return r.valid ? r : bsdf_eval_invalid();
}

__device__ __forceinline__ bool metallic_lobe_probabilities(const BsdfParams& p, f3 wo, float& pd, float& ps) {
    pd = 0.f;
    ps = 0.f;
    const bool allow_d = has_flags(p.lobes, kLobeDiffuseReflection);
    const bool allow_s = has_flags(p.lobes, kLobeGlossyReflection);
    const float dscale = (1.f - p.metallic) * (1.f - p.transmission);
    const float dw = allow_d ? luminance(p.base_color) * dscale : 0.f;
    const float sw = allow_s ? luminance(fresnel_schlick(fabsf(wo.z), p.f0)) : 0.f;
    const float tw = dw + sw;
    if (!isfinite(tw) || tw <= 0.f) return false;
    pd = dw / tw;
    ps = sw / tw;
    return isfinite(pd) && isfinite(ps);
}

__device__ __forceinline__ BsdfEval eval_metallic_roughness(const BsdfParams& p, f3 wo, f3 wi) {
    BsdfEval r = bsdf_eval_invalid();
    if (wo.z <= kDirEps || wi.z <= kDirEps) return r;
    float pd, ps;
    if (!metallic_lobe_probabilities(p, wo, pd, ps)) return r;
    const float alpha = p.roughness * p.roughness;
    f3 m;
    float d, g, spdf;
    const bool ok_spec = ggx_reflection_terms(wo, wi, alpha, m, d, g, spdf);
    if (ps > 0.f && !ok_spec) return r;
    const f3 fr = ok_spec ? fresnel_schlick(fabsf(dot(wo, m)), p.f0) : f3s(0.f);
    const float dscale = (1.f - p.metallic) * (1.f - p.transmission);
    if (pd > 0.f) {
        r.diffuse = (f3s(1.f) - fr) * p.base_color * (dscale * kInvPi);
        r.lobe |= kLobeDiffuseReflection;
    }
    if (ps > 0.f) {
        const float den = 4.f * fabsf(wo.z * wi.z);
        if (den <= kDirEps) return bsdf_eval_invalid();
        r.specular = fr * (d * g / den);
        r.lobe |= kLobeGlossyReflection;
    }
    r.value = r.diffuse + r.specular;
    r.pdf = pd * wi.z * kInvPi + ps * spdf;
    r.measure = kMeasureSolidAngle;
    r.valid = finite3(r.value) && finite3(r.diffuse) && finite3(r.specular) && isfinite(r.pdf) && r.pdf > 0.f;
    return r.valid ? r : bsdf_eval_invalid();
}

__device__ __forceinline__ bool rough_dielectric_half(f3 wo, f3 wi, float eta_rel, bool& refl, f3& m) {
    refl = wo.z * wi.z > 0.f;
    m = f3s(0.f);
    const f3 h = refl ? wo + wi : wo + wi * eta_rel;
    if (fabsf(wo.z) <= kDirEps || fabsf(wi.z) <= kDirEps || !safe_normalize(h, m)) return false;
    if (m.z < 0.f) m = -m;
    return dot(m, wi) * wi.z >= 0.f && dot(m, wo) * wo.z >= 0.f;
}

__device__ __forceinline__ bool rough_dielectric_probabilities(const BsdfParams& p, float fr, float& pr, float& pt) {
    pr = has_flags(p.lobes, kLobeGlossyReflection) ? fr : 0.f;
    pt = has_flags(p.lobes, kLobeGlossyTransmission) ? (1.f - fr) * p.transmission : 0.f;
    const float tot = pr + pt;
    if (!isfinite(tot) || tot <= 0.f) return false;
    pr /= tot;
    pt /= tot;
    return true;
}

__device__ __forceinline__ BsdfEval eval_rough_dielectric(const BsdfContext& c, const BsdfParams& p, f3 wo, f3 wi) {
    BsdfEval r = bsdf_eval_invalid();
    const float eta_rel = c.eta_t / c.eta_i;
    if (!isfinite(eta_rel) || eta_rel <= 0.f) return r;
    bool refl;
    f3 m;
    if (!rough_dielectric_half(wo, wi, eta_rel, refl, m)) return r;
    float fr;
    if (!fresnel_dielectric(dot(wo, m), c.eta_i, c.eta_t, fr)) return r;
    float pr, pt;
    if (!rough_dielectric_probabilities(p, fr, pr, pt)) return r;
    const float alpha = p.roughness * p.roughness;
    const float d = ggx_d(m, alpha);
    const float g = ggx_g2(wo, wi, alpha);
    const float npdf = ggx_vndf_pdf(wo, m, alpha);
    if (d <= 0.f || g < 0.f || npdf <= 0.f) return r;
    if (refl) {
        if (pr <= 0.f) return r;
        const float wom = fabsf(dot(wo, m));
        const float vden = 4.f * fabsf(wo.z * wi.z);
        if (wom <= kDirEps || vden <= kDirEps) return r;
        r.specular = f3s(fr) * (d * g / vden);
        r.pdf = npdf / (4.f * wom) * pr;
        r.lobe = kLobeGlossyReflection;
    } else {
        if (pt <= 0.f) return r;
        const float wom = dot(wo, m);
        const float wim = dot(wi, m);
        const float dt = wim + wom / eta_rel;
        const float jden = dt * dt;
        const float cp = wo.z * wi.z;
        if (jden <= kDirEps || fabsf(cp) <= kDirEps) return r;
        const float dmdwi = fabsf(wim) / jden;
        float tv = p.transmission * (1.f - fr) * d * g * fabsf(wim * wom / (cp * jden));
        if (c.transport == 0u) tv /= eta_rel * eta_rel;
        r.specular = f3s(tv);
        r.pdf = npdf * dmdwi * pt;
        r.lobe = kLobeGlossyTransmission;
    }
    r.value = r.specular;
    r.measure = kMeasureSolidAngle;
    r.valid = finite3(r.value) && isfinite(r.pdf) && r.pdf > 0.f;
    return r.valid ? r : bsdf_eval_invalid();
}

// EvaluateBsdfL6 (PbrBsdf.hlsli:1115-1229).
__device__ __forceinline__ BsdfEval bsdf_evaluate_body(const BsdfContext& c, const BsdfParams& p, f3 wo_in, f3 wi_in) {
    BsdfEval r = bsdf_eval_invalid();
    if (!validate_params(c, p)) return r;
    Frame f;
    if (!build_frame(c, wo_in, f)) return r;
    f3 wi;
    if (!safe_normalize(wi_in, wi)) return r;
    const f3 wil = to_local(wi, f);
    if (p.model == kModelLambert) r = eval_lambert(p, f.wo_local, wil);
    else if (p.model == kModelGgxConductor || p.model == kModelGgxDielectricReflection)
        r = eval_ggx_reflection(c, p, f.wo_local, wil);
    else if (p.model == kModelRoughDielectric) r = eval_rough_dielectric(c, p, f.wo_local, wil);
    else if (p.model == kModelMetallicRoughness) r = eval_metallic_roughness(p, f.wo_local, wil);
    else if (p.model == kModelSmoothGlass) {
        r.measure = kMeasureDiscrete;
        return r;
    }
    if (!r.valid || !validate_world_event(f.wo, wi, f.ng, r.lobe)) return bsdf_eval_invalid();
    float corr;
    if (!shading_correction(c, f, wi, corr)) return bsdf_eval_invalid();
    r.value *= corr;
    r.diffuse *= corr;
    r.specular *= corr;
    if (!finite3(r.value) || !finite3(r.diffuse) || !finite3(r.specular)) return bsdf_eval_invalid();
    return r;
}

__device__ __forceinline__ f3 sample_cosine_hemisphere(float u1, float u2) {
    const float r = sqrtf(u1);
    const float phi = 2.f * kPi * u2;
    return mk(r * cosf(phi), r * sinf(phi), sqrtf(fmaxf(0.f, 1.f - u1)));
}

__device__ __forceinline__ bool refract_local(f3 wo, f3 m_in, float eta_rel, f3& wi) {
    wi = f3s(0.f);
    f3 m = m_in;
    float ci = dot(m, wo);
    if (ci < 0.f) {
        m = -m;
        ci = -ci;
    }
    if (ci <= kDirEps || !isfinite(eta_rel) || eta_rel <= 0.f) return false;
    const float st2 = fmaxf(0.f, 1.f - ci * ci) / (eta_rel * eta_rel);
    if (st2 >= 1.f) return false;
    const float ct = sqrtf(fmaxf(0.f, 1.f - st2));
    const f3 cand = (-wo) / eta_rel + m * (ci / eta_rel - ct);
    return safe_normalize(cand, wi);
}

__device__ __forceinline__ BsdfSample sample_smooth_glass(const BsdfContext& c, const BsdfParams& p, f3 wo,
                                                          float ev) {
    BsdfSample r = bsdf_sample_invalid();
    float fr;
    if (!fresnel_dielectric(wo.z, c.eta_i, c.eta_t, fr)) return r;
    const float rw = has_flags(p.lobes, kLobeSpecularReflection) ? fr : 0.f;
    const float tw = has_flags(p.lobes, kLobeSpecularTransmission) ? (1.f - fr) * p.transmission : 0.f;
    const float tot = rw + tw;
    if (!isfinite(tot) || tot <= 0.f) return r;
    const float pr = rw / tot;
    const float pt = tw / tot;
    r.measure = kMeasureDiscrete;
    r.delta = true;
    r.eta = 1.f;
    if (ev < pr) {
        r.dir = mk(-wo.x, -wo.y, wo.z);
        const float cs = fabsf(r.dir.z);
        if (cs <= kDirEps || pr <= 0.f) return bsdf_sample_invalid();
        r.pdf = pr;
        r.value = f3s(fr) / cs;
        r.specular = r.value;
        r.lobe = kLobeSpecularReflection;
    } else {
        const float eta_rel = c.eta_t / c.eta_i;
        if (pt <= 0.f || !refract_local(wo, mk(0.f, 0.f, 1.f), eta_rel, r.dir)) return bsdf_sample_invalid();
        const float cs = fabsf(r.dir.z);
        if (cs <= kDirEps) return bsdf_sample_invalid();
        r.pdf = pt;
        float v = (1.f - fr) * p.transmission / cs;
        if (c.transport == 0u) v /= eta_rel * eta_rel;
        r.value = f3s(v);
        r.specular = r.value;
        r.eta = eta_rel;
        r.lobe = kLobeSpecularTransmission;
    }
    r.valid = finite3(r.dir) && finite3(r.value) && isfinite(r.pdf) && r.pdf > 0.f;
    return r.valid ? r : bsdf_sample_invalid();
}

__device__ __forceinline__ BsdfSample sample_finite_local(const BsdfContext& c, const BsdfParams& p, f3 wo, f3 u) {
    BsdfSample r = bsdf_sample_invalid();
    r.measure = kMeasureSolidAngle;
    r.eta = 1.f;
    if (p.model == kModelLambert) {
        if (!has_flags(p.lobes, kLobeDiffuseReflection)) return bsdf_sample_invalid();
        r.dir = sample_cosine_hemisphere(u.y, u.z);
        r.lobe = kLobeDiffuseReflection;
        r.valid = true;
        return r;
    }
    const float alpha = p.roughness * p.roughness;
    if (p.model == kModelGgxConductor || p.model == kModelGgxDielectricReflection) {
        if (!has_flags(p.lobes, kLobeGlossyReflection)) return bsdf_sample_invalid();
        f3 m;
        if (!ggx_sample_vndf(wo, alpha, u.y, u.z, m)) return bsdf_sample_invalid();
        r.dir = -wo + m * (2.f * dot(wo, m));
        if (r.dir.z <= kDirEps) return bsdf_sample_invalid();
        r.lobe = kLobeGlossyReflection;
        r.valid = true;
        return r;
    }
    if (p.model == kModelMetallicRoughness) {
        float pd, ps;
        if (!metallic_lobe_probabilities(p, wo, pd, ps)) return bsdf_sample_invalid();
        if (u.x < pd) {
            r.dir = sample_cosine_hemisphere(u.y, u.z);
            r.lobe = kLobeDiffuseReflection;
        } else {
            f3 m;
            if (ps <= 0.f || !ggx_sample_vndf(wo, alpha, u.y, u.z, m)) return bsdf_sample_invalid();
            r.dir = -wo + m * (2.f * dot(wo, m));
            if (r.dir.z <= kDirEps) return bsdf_sample_invalid();
            r.lobe = kLobeGlossyReflection;
        }
        r.valid = true;
        return r;
    }
    if (p.model == kModelRoughDielectric) {
        f3 m;
        if (!ggx_sample_vndf(wo, alpha, u.y, u.z, m)) return bsdf_sample_invalid();
        float fr;
        if (!fresnel_dielectric(dot(wo, m), c.eta_i, c.eta_t, fr)) return bsdf_sample_invalid();
        float pr, pt;
        if (!rough_dielectric_probabilities(p, fr, pr, pt)) return bsdf_sample_invalid();
        if (u.x < pr) {
            r.dir = -wo + m * (2.f * dot(wo, m));
            if (r.dir.z <= kDirEps) return bsdf_sample_invalid();
            r.lobe = kLobeGlossyReflection;
        } else {
            const float eta_rel = c.eta_t / c.eta_i;
            if (pt <= 0.f || !refract_local(wo, m, eta_rel, r.dir) || r.dir.z >= -kDirEps)
                return bsdf_sample_invalid();
            r.eta = eta_rel;
            r.lobe = kLobeGlossyTransmission;
        }
        r.valid = true;
        return r;
    }
    return bsdf_sample_invalid();
}

// SampleBsdfL6 (PbrBsdf.hlsli:1569-1677).
__device__ __forceinline__ BsdfSample bsdf_sample_body(const BsdfContext& c, const BsdfParams& p, f3 wo_in, f3 u) {
    BsdfSample r = bsdf_sample_invalid();
    const bool unit_u = finite3(u) && u.x >= 0.f && u.y >= 0.f && u.z >= 0.f && u.x < 1.f && u.y < 1.f && u.z < 1.f;
    if (!validate_params(c, p) || !unit_u) return r;
    Frame f;
    if (!build_frame(c, wo_in, f)) return r;
    const BsdfSample ls =
        p.model == kModelSmoothGlass ? sample_smooth_glass(c, p, f.wo_local, u.x) : sample_finite_local(c, p, f.wo_local, u);
    if (!ls.valid) return r;
    f3 wi;
    if (!safe_normalize(to_world(ls.dir, f), wi) || !validate_world_event(f.wo, wi, f.ng, ls.lobe))
        return bsdf_sample_invalid();
    if (ls.measure == kMeasureSolidAngle) {
        const BsdfEval e = bsdf_evaluate_body(c, p, f.wo, wi);
        if (!e.valid) return bsdf_sample_invalid();
        r.dir = wi;
        r.pdf = e.pdf;
        r.value = e.value;
        r.eta = ls.eta;
        r.diffuse = e.diffuse;
        r.specular = e.specular;
        r.measure = kMeasureSolidAngle;
        r.lobe = ls.lobe;
        r.delta = false;
        r.valid = true;
        return r;
    }
    float corr;
    if (!shading_correction(c, f, wi, corr)) return bsdf_sample_invalid();
    r = ls;
    r.dir = wi;
    r.value *= corr;
    r.diffuse *= corr;
    r.specular *= corr;
    r.valid = finite3(r.value) && finite3(r.specular);
    return r.valid ? r : bsdf_sample_invalid();
}

// Call-site variants: out-of-line calls keep the caller's register footprint
// small; inlined bodies avoid the call ABI.  The wavefront Shade kernel is
// built both ways and the autotuner picks one.
static __device__ __noinline__ BsdfEval bsdf_evaluate_call(const BsdfContext& c, const BsdfParams& p, f3 wo, f3 wi) {
    return bsdf_evaluate_body(c, p, wo, wi);
}
static __device__ __noinline__ BsdfSample bsdf_sample_call(const BsdfContext& c, const BsdfParams& p, f3 wo, f3 u) {
    return bsdf_sample_body(c, p, wo, u);
}
template <bool INLINE>
__device__ __forceinline__ BsdfEval bsdf_evaluate(const BsdfContext& c, const BsdfParams& p, f3 wo, f3 wi) {
    if constexpr (INLINE) return bsdf_evaluate_body(c, p, wo, wi);
    else return bsdf_evaluate_call(c, p, wo, wi);
}
template <bool INLINE>
__device__ __forceinline__ BsdfSample bsdf_sample(const BsdfContext& c, const BsdfParams& p, f3 wo, f3 u) {
    if constexpr (INLINE) return bsdf_sample_body(c, p, wo, u);
    else return bsdf_sample_call(c, p, wo, u);
}

}  // namespace re
