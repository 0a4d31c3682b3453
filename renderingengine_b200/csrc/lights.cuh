// Light selection and sampling on the device: alias-table light selection,
// emissive-triangle, sphere, point/spot and directional lights, the selected
// light PDF used by MIS on emitter hits, the power heuristic and the ray
// origin offset.  Semantics follow
// resources/shaders/integrators/pbr_light_sampling.hlsli:14-726 and
// pbr_l6_types.hlsli:423-439.
#pragma once

#include "bsdf.cuh"

namespace re {

constexpr uint32_t kLightPoint = 0, kLightDirectional = 1, kLightSpot = 2, kLightSphere = 3, kLightTriangle = 4,
                   kLightEnvironment = 5;
constexpr uint32_t kLightEnabled = 1u, kLightTwoSided = 2u;
constexpr uint32_t kSampleValid = 1u, kSampleDelta = 2u, kSampleInfinite = 4u, kSampleTwoSided = 8u;
constexpr uint32_t kMeasureLightDiscrete = 0, kMeasureLightArea = 1, kMeasureLightSolidAngle = 2;

// Device copies of PbrLightGpu (96 B), AliasEntryGpu (16 B) and
// FixtureTriangleGpu (64 B) records, read as float4/uint4 lanes.
struct LightView {
    const float4* lights;       // 6 x float4 per light
    const float4* alias;        // 1 x float4 per entry (q, pmf, alias bits, item bits)
    const float* pmf_by_light;  // selection PMF per light
    const float4* fixtures;     // 4 x float4 per emissive triangle
    uint32_t light_count;
    uint32_t alias_count;
    uint32_t fixture_count;
    // Environment light: equirectangular linear-RGBA texels (row 0 at
    // theta = 0), the row alias table (height entries) and one column alias
    // table per row (width entries each), as BuildEnvironmentDistribution
    // (MegakernelBridge.cpp:191-273) lays them out.  env_light = ~0: none.
    uint32_t env_light;
    const float4* env_texels;
    const float4* env_rows;
    const float4* env_cols;
    uint32_t env_width, env_height;
    uint32_t env_uniform;       // 1: uniform-sphere sampling (a black map)
};

struct LightRecord {
    float4 position_range;
    float4 direction_cos_outer;
    float4 radiance_scale;
    float4 shape;
    uint4 identity;
    uint4 payload;
};

__device__ __forceinline__ LightRecord load_light(const LightView& v, uint32_t i) {
    const float4* p = v.lights + size_t(i) * 6u;
    LightRecord l;
    l.position_range = __ldg(p + 0);
    l.direction_cos_outer = __ldg(p + 1);
    l.radiance_scale = __ldg(p + 2);
    l.shape = __ldg(p + 3);
    l.identity = __ldg(reinterpret_cast<const uint4*>(p + 4));
    l.payload = __ldg(reinterpret_cast<const uint4*>(p + 5));
    return l;
}

struct LightContext {
    f3 p;
    f3 ng;
    f3 ns;
    // The frame's environment_to_world (rows 0..2) and world_to_environment
    // (rows 3..5) transforms, read only by environment lights.
    const float4* env_xf;
};

struct LightRandom {
    float selection, s0, s1, s2, s3;
};

struct LightSample {
    f3 wi;
    float distance;
    f3 li;
    float selection_pmf;
    float conditional_pdf;
    float combined_pdf;
    uint32_t light;
    uint32_t instance;
    uint32_t primitive;
    f3 position;
    uint32_t measure;
    f3 normal;
    uint32_t flags;
};

__device__ __forceinline__ LightSample light_sample_invalid() {
    LightSample s;
    s.wi = f3s(0.f); s.distance = 0.f; s.li = f3s(0.f); s.selection_pmf = 0.f; s.conditional_pdf = 0.f;
    s.combined_pdf = 0.f; s.light = 0xffffffffu; s.instance = 0xffffffffu; s.primitive = 0xffffffffu;
    s.position = f3s(0.f); s.measure = 0xffffffffu; s.normal = f3s(0.f); s.flags = 0u;
    return s;
}

// Orthonormal basis around a unit normal (PbrBuildBasisL6, :33-40).
__device__ __forceinline__ void build_basis(f3 n, f3& t, f3& b) {
    const float sign = n.z >= 0.f ? 1.f : -1.f;
    const float a = -1.f / (sign + n.z);
    const float bb = n.x * n.y * a;
    t = mk(1.f + sign * n.x * n.x * a, sign * bb, -sign * n.x);
    b = mk(bb, sign + n.y * n.y * a, -n.y);
}

__device__ __forceinline__ f3 light_radiance(const LightRecord& l) {
    return mk(l.radiance_scale.x, l.radiance_scale.y, l.radiance_scale.z) * l.radiance_scale.w;
}

// PbrSampleAliasL6 (:47-69): returns the selected entry's item and pmf.
__device__ __forceinline__ bool sample_alias(const float4* table, uint32_t count, float u, uint32_t& item,
                                             float& pmf) {
    item = 0xffffffffu;
    pmf = 0.f;
    if (count == 0u) return false;
    const float scaled = u * float(count);
    const uint32_t bin = min(uint32_t(scaled), count - 1u);
    const float within = scaled - float(bin);
    const float4 e = __ldg(table + bin);
    const uint32_t sel = within < e.x ? bin : __float_as_uint(e.z);
    if (sel >= count) return false;
    const float4 s = __ldg(table + sel);
    item = __float_as_uint(s.w);
    pmf = s.y;
    return true;
}

__device__ __forceinline__ LightSample sample_point_spot(const LightContext& c, const LightRecord& l, uint32_t idx,
                                                         float pmf) {
    LightSample s = light_sample_invalid();
    const f3 to = mk(l.position_range.x, l.position_range.y, l.position_range.z) - c.p;
    const float d2 = dot(to, to);
    if (!(d2 > 0.f) || !(pmf > 0.f)) return s;
    const float d = sqrtf(d2);
    if (l.position_range.w > 0.f && d > l.position_range.w) return s;
    const f3 wi = to / d;
    float falloff = 1.f;
    if (l.identity.x == kLightSpot) {
        const f3 dir = mk(l.direction_cos_outer.x, l.direction_cos_outer.y, l.direction_cos_outer.z);
        const float dl2 = dot(dir, dir);
        if (!(dl2 > 0.f) || !isfinite(dl2)) return s;
        const f3 fwd = dir / sqrtf(dl2);
        const float ca = dot(fwd, -wi);
        const float co = l.direction_cos_outer.w, ci = l.shape.y;
        if (ci == co) {
            falloff = ca >= co ? 1.f : 0.f;
        } else {
            float t = (ca - co) / (ci - co);  // HLSL smoothstep
            t = fminf(fmaxf(t, 0.f), 1.f);
            falloff = t * t * (3.f - 2.f * t);
        }
        if (!(falloff > 0.f)) return s;
    }
    s.wi = wi;
    s.distance = d;
    s.li = light_radiance(l) * (falloff / d2);
    s.selection_pmf = pmf;
    s.conditional_pdf = 1.f;
    s.combined_pdf = 0.f;
    s.light = idx;
    s.primitive = 0xffffffffu;
    s.position = mk(l.position_range.x, l.position_range.y, l.position_range.z);
    s.measure = kMeasureLightDiscrete;
    s.flags = kSampleValid | kSampleDelta;
    return s;
}

__device__ __forceinline__ LightSample sample_directional(const LightRecord& l, uint32_t idx, float pmf) {
    LightSample s = light_sample_invalid();
    const f3 dir = mk(l.direction_cos_outer.x, l.direction_cos_outer.y, l.direction_cos_outer.z);
    const float dl2 = dot(dir, dir);
    if (!(dl2 > 0.f) || !(pmf > 0.f)) return s;
    s.wi = (-dir) / sqrtf(dl2);
    s.distance = 1.0e30f;
    s.li = light_radiance(l);
    s.selection_pmf = pmf;
    s.conditional_pdf = 1.f;
    s.combined_pdf = 0.f;
    s.light = idx;
    s.primitive = 0xffffffffu;
    s.measure = kMeasureLightDiscrete;
    s.flags = kSampleValid | kSampleDelta | kSampleInfinite;
    return s;
}

__device__ __forceinline__ bool load_fixture(const LightView& v, const LightRecord& l, f3& p0, f3& p1, f3& p2) {
    if (l.payload.x >= v.fixture_count) return false;
    const float4* f = v.fixtures + size_t(l.payload.x) * 4u;
    const uint4 meta = __ldg(reinterpret_cast<const uint4*>(f + 3));
    if (meta.z != l.payload.w || meta.y != l.identity.w) return false;
    p0 = from4(__ldg(f + 0));
    p1 = from4(__ldg(f + 1));
    p2 = from4(__ldg(f + 2));
    return true;
}

// PbrSampleTriangleLightL6 (:240-300).
__device__ __forceinline__ LightSample sample_triangle(const LightView& v, const LightContext& c,
                                                       const LightRecord& l, uint32_t idx, float pmf, float u1,
                                                       float u2) {
    LightSample s = light_sample_invalid();
    f3 p0, p1, p2;
    if (!(pmf > 0.f) || !load_fixture(v, l, p0, p1, p2)) return s;
    const f3 e1 = p1 - p0, e2 = p2 - p0;
    const f3 nu = cross(e1, e2);
    const float twice = sqrtf(dot(nu, nu));
    if (!(twice > 0.f)) return s;
    const float root = sqrtf(u1);
    const float b0 = 1.f - root, b1 = root * (1.f - u2), b2 = root * u2;
    const f3 lp = p0 * b0 + p1 * b1 + p2 * b2;
    const f3 to = lp - c.p;
    const float d2 = dot(to, to);
    if (!(d2 > 0.f)) return s;
    const float d = sqrtf(d2);
    const f3 wi = to / d;
    const f3 ln = nu / twice;
    const float lc = dot(ln, -wi);
    const bool two = (l.identity.y & kLightTwoSided) != 0u;
    const float ac = two ? fabsf(lc) : lc;
    if (!(ac > 0.f)) return s;
    const float area = 0.5f * twice;
    const float pdf_area = 1.f / area;
    const float pdf_sa = pdf_area * d2 / ac;
    s.wi = wi;
    s.distance = d;
    s.li = light_radiance(l);
    s.selection_pmf = pmf;
    s.conditional_pdf = pdf_area;
    s.combined_pdf = pmf * pdf_sa;
    s.light = idx;
    s.instance = l.payload.w;
    s.primitive = l.identity.w;
    s.position = lp;
    s.measure = kMeasureLightArea;
    s.normal = ln;
    s.flags = kSampleValid | (two ? kSampleTwoSided : 0u);
    return s;
}

// PbrSampleSphereLightL6 (:302-421).
__device__ __forceinline__ LightSample sample_sphere(const LightContext& c, const LightRecord& l, uint32_t idx,
                                                     float pmf, float u1, float u2) {
    LightSample s = light_sample_invalid();
    const float radius = l.shape.x;
    const f3 center = mk(l.position_range.x, l.position_range.y, l.position_range.z);
    if (!(radius > 0.f) || !(pmf > 0.f)) return s;
    const f3 tc = center - c.p;
    const float d2 = dot(tc, tc);
    const float r2 = radius * radius;
    const bool two = (l.identity.y & kLightTwoSided) != 0u;
    f3 wi, lp, ln;
    float dist, cpdf;
    uint32_t measure;
    if (d2 > r2 * 1.000001f) {
        const float cd = sqrtf(d2);
        const f3 cdir = tc / cd;
        const float sin2max = r2 / d2;
        const float cosmax = sqrtf(fmaxf(0.f, 1.f - sin2max));
        const float omc = sin2max < 0.00068523f ? 0.5f * sin2max : 1.f - cosmax;
        const float ct = 1.f - u1 * omc;
        const float st = sqrtf(fmaxf(0.f, 1.f - ct * ct));
        const float phi = kTwoPi * u2;
        f3 t, b;
        build_basis(cdir, t, b);
        wi = normalize3(cdir * ct + t * (cosf(phi) * st) + b * (sinf(phi) * st));
        const f3 oc = c.p - center;
        const float hb = dot(oc, wi);
        const float disc = hb * hb - (dot(oc, oc) - r2);
        if (!(disc >= 0.f)) return s;
        dist = -hb - sqrtf(disc);
        if (!(dist > 0.f)) dist = -hb + sqrtf(disc);
        if (!(dist > 0.f) || !(omc > 0.f)) return s;
        lp = c.p + wi * dist;
        ln = normalize3(lp - center);
        cpdf = 1.f / (kTwoPi * omc);
        measure = kMeasureLightSolidAngle;
    } else {
        const float z = 1.f - 2.f * u1;
        const float rd = sqrtf(fmaxf(0.f, 1.f - z * z));
        const float phi = kTwoPi * u2;
        ln = mk(rd * cosf(phi), z, rd * sinf(phi));
        lp = center + ln * radius;
        const f3 to = lp - c.p;
        const float sd2 = dot(to, to);
        if (!(sd2 > 0.f)) return s;
        dist = sqrtf(sd2);
        wi = to / dist;
        const float lc = dot(ln, -wi);
        const float ac = two ? fabsf(lc) : lc;
        if (!(ac > 0.f)) return s;
        cpdf = 1.f / (4.f * kPi * r2);
        s.combined_pdf = pmf * (cpdf * sd2 / ac);
        measure = kMeasureLightArea;
    }
    s.wi = wi;
    s.distance = dist;
    s.li = light_radiance(l);
    s.selection_pmf = pmf;
    s.conditional_pdf = cpdf;
    if (measure == kMeasureLightSolidAngle) s.combined_pdf = pmf * cpdf;
    s.light = idx;
    s.instance = l.payload.w;
    s.primitive = l.identity.w;
    s.position = lp;
    s.measure = measure;
    s.normal = ln;
    s.flags = kSampleValid | (two ? kSampleTwoSided : 0u);
    return s;
}

// ---------------------------------------------------------------------------
// Environment light (pbr_light_sampling.hlsli:74-158, 422-511).  Texels are
// fetched nearest, u wrapping and v clamped to the edge (the environment
// sampler of Wave2Runtime.cpp:2568-2579), so the radiance of a direction is
// exactly the texel whose importance the alias tables hold.
// ---------------------------------------------------------------------------
__device__ __forceinline__ f3 rows_transform(const float4* r, f3 d) {
    return mk(r[0].x * d.x + r[0].y * d.y + r[0].z * d.z, r[1].x * d.x + r[1].y * d.y + r[1].z * d.z,
              r[2].x * d.x + r[2].y * d.y + r[2].z * d.z);
}

// PbrEnvironmentTexelSolidAngleL6 (:74-86).
__device__ __forceinline__ float env_texel_solid_angle(const LightView& v, uint32_t row) {
    if (v.env_width == 0u || v.env_height == 0u || row >= v.env_height) return 0.f;
    const float t0 = kPi * float(row) / float(v.env_height);
    const float t1 = kPi * float(row + 1u) / float(v.env_height);
    return (kTwoPi / float(v.env_width)) * (cosf(t0) - cosf(t1));
}

// PbrEnvironmentUvFromLocalDirectionL6 (:88-98).
__device__ __forceinline__ void env_uv(f3 local, float& u, float& v) {
    const f3 d = normalize3(local);
    float phi = atan2f(d.z, d.x);
    if (phi < 0.f) phi += kTwoPi;
    const float theta = acosf(fminf(fmaxf(d.y, -1.f), 1.f));
    u = phi / kTwoPi;
    v = theta / kPi;
}

__device__ __forceinline__ f3 env_texel(const LightView& v, float u, float vv) {
    const int w = int(v.env_width), h = int(v.env_height);
    int i = int(floorf(u * float(w)));
    i %= w;
    if (i < 0) i += w;
    int j = int(floorf(vv * float(h)));
    j = min(max(j, 0), h - 1);
    const float4 t = __ldg(v.env_texels + size_t(j) * size_t(w) + size_t(i));
    return mk(t.x, t.y, t.z);
}

// PbrEnvironmentRadianceL6 (:100-129).
__device__ __forceinline__ f3 env_radiance(const LightView& v, const float4* xf, f3 world_dir) {
    if (v.env_light == 0xffffffffu || v.env_light >= v.light_count) return f3s(0.f);
    const LightRecord l = load_light(v, v.env_light);
    if (l.identity.x != kLightEnvironment || (l.identity.y & kLightEnabled) == 0u) return f3s(0.f);
    float u, vv;
    env_uv(normalize3(rows_transform(xf + 3, world_dir)), u, vv);
    return env_texel(v, u, vv) * light_radiance(l);
}

// PbrEnvironmentPdfL6 (:131-158): solid-angle PDF of a direction.
__device__ __forceinline__ float env_pdf(const LightView& v, const float4* xf, f3 world_dir) {
    if (v.env_width == 0u || v.env_height == 0u) return 0.f;
    if (v.env_uniform) return 1.f / (4.f * kPi);
    float u, vv;
    env_uv(normalize3(rows_transform(xf + 3, world_dir)), u, vv);
    const uint32_t row = min(uint32_t(vv * float(v.env_height)), v.env_height - 1u);
    const uint32_t col = min(uint32_t(u * float(v.env_width)), v.env_width - 1u);
    const float pmf = __ldg(v.env_rows + row).y * __ldg(v.env_cols + size_t(row) * v.env_width + col).y;
    const float sa = env_texel_solid_angle(v, row);
    return sa > 0.f ? pmf / sa : 0.f;
}

// PbrSampleEnvironmentLightL6 (:421-511).
__device__ __forceinline__ LightSample sample_environment(const LightView& v, const LightContext& c,
                                                          const LightRecord& l, uint32_t idx, float pmf,
                                                          const LightRandom& u) {
    LightSample s = light_sample_invalid();
    const uint32_t w = v.env_width, h = v.env_height;
    if (!(pmf > 0.f) || w == 0u || h == 0u) return s;
    f3 local;
    float tu, tv, pdf;
    if (v.env_uniform) {
        const float ct = 1.f - 2.f * u.s0;
        const float st = sqrtf(fmaxf(0.f, 1.f - ct * ct));
        const float phi = kTwoPi * u.s1;
        local = mk(st * cosf(phi), ct, st * sinf(phi));
        env_uv(local, tu, tv);
        pdf = 1.f / (4.f * kPi);
    } else {
        uint32_t row, col;
        float rp, cp;
        if (!sample_alias(v.env_rows, h, u.s0, row, rp) || row >= h || !(rp > 0.f)) return s;
        if (!sample_alias(v.env_cols + size_t(row) * w, w, u.s1, col, cp) || col >= w || !(cp > 0.f)) return s;
        const float t0 = kPi * float(row) / float(h);
        const float t1 = kPi * float(row + 1u) / float(h);
        const float c0 = cosf(t0), c1 = cosf(t1);
        const float ct = c0 + (c1 - c0) * u.s3;  // HLSL lerp
        const float st = sqrtf(fmaxf(0.f, 1.f - ct * ct));
        const float phi = kTwoPi * (float(col) + u.s2) / float(w);
        local = mk(st * cosf(phi), ct, st * sinf(phi));
        const float sa = env_texel_solid_angle(v, row);
        if (!(sa > 0.f)) return s;
        tu = (float(col) + u.s2) / float(w);
        tv = acosf(fminf(fmaxf(ct, -1.f), 1.f)) / kPi;
        pdf = rp * cp / sa;
    }
    s.wi = normalize3(rows_transform(c.env_xf, local));
    s.distance = 1.0e30f;
    s.li = env_texel(v, tu, tv) * light_radiance(l);
    s.selection_pmf = pmf;
    s.conditional_pdf = pdf;
    s.combined_pdf = pmf * pdf;
    s.light = idx;
    s.primitive = 0xffffffffu;
    s.measure = kMeasureLightSolidAngle;
    s.flags = kSampleValid | kSampleInfinite;
    return s;
}

// PbrSampleOneLightL6 (:512-600).
__device__ __forceinline__ LightSample sample_one_light_body(const LightView& v, const LightContext& c,
                                                            const LightRandom& u) {
    LightSample inv = light_sample_invalid();
    if (v.alias_count == 0u) return inv;
    uint32_t item;
    float pmf;
    if (!sample_alias(v.alias, v.alias_count, u.selection, item, pmf)) return inv;
    if (item >= v.light_count || !(pmf > 0.f)) return inv;
    const LightRecord l = load_light(v, item);
    if ((l.identity.y & kLightEnabled) == 0u) return inv;
    switch (l.identity.x) {
        case kLightPoint:
        case kLightSpot:
            return sample_point_spot(c, l, item, pmf);
        case kLightDirectional:
            return sample_directional(l, item, pmf);
        case kLightSphere:
            return sample_sphere(c, l, item, pmf, u.s0, u.s1);
        case kLightTriangle:
            return sample_triangle(v, c, l, item, pmf, u.s0, u.s1);
        case kLightEnvironment:
            return item == v.env_light ? sample_environment(v, c, l, item, pmf, u) : inv;
        default:
            return inv;
    }
}

static __device__ __noinline__ LightSample sample_one_light_call(const LightView& v, const LightContext& c,
                                                         const LightRandom& u) {
    return sample_one_light_body(v, c, u);
}
template <bool INLINE>
__device__ __forceinline__ LightSample sample_one_light(const LightView& v, const LightContext& c,
                                                        const LightRandom& u) {
    if constexpr (INLINE) return sample_one_light_body(v, c, u);
    else return sample_one_light_call(v, c, u);
}

// PbrLightPdfLiL6 (:602-700).
__device__ __forceinline__ float light_pdf_li(const LightView& v, uint32_t idx, const LightContext& c, f3 wi,
                                              float dist, f3 emitter_normal) {
    if (idx == 0xffffffffu || idx >= v.light_count) return 0.f;
    const LightRecord l = load_light(v, idx);
    if ((l.identity.y & kLightEnabled) == 0u) return 0.f;
    const uint32_t type = l.identity.x;
    if (type == kLightEnvironment) return idx == v.env_light ? env_pdf(v, c.env_xf, wi) : 0.f;
    if (type == kLightTriangle) {
        f3 p0, p1, p2;
        if (!(dist > 0.f) || !load_fixture(v, l, p0, p1, p2)) return 0.f;
        const f3 cr = cross(p1 - p0, p2 - p0);
        const float area = 0.5f * sqrtf(dot(cr, cr));
        const float lc = dot(emitter_normal, -wi);
        const float cosine = (l.identity.y & kLightTwoSided) != 0u ? fabsf(lc) : lc;
        return area > 0.f && cosine > 0.f ? dist * dist / (area * cosine) : 0.f;
    }
    if (type == kLightSphere) {
        const float radius = l.shape.x;
        const f3 tc = mk(l.position_range.x, l.position_range.y, l.position_range.z) - c.p;
        const float d2 = dot(tc, tc);
        const float r2 = radius * radius;
        if (!(radius > 0.f)) return 0.f;
        if (d2 > r2 * 1.000001f) {
            const float sin2max = r2 / d2;
            const float cosmax = sqrtf(fmaxf(0.f, 1.f - sin2max));
            const float omc = sin2max < 0.00068523f ? 0.5f * sin2max : 1.f - cosmax;
            return omc > 0.f ? 1.f / (kTwoPi * omc) : 0.f;
        }
        const float lc = dot(emitter_normal, -wi);
        const float cosine = (l.identity.y & kLightTwoSided) != 0u ? fabsf(lc) : lc;
        const float area = 4.f * kPi * r2;
        return dist > 0.f && cosine > 0.f ? dist * dist / (area * cosine) : 0.f;
    }
    return 0.f;
}

__device__ __forceinline__ float selected_light_pdf(const LightView& v, uint32_t idx, const LightContext& c, f3 wi,
                                                    float dist, f3 emitter_normal) {
    if (idx == 0xffffffffu || idx >= v.light_count) return 0.f;
    return __ldg(v.pmf_by_light + idx) * light_pdf_li(v, idx, c, wi, dist, emitter_normal);
}

// PbrPowerHeuristicL6 (pbr_l6_types.hlsli:423-439).
__device__ __forceinline__ float power_heuristic(float a, float b) {
    if (!isfinite(a) || !isfinite(b) || a < 0.f || b < 0.f) return 0.f;
    const float m = fmaxf(a, b);
    if (!(m > 0.f) || !isfinite(m)) return 0.f;
    const float na = a / m, nb = b / m;
    const float sa = na * na, sb = nb * nb;
    return sa / (sa + sb);
}

// PbrOffsetRayOriginL6 (pbr_light_sampling.hlsli:719-724).
__device__ __forceinline__ f3 offset_origin(f3 p, f3 ng, f3 dir, float eps) {
    const float side = dot(ng, dir) >= 0.f ? 1.f : -1.f;
    return p + ng * (side * eps);
}

}  // namespace re
