// TEST INFRASTRUCTURE ONLY -- FP32 CPU oracle of the wavefront PBR integrator.
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
//
// A scalar, one-path-at-a-time restatement of the reference's wavefront PBR
// path (the GPU path has no CPU implementation in the reference):
//   RayGen      integrators/wavefront/shaders/RayGen.hlsl:10-93
//   Shade       integrators/wavefront/shaders/Shade.hlsl:6-479
//   NEE split   integrators/wavefront/shaders/include/PbrWavefrontShading.hlsli:127-330
//   TraceShadow integrators/wavefront/shaders/TraceShadow.hlsl:5-92 (Physical)
//   NextBounce  integrators/wavefront/shaders/NextBounce.hlsl:6-115
//   Resolve     integrators/wavefront/shaders/Resolve.hlsl:6-90
//   BSDF        resources/shaders/include/bsdf/PbrBsdf.hlsli:82-1679
//   lights      resources/shaders/integrators/pbr_light_sampling.hlsli:14-726
//   material    resources/shaders/integrators/pbr_material_bsdf.hlsli:8-131
//   Philox/MIS  resources/shaders/integrators/pbr_l6_types.hlsli:352-439
//   alias table integrators/megakernel/MegakernelBridge.cpp:40-144, 403-455
// Per-path RNG is counter based, so evaluating each path to completion is the
// same computation the wavefront schedule performs stage by stage.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <unordered_map>
#include <vector>

#include "oracle_common.h"

using namespace oracle;

namespace {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTwoPi = 6.28318530717958647692f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kEps = 1.0e-7f;
constexpr float kMinAlpha = 1.0e-4f;
constexpr uint32_t kInv = 0xffffffffu;


// ---------------------------------------------------------------------------
// Philox4x32-10 (pbr_l6_types.hlsli:352-420; MegakernelBridge.cpp:552-589)
// ---------------------------------------------------------------------------
float counter_random(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = uint64_t(0xd2511f53u) * c0;
        const uint64_t p1 = uint64_t(0xcd9e8d57u) * c2;
        const uint32_t n0 = uint32_t(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n1 = uint32_t(p1);
        const uint32_t n2 = uint32_t(p0 >> 32) ^ c3 ^ k1;
        const uint32_t n3 = uint32_t(p0);
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9e3779b9u;
        k1 += 0xbb67ae85u;
    }
    return float(c0 >> 8) * (1.0f / 16777216.0f);
}

uint32_t bdim(uint32_t bounce, uint32_t local) { return 4u + bounce * 16u + local; }

// ---------------------------------------------------------------------------
// BSDF (PbrBsdf.hlsli)
// ---------------------------------------------------------------------------
// libm transcendentals evaluated by the path being traced (this thread):
// the places where CUDA's sinf / cosf / powf / acosf / atan2f and glibc's
// may differ in the last bit, which is what lets a device film pixel differ
// from the oracle's.
thread_local uint32_t g_libm_calls = 0;
inline float lcos(float x) { ++g_libm_calls; return std::cos(x); }
inline float lsin(float x) { ++g_libm_calls; return std::sin(x); }
inline float lpow(float x, float y) { ++g_libm_calls; return std::pow(x, y); }
inline float lacos(float x) { ++g_libm_calls; return std::acos(x); }
inline float latan2(float y, float x) { ++g_libm_calls; return std::atan2(y, x); }

using R = float;
using V = V3;
inline V vv(R x, R y, R z) { return v3(x, y, z); }
inline V spl(R s) { return splat(s); }
#include "oracle_bsdf.inc"

// ---------------------------------------------------------------------------
// Lights (pbr_light_sampling.hlsli)
// ---------------------------------------------------------------------------
struct Light { float pos[4], dir[4], rad[4], shape[4]; uint32_t id[4], payload[4]; };
struct Fixture { float p0[4], p1[4], p2[4]; uint32_t meta[4]; };
struct Alias { float q, pmf; uint32_t alias, item; };
// measure: 0 discrete, 1 area, 2 solid angle (kInv when invalid).
struct LSmp {
    V3 wi; float dist; V3 li; float sel_pmf, cond_pdf, comb_pdf; uint32_t light, inst, prim; uint32_t flags;
    V3 pos; uint32_t measure;
};
LSmp ls_inv() { return {splat(0), 0, splat(0), 0, 0, 0, kInv, kInv, kInv, 0, splat(0), kInv}; }

struct Scene {
    const void* nodes; uint32_t node_count;
    const float* tri_v; const uint32_t* tri_key; const float* tri_n; const uint32_t* tri_ids; const uint32_t* emitter;
    const float* materials; uint32_t material_count;
    const Light* lights; uint32_t light_count;
    std::vector<Alias> alias; std::vector<float> pmf;
    const Fixture* fixtures; uint32_t fixture_count;
    // Environment map (row 0 at theta = 0), its importance tables and the
    // enabled environment light (kInv: none).
    const float* env = nullptr; uint32_t env_w = 0, env_h = 0, env_light = 0xffffffffu;
    bool env_uniform = false; double env_integrated = 0.0;
    std::vector<Alias> env_rows, env_cols;
    const float* xf = nullptr;  // frame rows: environment_to_world 0..2, world_to_environment 3..5 (4 floats each)
    const AlphaData* alpha = nullptr;  // alpha-masked triangles' coverage data
};

void basis(V3 n, V3& t, V3& b) {
    const float s = n.z >= 0.f ? 1.f : -1.f;
    const float a = -1.f / (s + n.z), bb = n.x * n.y * a;
    t = v3(1.f + s * n.x * n.x * a, s * bb, -s * n.x);
    b = v3(bb, s + n.y * n.y * a, -n.y);
}
V3 lrad(const Light& l) { return v3(l.rad[0], l.rad[1], l.rad[2]) * l.rad[3]; }
bool fixture(const Scene& s, const Light& l, V3& p0, V3& p1, V3& p2) {
    if (l.payload[0] >= s.fixture_count) return false;
    const Fixture& f = s.fixtures[l.payload[0]];
    if (f.meta[2] != l.payload[3] || f.meta[1] != l.id[3]) return false;
    p0 = v3(f.p0[0], f.p0[1], f.p0[2]); p1 = v3(f.p1[0], f.p1[1], f.p1[2]); p2 = v3(f.p2[0], f.p2[1], f.p2[2]);
    return true;
}
// ---- environment light (pbr_light_sampling.hlsli:74-158, 422-511) ----
V3 rows3(const float* r, V3 d) {
    return v3(r[0] * d.x + r[1] * d.y + r[2] * d.z, r[4] * d.x + r[5] * d.y + r[6] * d.z,
              r[8] * d.x + r[9] * d.y + r[10] * d.z);
}
float env_solid_angle(const Scene& s, uint32_t row) {  // :74-86
    if (s.env_w == 0 || s.env_h == 0 || row >= s.env_h) return 0.f;
    const float t0 = kPi * float(row) / float(s.env_h), t1 = kPi * float(row + 1u) / float(s.env_h);
    return (kTwoPi / float(s.env_w)) * (lcos(t0) - lcos(t1));
}
void env_uv(V3 local, float& u, float& v) {  // :88-98
    const V3 d = normalize(local);
    float phi = latan2(d.z, d.x);
    if (phi < 0.f) phi += kTwoPi;
    u = phi / kTwoPi;
    v = lacos(std::fmin(std::fmax(d.y, -1.f), 1.f)) / kPi;
}
V3 env_texel(const Scene& s, float u, float v) {  // nearest, u repeat, v clamp
    const int w = int(s.env_w), h = int(s.env_h);
    int i = int(std::floor(u * float(w))) % w;
    if (i < 0) i += w;
    const int j = std::min(std::max(int(std::floor(v * float(h))), 0), h - 1);
    const float* t = s.env + (size_t(j) * size_t(w) + size_t(i)) * 4u;
    return v3(t[0], t[1], t[2]);
}
V3 env_radiance(const Scene& s, V3 wd) {  // :100-129
    if (s.env_light == kInv || s.env_light >= s.light_count) return splat(0);
    const Light& l = s.lights[s.env_light];
    if (l.id[0] != 5 || (l.id[1] & 1u) == 0u) return splat(0);
    float u, v;
    env_uv(normalize(rows3(s.xf + 12, wd)), u, v);
    return env_texel(s, u, v) * lrad(l);
}
float env_pdf(const Scene& s, V3 wd) {  // :131-158
    if (s.env_w == 0 || s.env_h == 0) return 0.f;
    if (s.env_uniform) return 1.f / (4.f * kPi);
    float u, v;
    env_uv(normalize(rows3(s.xf + 12, wd)), u, v);
    const uint32_t row = std::min(uint32_t(v * float(s.env_h)), s.env_h - 1u);
    const uint32_t col = std::min(uint32_t(u * float(s.env_w)), s.env_w - 1u);
    const float pmf = s.env_rows[row].pmf * s.env_cols[size_t(row) * s.env_w + col].pmf;
    const float sa = env_solid_angle(s, row);
    return sa > 0.f ? pmf / sa : 0.f;
}
bool alias_pick(const Alias* t, uint32_t n, float u, uint32_t& item, float& pmf) {  // PbrSampleAliasL6 :47-69
    if (n == 0) return false;
    const float scaled = u * float(n);
    const uint32_t bin = std::min(uint32_t(scaled), n - 1u);
    const float within = scaled - float(bin);
    const uint32_t sel = within < t[bin].q ? bin : t[bin].alias;
    if (sel >= n) return false;
    item = t[sel].item;
    pmf = t[sel].pmf;
    return true;
}

LSmp sample_light(const Scene& s, V3 P, const float u[5]) {
    LSmp r = ls_inv();
    const uint32_t n = uint32_t(s.alias.size());
    if (n == 0) return r;
    const float scaled = u[0] * float(n);
    const uint32_t bin = std::min(uint32_t(scaled), n - 1u);
    const float within = scaled - float(bin);
    const uint32_t sel = within < s.alias[bin].q ? bin : s.alias[bin].alias;
    if (sel >= n) return r;
    const uint32_t idx = s.alias[sel].item;
    const float pmf = s.alias[sel].pmf;
    if (idx >= s.light_count || !(pmf > 0.f)) return r;
    const Light& l = s.lights[idx];
    if ((l.id[1] & 1u) == 0u) return r;
    const bool two = (l.id[1] & 2u) != 0u;
    if (l.id[0] == 4) {  // triangle :240-300
        V3 p0, p1, p2;
        if (!fixture(s, l, p0, p1, p2)) return r;
        const V3 nu = cross(p1 - p0, p2 - p0);
        const float tw = std::sqrt(dot(nu, nu));
        if (!(tw > 0.f)) return r;
        const float root = std::sqrt(u[1]);
        const V3 lp = p0 * (1.f - root) + p1 * (root * (1.f - u[2])) + p2 * (root * u[2]);
        const V3 to = lp - P;
        const float d2 = dot(to, to);
        if (!(d2 > 0.f)) return r;
        const float d = std::sqrt(d2);
        const V3 wi = to / d;
        const V3 ln = nu / tw;
        const float lc = dot(ln, -wi), ac = two ? std::fabs(lc) : lc;
        if (!(ac > 0.f)) return r;
        const float pa = 1.f / (0.5f * tw);
        r.wi = wi; r.dist = d; r.li = lrad(l); r.sel_pmf = pmf; r.cond_pdf = pa; r.comb_pdf = pmf * (pa * d2 / ac);
        r.light = idx; r.inst = l.payload[3]; r.prim = l.id[3]; r.flags = 1u | (two ? 8u : 0u);
        r.pos = lp; r.measure = 1u;
        return r;
    }
    if (l.id[0] == 3) {  // sphere :302-421
        const float rad = l.shape[0];
        const V3 c = v3(l.pos[0], l.pos[1], l.pos[2]);
        if (!(rad > 0.f)) return r;
        const V3 tc = c - P;
        const float d2 = dot(tc, tc), r2 = rad * rad;
        V3 wi, lpos; float dist, cpdf; bool solid;
        if (d2 > r2 * 1.000001f) {
            const float cd = std::sqrt(d2);
            const V3 cdir = tc / cd;
            const float s2 = r2 / d2, cm = std::sqrt(std::fmax(0.f, 1.f - s2));
            const float omc = s2 < 0.00068523f ? 0.5f * s2 : 1.f - cm;
            const float ct = 1.f - u[1] * omc, st = std::sqrt(std::fmax(0.f, 1.f - ct * ct));
            const float phi = kTwoPi * u[2];
            V3 t, b;
            basis(cdir, t, b);
            wi = normalize(cdir * ct + t * (lcos(phi) * st) + b * (lsin(phi) * st));
            const V3 oc = P - c;
            const float hb = dot(oc, wi), disc = hb * hb - (dot(oc, oc) - r2);
            if (!(disc >= 0.f)) return r;
            dist = -hb - std::sqrt(disc);
            if (!(dist > 0.f)) dist = -hb + std::sqrt(disc);
            if (!(dist > 0.f) || !(omc > 0.f)) return r;
            lpos = P + wi * dist;
            cpdf = 1.f / (kTwoPi * omc);
            solid = true;
        } else {
            const float z = 1.f - 2.f * u[1], rd = std::sqrt(std::fmax(0.f, 1.f - z * z)), phi = kTwoPi * u[2];
            const V3 ln = v3(rd * lcos(phi), z, rd * lsin(phi));
            const V3 lp = c + ln * rad;
            const V3 to = lp - P;
            const float sd2 = dot(to, to);
            if (!(sd2 > 0.f)) return r;
            dist = std::sqrt(sd2);
            wi = to / dist;
            const float lc = dot(ln, -wi), ac = two ? std::fabs(lc) : lc;
            if (!(ac > 0.f)) return r;
            cpdf = 1.f / (4.f * kPi * r2);
            r.comb_pdf = pmf * (cpdf * sd2 / ac);
            lpos = lp;
            solid = false;
        }
        r.wi = wi; r.dist = dist; r.li = lrad(l); r.sel_pmf = pmf; r.cond_pdf = cpdf;
        if (solid) r.comb_pdf = pmf * cpdf;
        r.light = idx; r.inst = l.payload[3]; r.prim = l.id[3]; r.flags = 1u | (two ? 8u : 0u);
        r.pos = lpos; r.measure = solid ? 2u : 1u;
        return r;
    }
    if (l.id[0] == 5) {  // environment :421-511
        if (idx != s.env_light || s.env_w == 0 || s.env_h == 0) return r;
        V3 local;
        float tu, tv, pdf;
        if (s.env_uniform) {
            const float ct = 1.f - 2.f * u[1], st = std::sqrt(std::fmax(0.f, 1.f - ct * ct)), phi = kTwoPi * u[2];
            local = v3(st * lcos(phi), ct, st * lsin(phi));
            env_uv(local, tu, tv);
            pdf = 1.f / (4.f * kPi);
        } else {
            uint32_t row, col;
            float rp, cp;
            if (!alias_pick(s.env_rows.data(), s.env_h, u[1], row, rp) || row >= s.env_h || !(rp > 0.f)) return r;
            if (!alias_pick(s.env_cols.data() + size_t(row) * s.env_w, s.env_w, u[2], col, cp) || col >= s.env_w ||
                !(cp > 0.f))
                return r;
            const float t0 = kPi * float(row) / float(s.env_h), t1 = kPi * float(row + 1u) / float(s.env_h);
            const float c0 = lcos(t0), c1 = lcos(t1);
            const float ct = c0 + (c1 - c0) * u[4], st = std::sqrt(std::fmax(0.f, 1.f - ct * ct));
            const float phi = kTwoPi * (float(col) + u[3]) / float(s.env_w);
            local = v3(st * lcos(phi), ct, st * lsin(phi));
            const float sa = env_solid_angle(s, row);
            if (!(sa > 0.f)) return r;
            tu = (float(col) + u[3]) / float(s.env_w);
            tv = lacos(std::fmin(std::fmax(ct, -1.f), 1.f)) / kPi;
            pdf = rp * cp / sa;
        }
        r.wi = normalize(rows3(s.xf, local)); r.dist = 1.0e30f; r.li = env_texel(s, tu, tv) * lrad(l);
        r.sel_pmf = pmf; r.cond_pdf = pdf; r.comb_pdf = pmf * pdf;
        r.light = idx; r.prim = kInv; r.flags = 1u | 4u; r.pos = splat(0); r.measure = 2u;
        return r;
    }
    if (l.id[0] == 1) {  // directional
        const V3 d = v3(l.dir[0], l.dir[1], l.dir[2]);
        const float dl2 = dot(d, d);
        if (!(dl2 > 0.f)) return r;
        r.wi = (-d) / std::sqrt(dl2); r.dist = 1.0e30f; r.li = lrad(l); r.sel_pmf = pmf; r.cond_pdf = 1.f;
        r.light = idx; r.flags = 1u | 2u | 4u;
        r.pos = splat(0); r.measure = 0u;
        return r;
    }
    return r;
}
float light_pdf(const Scene& s, uint32_t idx, V3 P, V3 wi, float dist, V3 en) {
    if (idx == kInv || idx >= s.light_count) return 0.f;
    const Light& l = s.lights[idx];
    if ((l.id[1] & 1u) == 0u) return 0.f;
    float pdf = 0.f;
    if (l.id[0] == 5) {
        pdf = idx == s.env_light ? env_pdf(s, wi) : 0.f;
    } else if (l.id[0] == 4) {
        V3 p0, p1, p2;
        if (!(dist > 0.f) || !fixture(s, l, p0, p1, p2)) return 0.f;
        const V3 cr = cross(p1 - p0, p2 - p0);
        const float area = 0.5f * std::sqrt(dot(cr, cr));
        const float lc = dot(en, -wi), cs = (l.id[1] & 2u) ? std::fabs(lc) : lc;
        pdf = area > 0.f && cs > 0.f ? dist * dist / (area * cs) : 0.f;
    } else if (l.id[0] == 3) {
        const float rad = l.shape[0];
        const V3 tc = v3(l.pos[0], l.pos[1], l.pos[2]) - P;
        const float d2 = dot(tc, tc), r2 = rad * rad;
        if (!(rad > 0.f)) return 0.f;
        if (d2 > r2 * 1.000001f) {
            const float s2 = r2 / d2, cm = std::sqrt(std::fmax(0.f, 1.f - s2));
            const float omc = s2 < 0.00068523f ? 0.5f * s2 : 1.f - cm;
            pdf = omc > 0.f ? 1.f / (kTwoPi * omc) : 0.f;
        } else {
            const float lc = dot(en, -wi), cs = (l.id[1] & 2u) ? std::fabs(lc) : lc;
            pdf = dist > 0.f && cs > 0.f ? dist * dist / ((4.f * kPi * r2) * cs) : 0.f;
        }
    }
    return s.pmf[idx] * pdf;
}
float power(float a, float b) {
    if (!std::isfinite(a) || !std::isfinite(b) || a < 0.f || b < 0.f) return 0.f;
    const float m = std::fmax(a, b);
    if (!(m > 0.f) || !std::isfinite(m)) return 0.f;
    const float na = a / m, nb = b / m, sa = na * na, sb = nb * nb;
    return sa / (sa + sb);
}
V3 offset(V3 p, V3 ng, V3 d, float eps) { return p + ng * ((dot(ng, d) >= 0.f ? 1.f : -1.f) * eps); }

// Vose alias table (MegakernelBridge.cpp:40-144): FP64 probabilities, LIFO
// small / large stacks, leftovers q = 1; items default to the index.
std::vector<Alias> vose(const std::vector<double>& w, const std::vector<uint32_t>& items) {
    const size_t n = w.size();
    std::vector<Alias> out(n);
    if (n == 0) return out;
    double sum = 0;
    for (double x : w) sum += x;
    const bool uni = sum == 0.0;
    const double norm = sum > 0 ? sum : double(n);
    std::vector<double> prob(n), sc(n);
    std::vector<uint32_t> small, large;
    for (size_t i = 0; i < n; ++i) {
        prob[i] = uni ? 1.0 / double(n) : w[i] / norm;
        sc[i] = prob[i] * double(n);
        out[i] = {0.f, float(prob[i]), uint32_t(i), items.empty() ? uint32_t(i) : items[i]};
        (sc[i] < 1.0 ? small : large).push_back(uint32_t(i));
    }
    while (!small.empty() && !large.empty()) {
        const uint32_t a = small.back(); small.pop_back();
        const uint32_t b = large.back(); large.pop_back();
        out[a].q = float(std::clamp(sc[a], 0.0, 1.0));
        out[a].alias = b;
        sc[b] = sc[b] + sc[a] - 1.0;
        (sc[b] < 1.0 ? small : large).push_back(b);
    }
    for (uint32_t i : large) { out[i].q = 1.f; out[i].alias = i; }
    for (uint32_t i : small) { out[i].q = 1.f; out[i].alias = i; }
    return out;
}

// Top-level distribution (BuildTopLevelLightDistribution, :403-455).
void build_distribution(Scene& s, uint32_t selection, float scene_radius) {
    std::vector<double> w;
    std::vector<uint32_t> items;
    const double pi = 3.141592653589793238462643383279502884;
    for (uint32_t i = 0; i < s.light_count; ++i) {
        const Light& l = s.lights[i];
        if ((l.id[1] & 1u) == 0u) continue;
        double wt = 1.0;
        if (selection == 1) {
            const double lu = (0.2126 * double(l.rad[0]) + 0.7152 * double(l.rad[1]) + 0.0722 * double(l.rad[2])) * double(l.rad[3]);
            const double two = (l.id[1] & 2u) ? 2.0 : 1.0;
            if (l.id[0] == 3) wt = 4.0 * pi * pi * double(l.shape[0]) * double(l.shape[0]) * lu * two;
            else if (l.id[0] == 4) wt = pi * double(l.shape[2]) * lu * two;
            else if (l.id[0] == 0) wt = 4.0 * pi * lu;
            else if (l.id[0] == 1) wt = pi * double(scene_radius) * double(scene_radius) * lu;
            else if (l.id[0] == 5) wt = pi * double(scene_radius) * double(scene_radius) * double(l.rad[3]) * s.env_integrated;
            else wt = 0.0;
        }
        w.push_back(wt);
        items.push_back(i);
    }
    s.pmf.assign(std::max(1u, s.light_count), 0.f);
    s.alias = vose(w, items);
    for (const Alias& a : s.alias) s.pmf[a.item] = a.pmf;
}

// BuildEnvironmentDistribution (MegakernelBridge.cpp:191-273) over the
// texels' luminance 0.2126 r + 0.7152 g + 0.0722 b (Wave2Runtime.cpp:589-600).
void build_environment(Scene& s) {
    const double pi = 3.141592653589793238462643383279502884;
    const uint32_t w = s.env_w, h = s.env_h;
    auto sa = [&](uint32_t row) {
        const double t0 = pi * double(row) / double(h), t1 = pi * double(row + 1u) / double(h);
        return 2.0 * pi / double(w) * (std::cos(t0) - std::cos(t1));
    };
    std::vector<double> tw(size_t(w) * h);
    s.env_integrated = 0.0;
    for (uint32_t r = 0; r < h; ++r)
        for (uint32_t c = 0; c < w; ++c) {
            const float* t = s.env + (size_t(r) * w + c) * 4u;
            const float lu = 0.2126f * t[0] + 0.7152f * t[1] + 0.0722f * t[2];
            tw[size_t(r) * w + c] = double(lu) * sa(r);
            s.env_integrated += double(lu) * sa(r);
        }
    s.env_uniform = s.env_integrated == 0.0;
    if (s.env_uniform)
        for (uint32_t r = 0; r < h; ++r)
            for (uint32_t c = 0; c < w; ++c) tw[size_t(r) * w + c] = sa(r);
    std::vector<double> rw(h, 0.0);
    s.env_cols.clear();
    for (uint32_t r = 0; r < h; ++r) {
        const std::vector<double> span(tw.begin() + size_t(r) * w, tw.begin() + size_t(r + 1) * w);
        for (double x : span) rw[r] += x;
        const std::vector<Alias> t = vose(span, {});
        s.env_cols.insert(s.env_cols.end(), t.begin(), t.end());
    }
    s.env_rows = vose(rw, {});
}

// ---------------------------------------------------------------------------
// Path integrator
// ---------------------------------------------------------------------------
struct Frame {
    float cam_pos[3], tan_half_fov, fwd[3], aspect, right[3], pad0, up[3], pad1;
    uint32_t width, height, sample, max_depth, seed_lo, seed_hi, estimator, stream;
    float rr_start, rr_min, rr_max, eps;
    float env_xf[24];  // environment_to_world rows, then world_to_environment rows
};

struct PathOut {
    V3 cam, dd, ds, id, is; float gb_pos[4], gb_nrm[4], gb_alb[4]; uint32_t rays, shadows, flags;
    float surf[24];  // GpuPrimarySurfaceV2, the ReSTIR copy (zero on a primary miss)
};

float sat1(float v) { return std::fmin(std::fmax(v, 0.f), 1.f); }

// PbrPublishPrimarySurfaceV2 (pbr_reconstruction_export_v2.hlsli:42-92).
void publish_surface(float* q, V3 P, float depth, V3 ng, V3 ns, uint32_t material, uint32_t instance,
                     uint32_t primitive, uint32_t front, V3 base, float metal, float rough, float trans, V3 f0,
                     bool supported) {
    const float m = sat1(metal);
    const V3 bc = v3(std::fmax(base.x, 0.f), std::fmax(base.y, 0.f), std::fmax(base.z, 0.f));
    const V3 da = bc * (1.f - m) * (1.f - sat1(trans));
    const V3 sl = f0 + (base - f0) * m;
    const V3 sa = v3(std::fmax(sl.x, 0.f), std::fmax(sl.y, 0.f), std::fmax(sl.z, 0.f));
    uint32_t flags = supported ? 1u : 0u;
    if (da.x > 0.f || da.y > 0.f || da.z > 0.f) flags |= 4u;
    if (sa.x > 0.f || sa.y > 0.f || sa.z > 0.f) flags |= 8u;
    if (front != 0u) flags |= 2u;
    const V3 gn = normalize(ng), sn = normalize(ns);
    const float vals[20] = {P.x, P.y, P.z, std::fmax(depth, 0.f), gn.x, gn.y, gn.z, sat1(rough),
                            sn.x, sn.y, sn.z, m, da.x, da.y, da.z, 0.f, sa.x, sa.y, sa.z, 0.f};
    std::memcpy(q, vals, sizeof(vals));
    const uint32_t id[4] = {material, instance, primitive, flags};
    std::memcpy(q + 20, id, 16);
}

bool acc_terminal(PathOut& o, uint32_t bounce, V3 beta, V3 bd, V3 bs, V3 e, float mis) {
    auto fnn = [](V3 v) { return finite3(v) && nonneg3(v); };
    if (!fnn(e) || !std::isfinite(mis) || mis < 0.f || !fnn(beta) || !fnn(bd) || !fnn(bs)) return false;
    const V3 w = e * mis;
    if (!fnn(w)) return false;
    if (bounce == 0) {
        const V3 a = o.cam + beta * w;
        if (!fnn(a)) return false;
        o.cam = a;
    } else {
        V3& D = bounce == 1 ? o.dd : o.id;
        V3& S = bounce == 1 ? o.ds : o.is;
        const V3 df = D + bd * w, sf = S + bs * w;
        if (!fnn(df) || !fnn(sf)) return false;
        D = df;
        S = sf;
    }
    return true;
}

PathOut trace_path(const Scene& s, const Frame& f, uint32_t pixel) {
    PathOut o{};
    o.gb_nrm[3] = 0.f;
    uint32_t kinv = kInv;
    std::memcpy(&o.gb_nrm[3], &kinv, 4);
    const uint32_t sample = f.sample;
    auto rnd = [&](uint32_t dim) { return counter_random(pixel, sample, dim, f.stream, f.seed_lo, f.seed_hi); };
    // RayGen
    const uint32_t x = pixel % f.width, y = pixel / f.width;
    const float jx = rnd(0), jy = rnd(1);
    float sx = (float(x) + jx) / float(f.width), sy = (float(y) + jy) / float(f.height);
    sx = sx * 2.f - 1.f;
    sy = sy * 2.f - 1.f;
    sy = -sy;
    const V3 cam = v3(f.cam_pos[0], f.cam_pos[1], f.cam_pos[2]);
    const V3 fwd = v3(f.fwd[0], f.fwd[1], f.fwd[2]);
    V3 ro = cam;
    V3 rd = normalize(fwd + v3(f.right[0], f.right[1], f.right[2]) * (sx * f.aspect * f.tan_half_fov) +
                      v3(f.up[0], f.up[1], f.up[2]) * (sy * f.tan_half_fov));
    float rtmin = f.eps, rtmax = 1.0e30f;
    V3 beta = splat(1.f), bd = splat(0.f), bs = splat(0.f);
    float eta_scale = 1.f;
    V3 prev_p = splat(0), prev_ng = splat(0), prev_ns = splat(0);
    float prev_pdf = 0.f;
    uint32_t flags = 1u | 2u;  // active | previous delta
    for (uint32_t bounce = 0; bounce < f.max_depth; ++bounce) {
        ++o.rays;
        const TraceResult h = trace_flat(s.nodes, s.node_count, s.tri_v, s.tri_key, ro, rtmin, rd, rtmax, false,
                                         false, kInv, kInv, s.alpha);
        if (h.status != 0) { o.flags = flags | 16u; return o; }
        if (h.tri == kInv) {  // miss (Shade.hlsl:74-118): the environment, MIS-weighted
            if (s.env_light != kInv) {
                const V3 env = env_radiance(s, rd);
                float mis = 1.f;
                if (bounce != 0 && (flags & 2u) == 0 && f.estimator != 0) {
                    if (f.estimator == 3 && bounce == 1 && (flags & 32u)) mis = 0.f;
                    else {
                        const float lp = light_pdf(s, s.env_light, prev_p, rd, 0.f, splat(0));
                        if (lp > 0.f) mis = power(prev_pdf, lp);
                    }
                }
                if (!finite3(env) || !std::isfinite(mis) || !acc_terminal(o, bounce, beta, bd, bs, env, mis)) {
                    o.flags = flags | 16u;
                    return o;
                }
            }
            break;
        }
        // Hit reconstruction (pbr_software_traversal.hlsli:150-186).
        const float* tv = s.tri_v + size_t(h.tri) * 9u;
        const V3 p0 = v3(tv[0], tv[1], tv[2]);
        const V3 e1 = v3(tv[3], tv[4], tv[5]) - p0, e2 = v3(tv[6], tv[7], tv[8]) - p0;
        const float* tn = s.tri_n + size_t(h.tri) * 9u;
        const float w0 = 1.0f - h.u - h.v;
        V3 ng = normalize(cross(e1, e2));
        V3 ns = normalize(w0 * v3(tn[0], tn[1], tn[2]) + h.u * v3(tn[3], tn[4], tn[5]) + h.v * v3(tn[6], tn[7], tn[8]));
        if (!h.front) { ng = -ng; ns = -ns; }
        const uint32_t* ids = s.tri_ids + size_t(h.tri) * 4u;
        const uint32_t mat_idx = ids[3];
        const uint32_t emitter = s.emitter[h.tri];
        const V3 P = ro + rd * h.t;
        const float gl2 = dot(ng, ng), sl2 = dot(ns, ns);
        if (!(std::isfinite(h.t) && h.t >= rtmin && h.t <= rtmax && finite3(P) && std::isfinite(gl2) && gl2 > 0.f &&
              std::isfinite(sl2) && sl2 > 0.f) || mat_idx >= s.material_count) {
            o.flags = flags | 16u;
            return o;
        }
        const float* m = s.materials + size_t(mat_idx) * 32u;
        uint32_t meta[4];
        std::memcpy(meta, m + 28, 16);
        const V3 emission = v3(m[4], m[5], m[6]);
        // PbrMaterialAuxiliaryIsValidL6
        if (!finite3(emission) || any_neg(emission) || !std::isfinite(m[12]) || !std::isfinite(m[13]) ||
            !std::isfinite(m[14]) || !std::isfinite(m[15]) || m[15] < 0.f ||
            (m[15] > 0.f && (!(m[12] > 0.f && m[13] > 0.f && m[14] > 0.f) || !(m[12] <= 1.f && m[13] <= 1.f && m[14] <= 1.f)))) {
            o.flags = flags | 16u;
            return o;
        }
        Params par{v3(m[0], m[1], m[2]), m[3], v3(m[16], m[17], m[18]), m[7], v3(m[20], m[21], m[22]), m[8],
                   v3(m[24], m[25], m[26]), meta[0], meta[1], meta[2]};
        if (par.model == RoughDielectric && std::isfinite(par.rough) && par.rough >= 0.f && par.rough * par.rough < kMinAlpha) {
            par.model = SmoothGlass;
            if (par.lobes & LG) par.lobes = (par.lobes & ~LG) | LS;
        }
        const bool owned = bounce == 0 && restir_primary(par);
        if (bounce == 0) {
            const V3 nf = normalize(fwd);
            o.gb_pos[0] = P.x; o.gb_pos[1] = P.y; o.gb_pos[2] = P.z; o.gb_pos[3] = dot(P - cam, nf);
            o.gb_nrm[0] = ns.x; o.gb_nrm[1] = ns.y; o.gb_nrm[2] = ns.z; std::memcpy(&o.gb_nrm[3], &mat_idx, 4);
            o.gb_alb[0] = m[0]; o.gb_alb[1] = m[1]; o.gb_alb[2] = m[2]; o.gb_alb[3] = m[7];
            publish_surface(o.surf, P, o.gb_pos[3], ng, ns, mat_idx, ids[0], ids[1], h.front, v3(m[0], m[1], m[2]),
                            m[3], m[7], m[8], v3(m[16], m[17], m[18]), owned);
        }
        // Beer-Lambert (pbr_material_bsdf.hlsli:78-129)
        if (!h.front && m[8] > 0.f && m[15] > 0.f) {
            const float e = h.t / m[15];
            const V3 att = v3(lpow(m[12], e), lpow(m[13], e), lpow(m[14], e));
            beta = beta * att; bd = bd * att; bs = bs * att;
            if (!finite3(att) || !finite3(beta) || !finite3(bd) || !finite3(bs)) { o.flags = flags | 16u; return o; }
        }
        // Emission + MIS
        bool visible = h.front != 0;
        if (!visible && emitter < s.light_count) visible = (s.lights[emitter].id[1] & 2u) != 0u;
        if (visible && maxc(emission) > 0.f) {
            float mis = 1.f;
            if (bounce != 0 && (flags & 2u) == 0 && f.estimator != 0) {
                if (f.estimator == 3 && bounce == 1 && (flags & 32u)) mis = 0.f;
                else {
                    const float lp = light_pdf(s, emitter, prev_p, rd, h.t, ng);
                    if (lp > 0.f) mis = power(prev_pdf, lp);
                }
            }
            if (!acc_terminal(o, bounce, beta, bd, bs, emission, mis)) { o.flags = flags | 16u; return o; }
        }
        if ((meta[3] & 1u) || !finite3(beta) || any_neg(beta)) break;
        Ctx ctx;
        ctx.ng = ng;
        ctx.ns = ns;
        V3 tb;
        basis(ns, ctx.tan, tb);
        const float ior = m[9];
        ctx.ei = h.front ? 1.f : ior;
        ctx.et = h.front ? ior : 1.f;
        ctx.transport = 0;
        if (!validate(ctx, par)) { o.flags = flags | 16u; return o; }
        const V3 wo = -rd;
        // NEE -> shadow ray -> accumulate when visible.
        if (f.estimator != 0 && !s.alias.empty() && !(f.estimator == 3 && bounce == 0 && owned)) {
            float u[5] = {rnd(bdim(bounce, 0)), rnd(bdim(bounce, 1)), rnd(bdim(bounce, 2)), rnd(bdim(bounce, 3)),
                          rnd(bdim(bounce, 4))};
            const LSmp ls = sample_light(s, P, u);
            if (ls.flags & 1u) {
                const Eval ev = evaluate(ctx, par, wo, ls.wi);
                bool go = ev.valid && std::isfinite(ev.pdf) && finite3(ev.value) && ev.pdf >= 0.f;
                const bool delta = (ls.flags & 2u) != 0u;
                const float est = delta ? ls.sel_pmf : ls.comb_pdf;
                go = go && std::isfinite(est) && est > 0.f;
                const float cosine = std::fabs(dot(ng, ls.wi));
                go = go && cosine > 0.f;
                if (go) {
                    const float mis = delta ? 1.f : power(ls.comb_pdf, ev.pdf);
                    const V3 scale = ls.li * (cosine * mis / est);
                    const V3 cd = bounce == 0 ? beta * ev.diff * scale : bd * ev.value * scale;
                    const V3 cs = bounce == 0 ? beta * ev.spec * scale : bs * ev.value * scale;
                    go = finite3(cd) && finite3(cs) && !any_neg(cd) && !any_neg(cs);
                    const float smax = (ls.flags & 4u) ? 1.0e30f : ls.dist - f.eps;
                    if (go && smax > f.eps) {
                        ++o.shadows;
                        const V3 so = offset(P, ng, ls.wi, f.eps);
                        // The sampled light's own (instance, primitive) is excluded from the
                        // visibility query, as PbrEvaluateShadowVisibilityL6 does
                        // (pbr_megakernel.hlsl:178-186); the normal-offset origin with
                        // tMax = distance - epsilon otherwise meets the light itself.
                        const TraceResult sh = trace_flat(s.nodes, s.node_count, s.tri_v, s.tri_key, so, f.eps, ls.wi,
                                                          smax, true, true, ls.inst, ls.prim, s.alpha);
                        if (sh.status != 0) { o.flags = flags | 16u; return o; }
                        if (sh.tri == kInv) {
                            V3& D = bounce == 0 ? o.dd : o.id;
                            V3& S = bounce == 0 ? o.ds : o.is;
                            D = D + cd;
                            S = S + cs;
                        }
                    }
                }
            }
        }
        if (bounce + 1 >= f.max_depth) break;
        const V3 u = v3(rnd(bdim(bounce, 5)), rnd(bdim(bounce, 6)), rnd(bdim(bounce, 7)));
        const Smp b = sample_bsdf(ctx, par, wo, u);
        bool valid = b.valid && std::isfinite(b.pdf) && b.pdf > 0.f && finite3(b.value) && finite3(b.dir) && !any_neg(b.value);
        V3 nb = splat(0), nd = splat(0), nsv = splat(0);
        float es = eta_scale;
        if (valid) {
            const float cosine = std::fabs(dot(ng, b.dir));
            const V3 factor = b.value * (cosine / b.pdf);
            if (bounce == 0) {
                nd = beta * b.diff * (cosine / b.pdf);
                nsv = beta * b.spec * (cosine / b.pdf);
            } else {
                nd = bd * factor;
                nsv = bs * factor;
            }
            nb = nd + nsv;
            valid = finite3(nb) && finite3(nd) && finite3(nsv) && !any_neg(nb);
            if (b.lobe & LT) {
                es *= b.eta * b.eta;
                valid = valid && std::isfinite(es) && es > 0.f;
            }
        }
        const uint32_t next = bounce + 1;
        if (valid && float(next) >= f.rr_start) {
            const float mag = maxc(nb * es);
            if (!(mag > 0.f) || !std::isfinite(mag)) valid = false;
            else {
                const float cont = std::fmin(std::fmax(mag, f.rr_min), f.rr_max);
                if (rnd(bdim(bounce, 9)) >= cont) valid = false;
                else { nb = nb / cont; nd = nd / cont; nsv = nsv / cont; }
            }
        }
        if (!valid) break;
        uint32_t ev = 0;
        if (b.delta) ev |= 2u;
        if ((b.lobe & LD) == 0) ev |= 4u;
        if (owned) ev |= 32u;
        ro = offset(P, ng, b.dir, f.eps);
        rd = normalize(b.dir);
        rtmin = f.eps;
        rtmax = 1.0e30f;
        beta = nb; bd = nd; bs = nsv; eta_scale = es;
        prev_p = P; prev_pdf = b.pdf; prev_ng = ng; prev_ns = ns;
        flags = (flags & 16u) | 1u | ev;
    }
    o.flags = flags;
    return o;
}

// ---------------------------------------------------------------------------
// ReSTIR DI on the primary surface: the production passes of
// resources/shaders/restir/Restir*V3.comp.hlsl and the candidate export of
// resources/shaders/integrators/pbr_restir_candidate_export_v3.hlsl, with the
// reservoir arithmetic of RestirProductionV3.hlsli, in float.
// Records are the ABI words: GpuPrimarySurfaceV2 (24 words),
// GpuRestirReservoirV3 (64 words).
// ---------------------------------------------------------------------------
struct F4 { float x, y, z, w; };
struct U4 { uint32_t x, y, z, w; };
struct RSample { F4 pos_dist, dir_pdf, rad_pmf, cond; U4 identity, generation, metadata, source; };
struct Resv { RSample sel; F4 weight, terms; U4 state, prov, h_surface, h_scene, h_frame, h_reproj; };
struct Surf { F4 pos_depth, gn_rough, sn_metal, dalb, salb; U4 identity; };
struct Cand { RSample s; F4 t; U4 prov; };
static_assert(sizeof(Resv) == 256, "GpuRestirReservoirV3");
static_assert(sizeof(Surf) == 96, "GpuPrimarySurfaceV2");

// ReSTIR parameters of one frame (the GPU's per-frame ReSTIR block).
struct RParams {
    uint32_t candidates, neighbors, max_m, max_age;
    uint32_t history_enabled, neighbor_mode, scene_gen, light_gen;
    uint32_t camera_gen, resolution_gen, history_gen, frame_lo;
    uint32_t frame_hi, prev_valid, candidate_source, light_count;
    uint32_t prev_light_count, estimator, pad1, pad2;  // estimator: 0 biased, 1 reference correction
    float normal_cos, rel_depth, position_dist, disk_radius;
    float prev_pos[3], prev_tan, prev_fwd[3], prev_aspect, prev_right[3], pad3, prev_up[3], pad4;
};

uint32_t rhash(uint32_t v) {
    v ^= v >> 16u; v *= 0x7feb352du; v ^= v >> 15u; v *= 0x846ca68bu; v ^= v >> 16u;
    return v;
}
float rrandom(uint32_t& s) {
    s = rhash(s + 0x9e3779b9u);
    return float(s >> 8u) * (1.0f / 16777216.0f);
}
bool fin4(F4 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z) && std::isfinite(v.w); }
V3 xyz(F4 v) { return v3(v.x, v.y, v.z); }
F4 f4(V3 v, float w) { return {v.x, v.y, v.z, w}; }
bool fnn(float v) { return std::isfinite(v) && v >= 0.f; }

bool surf_valid(const Surf& s) {  // RestirSurfaceValidV3
    const V3 da = xyz(s.dalb), sa = xyz(s.salb), gn = xyz(s.gn_rough), sn = xyz(s.sn_metal);
    return (s.identity.w & 1u) != 0u && fin4(s.pos_depth) && fin4(s.gn_rough) && fin4(s.sn_metal) && fin4(s.dalb) &&
           fin4(s.salb) && da.x >= 0.f && da.y >= 0.f && da.z >= 0.f && da.x <= 1.f && da.y <= 1.f && da.z <= 1.f &&
           sa.x >= 0.f && sa.y >= 0.f && sa.z >= 0.f && sa.x <= 1.f && sa.y <= 1.f && sa.z <= 1.f &&
           s.sn_metal.w >= 0.f && s.sn_metal.w <= 1.f && rough_ok(s.gn_rough.w) && dot(gn, gn) > 1.0e-12f &&
           dot(sn, sn) > 1.0e-12f;
}
bool rsample_valid(const RSample& s, uint32_t scene_gen) {  // RestirSampleValidV3
    return (s.metadata.y & 1u) != 0u && s.identity.x != kInv && s.generation.x != 0u && s.generation.y == scene_gen &&
           fnn(s.dir_pdf.w) && fnn(s.rad_pmf.w) && finite3(xyz(s.dir_pdf)) && finite3(xyz(s.rad_pmf));
}
float rlum(V3 v) {  // RestirLuminanceV3
    return std::fmax(v.x, 0.f) * 0.2126f + std::fmax(v.y, 0.f) * 0.7152f + std::fmax(v.z, 0.f) * 0.0722f;
}
float unshadowed(const RSample& s, const Surf& sf, V3 cam, uint32_t scene_gen, V3& dif, V3& spec) {
    dif = splat(0.f);
    spec = splat(0.f);
    if (!rsample_valid(s, scene_gen) || !surf_valid(sf)) return 0.f;
    const V3 n = normalize(xyz(sf.sn_metal)), l = normalize(xyz(s.dir_pdf)), v = normalize(cam - xyz(sf.pos_depth));
    const float nol = sat1(dot(n, l)), nov = sat1(dot(n, v));
    if (!(nol > 0.f) || !(nov > 0.f)) return 0.f;
    const V3 h = normalize(l + v);
    const float noh = sat1(dot(n, h)), voh = sat1(dot(v, h));
    const float rough = sf.gn_rough.w;
    const V3 da = v3(std::fmax(sf.dalb.x, 0.f), std::fmax(sf.dalb.y, 0.f), std::fmax(sf.dalb.z, 0.f));
    const V3 f0 = v3(std::fmax(sf.salb.x, 0.f), std::fmax(sf.salb.y, 0.f), std::fmax(sf.salb.z, 0.f));
    const V3 f = schlick(voh, f0);
    const float alpha = rough * rough;
    const float d = ggx_d(v3(0.f, 0.f, noh), alpha);
    const float g = g2(v3(std::sqrt(std::fmax(0.f, 1.f - nov * nov)), 0.f, nov),
                       v3(std::sqrt(std::fmax(0.f, 1.f - nol * nol)), 0.f, nol), alpha);
    const V3 rad = v3(std::fmax(s.rad_pmf.x, 0.f), std::fmax(s.rad_pmf.y, 0.f), std::fmax(s.rad_pmf.z, 0.f));
    dif = rad * da * (splat(1.f) - f) * (nol * kInvPi);
    spec = rad * f * (d * g / std::fmax(4.f * nov, 1.0e-6f));
    if (!finite3(dif) || !finite3(spec)) {
        dif = splat(0.f);
        spec = splat(0.f);
        return 0.f;
    }
    return rlum(dif + spec);
}
Cand make_cand(const RSample& s, const Surf& sf, V3 cam, uint32_t scene_gen, uint32_t src, uint32_t reuse,
               uint32_t surf_index) {
    Cand c;
    c.s = s;
    V3 dif, spec;
    const float target = unshadowed(s, sf, cam, scene_gen, dif, spec);
    const float proposal = s.dir_pdf.w;
    const bool sv = surf_valid(sf);
    const float support = rsample_valid(s, scene_gen) && sv && target > 0.f && proposal > 0.f ? 1.f : 0.f;
    c.t = {target, proposal, support, sv ? 1.f : 0.f};
    c.prov = {src, reuse, surf_index, s.metadata.y};
    return c;
}
bool cand_valid(const Cand& c, uint32_t scene_gen) {
    const F4 t = c.t;
    const bool consistent = t.x > 0.f ? t.z == 1.f : t.z == 0.f;
    return rsample_valid(c.s, scene_gen) && fnn(t.x) && std::isfinite(t.y) && t.y > 0.f && (t.z == 0.f || t.z == 1.f) &&
           fnn(t.w) && t.w > 0.f && consistent;
}
float cand_weight(const Cand& c, uint32_t scene_gen) {
    if (!cand_valid(c, scene_gen)) return 0.f;
    return c.t.x * c.t.z * c.t.w / c.t.y;
}
Resv empty_resv() {
    Resv r;
    std::memset(&r, 0, sizeof(r));
    r.sel.identity.x = kInv;
    r.sel.identity.y = kInv;
    return r;
}
void update(Resv& r, const Cand& c, float w, uint32_t mult, float u, uint32_t scene_gen) {
    if (!cand_valid(c, scene_gen) || !std::isfinite(w) || w < 0.f || mult == 0u) return;
    const uint32_t old_m = r.state.x;
    const uint32_t new_m = old_m > 0xffffffffu - mult ? 0xffffffffu : old_m + mult;
    if (w == 0.f) {
        r.state.x = new_m;
        return;
    }
    const float ns = r.weight.x + w;
    if (!(ns > 0.f) || !std::isfinite(ns)) return;
    r.weight.x = ns;
    r.state.x = new_m;
    if (u * ns < w) {
        r.sel = c.s;
        r.weight.z = c.t.x;
        r.weight.w = c.t.y;
        r.terms = {c.t.z, c.t.w, w, 0.f};
        r.prov = c.prov;
    }
}
void finalize(Resv& r) {
    auto invalidate = [&] { r.state.z &= ~1u; r.weight.y = 0.f; };
    if (r.state.x == 0u || !(r.weight.z > 0.f) || !(r.weight.x > 0.f) || !std::isfinite(r.weight.z) ||
        !std::isfinite(r.weight.x)) { invalidate(); return; }
    const float den = float(r.state.x) * r.weight.z;
    if (!(den > 0.f) || !std::isfinite(den)) { invalidate(); return; }
    r.weight.y = r.weight.x / den;
    if (!(r.weight.y > 0.f) || !std::isfinite(r.weight.y)) { invalidate(); return; }
    r.terms.w = r.weight.y;
    r.state.z |= 1u;
}
void clampm(Resv& r, uint32_t max_m) {
    if (r.state.x > max_m) {
        const float scale = float(max_m) / float(r.state.x);
        r.weight.x *= scale;
        r.state.x = max_m;
        r.state.z |= 2u;
    }
}
uint32_t validate_pair(const Surf& a, const Surf& b, const RParams& rp) {  // RestirValidateSurfacePairV3
    if (!surf_valid(a) || !surf_valid(b)) return 1u;
    if (a.identity.x != b.identity.x) return 13u;
    if (a.identity.y != b.identity.y) return 8u;
    const float scale = std::fmax(1.f, std::fmax(std::fabs(a.pos_depth.w), std::fabs(b.pos_depth.w)));
    if (std::fabs(a.pos_depth.w - b.pos_depth.w) / scale > rp.rel_depth) return 6u;
    if (dot(normalize(xyz(a.sn_metal)), normalize(xyz(b.sn_metal))) < rp.normal_cos) return 7u;
    const V3 dd = xyz(a.pos_depth) - xyz(b.pos_depth);
    if (std::sqrt(dot(dd, dd)) > rp.position_dist) return 9u;
    return 0u;
}
// Rejection reason of a temporal history reservoir after reprojection
// (`rej` = 2 outside, 3 no valid reprojection, else 0), in the temporal
// pass's order (RestirTemporalV3.comp.hlsl:20-215): an empty or stale history
// record (1: not published by the previous frame of this history
// generation), scene (10), light (11), camera (4) and resolution (5)
// generations, age (12), a prior pixel outside the frame (2), the surface
// pair (validate_pair), the reprojected depth against the history's depth (6),
// then the selected light's index and generation (11).  `hist` is the prior
// pixel's previous surface, null when the prior pixel is outside the frame.
uint32_t temporal_gate(const Surf& sf, const Surf* hist, const Resv& hs, const RParams& rp, uint32_t rej, float pdepth) {
    if (rej == 0u && ((hs.state.z & 1u) == 0u || hs.state.x == 0u || (hs.h_frame.w & 1u) == 0u)) rej = 1u;
    uint32_t elo = rp.frame_lo, ehi = rp.frame_hi;
    if (elo == 0u) { elo = 0xffffffffu; ehi -= 1u; } else { elo -= 1u; }
    if (rej == 0u && (hs.h_frame.x != elo || hs.h_frame.y != ehi || hs.h_frame.z != rp.history_gen)) rej = 1u;
    else if (rej == 0u && hs.h_scene.x != rp.scene_gen) rej = 10u;
    else if (rej == 0u && hs.h_scene.y != rp.light_gen) rej = 11u;
    else if (rej == 0u && hs.h_scene.z != rp.camera_gen) rej = 4u;
    else if (rej == 0u && hs.h_scene.w != rp.resolution_gen) rej = 5u;
    else if (rej == 0u && hs.state.y >= rp.max_age) rej = 12u;
    else if (rej == 0u && hist == nullptr) rej = 2u;
    else if (rej == 0u) rej = validate_pair(sf, *hist, rp);
    if (rej == 0u) {
        const float hd = hist->pos_depth.w;
        const float scale = std::fmax(1.f, std::fmax(std::fabs(pdepth), std::fabs(hd)));
        if (std::fabs(pdepth - hd) / scale > rp.rel_depth) rej = 6u;
    }
    const uint32_t pl = hs.sel.metadata.w;
    if (rej == 0u && (pl >= rp.prev_light_count || pl >= rp.light_count || rp.light_gen != hs.sel.generation.x))
        rej = 11u;
    return rej;
}

uint32_t measure_abi(uint32_t m) { return m == 0u ? 1u : (m == 1u ? 3u : (m == 2u ? 2u : 0u)); }

RSample persistent(const Scene& s, const RParams& rp, const LSmp& ls, uint32_t flattened) {
    RSample r;
    std::memset(&r, 0, sizeof(r));
    if ((ls.flags & 1u) == 0u || ls.light >= s.light_count) return r;
    const Light& l = s.lights[ls.light];
    r.pos_dist = f4(ls.pos, ls.dist);
    r.dir_pdf = f4(ls.wi, ls.comb_pdf);
    r.rad_pmf = f4(ls.li, ls.sel_pmf);
    if (ls.measure == 1u) r.cond.x = ls.cond_pdf;
    else if (ls.measure == 2u) r.cond.y = ls.cond_pdf;
    r.identity = {l.id[2], ls.prim, flattened, rp.frame_lo};
    r.generation = {rp.light_gen, rp.scene_gen, rp.frame_lo, 0u};
    uint32_t flags = 1u;
    if (ls.flags & 2u) flags |= 2u;
    if (ls.measure == 1u) flags |= 4u;
    if (ls.measure == 2u) flags |= 8u;
    r.metadata = {measure_abi(ls.measure), flags, l.id[1], ls.light};
    return r;
}

bool prev_uv(const RParams& rp, V3 p, float& u, float& v, float& depth) {
    if (rp.prev_valid == 0u) return false;
    const V3 pos = v3(rp.prev_pos[0], rp.prev_pos[1], rp.prev_pos[2]);
    const V3 fwd = v3(rp.prev_fwd[0], rp.prev_fwd[1], rp.prev_fwd[2]);
    const V3 rt = v3(rp.prev_right[0], rp.prev_right[1], rp.prev_right[2]);
    const V3 up = v3(rp.prev_up[0], rp.prev_up[1], rp.prev_up[2]);
    const V3 d = p - pos;
    const float z = dot(d, fwd);
    if (!(z > 1.0e-8f) || !std::isfinite(z)) return false;
    const float sx = dot(d, rt) / (z * rp.prev_aspect * rp.prev_tan);
    const float sy = dot(d, up) / (z * rp.prev_tan);
    u = sx * 0.5f + 0.5f;
    v = 0.5f - sy * 0.5f;
    depth = dot(d, normalize(fwd));
    return std::isfinite(u) && std::isfinite(v) && std::isfinite(depth) && depth >= 0.f;
}

uint32_t neighbor(const RParams& rp, uint32_t w, uint32_t h, uint32_t p, uint32_t k) {
    const int x = int(p % w), y = int(p / w);
    static const int dirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, 1}, {1, -1}, {-1, -1}};
    const int ring = int(k / 8u) + 1;
    int dx = dirs[k % 8u][0] * ring, dy = dirs[k % 8u][1] * ring;
    if (rp.neighbor_mode == 1u) {
        const int r = std::max(1, int(rp.disk_radius));
        const uint32_t span = uint32_t(2 * r + 1);
        uint32_t st = rhash(p ^ rhash(rp.frame_lo + 0x68e31da4u * (k + 1u)));
        for (int a = 0; a < 8; ++a) {
            st = rhash(st + 0x9e3779b9u);
            const int ox = int(st % span) - r, oy = int((st >> 16) % span) - r;
            if ((ox != 0 || oy != 0) && ox * ox + oy * oy <= r * r) {
                dx = ox;
                dy = oy;
                break;
            }
        }
    }
    const int sx = std::min(std::max(x + dx, 0), int(w) - 1), sy = std::min(std::max(y + dy, 0), int(h) - 1);
    return uint32_t(sy) * w + uint32_t(sx);
}

}  // namespace

extern "C" {

// Renders one sample per pixel of a frame with the oracle.  Buffers are in
// leaf order: tri_v (9 floats), tri_key (instance, primitive, traversal,
// flags), tri_n (9 floats), tri_ids (instance, primitive, geometry, material),
// emitter (light index per triangle).  frame: the Frame record above.
// out_planes: 14 planes x pixels x 4 floats: sample, camera emission, direct
// diffuse, direct specular, indirect diffuse, indirect specular, primary
// position, primary normal, then the six 16-byte lanes of the pixel's
// GpuPrimarySurfaceV2.  counts: path rays, shadow rays.
// With an environment map: `env` (env_w x env_h linear RGBA, row 0 at
// theta = 0) radiated by the scene's one enabled environment light; with
// `alpha`, the coverage data of alpha-masked triangles (null: none).
void oracle_render_env(const void* nodes, uint32_t node_count, const float* tri_v, const uint32_t* tri_key,
                       const float* tri_n, const uint32_t* tri_ids, const uint32_t* emitter, const float* materials,
                       uint32_t material_count, const void* lights, uint32_t light_count, const void* fixtures,
                       uint32_t fixture_count, uint32_t light_selection, float scene_radius, const void* frame,
                       const uint32_t* pixels, uint32_t pixel_count, uint32_t threads, float* out_planes,
                       uint64_t* counts, const float* env, uint32_t env_w, uint32_t env_h,
                       const AlphaData* alpha) {
    Scene s{nodes, node_count, tri_v, tri_key, tri_n, tri_ids, emitter, materials, material_count,
            static_cast<const Light*>(lights), light_count, {}, {}, static_cast<const Fixture*>(fixtures), fixture_count};
    s.alpha = alpha;
    Frame f;
    std::memcpy(&f, frame, sizeof(Frame));
    s.xf = f.env_xf;
    if (env != nullptr && env_w != 0 && env_h != 0) {
        s.env = env;
        s.env_w = env_w;
        s.env_h = env_h;
        build_environment(s);
        for (uint32_t i = 0; i < light_count; ++i)
            if (s.lights[i].id[0] == 5 && (s.lights[i].id[1] & 1u)) { s.env_light = i; break; }
    }
    build_distribution(s, light_selection, scene_radius);
    const uint32_t nt = std::max(1u, threads);
    std::vector<uint64_t> rays(nt, 0), shadows(nt, 0);
    auto work = [&](uint32_t tid) {
        for (uint32_t k = tid; k < pixel_count; k += nt) {
            const uint32_t px = pixels != nullptr ? pixels[k] : k;
            g_libm_calls = 0;
            const PathOut o = trace_path(s, f, px);
            const float libm = float(g_libm_calls);
            rays[tid] += o.rays;
            shadows[tid] += o.shadows;
            const V3 planes[6] = {o.cam + o.dd + o.ds + o.id + o.is, o.cam, o.dd, o.ds, o.id, o.is};
            for (int p = 0; p < 6; ++p) {
                float* q = out_planes + (size_t(p) * pixel_count + k) * 4u;
                q[0] = planes[p].x; q[1] = planes[p].y; q[2] = planes[p].z; q[3] = p == 0 ? 1.f : 0.f;
            }
            std::memcpy(out_planes + (size_t(6) * pixel_count + k) * 4u, o.gb_pos, 16);
            std::memcpy(out_planes + (size_t(7) * pixel_count + k) * 4u, o.gb_nrm, 16);
            for (int j = 0; j < 6; ++j)
                std::memcpy(out_planes + (size_t(8 + j) * pixel_count + k) * 4u, o.surf + 4 * j, 16);
            float* lq = out_planes + (size_t(14) * pixel_count + k) * 4u;
            lq[0] = libm; lq[1] = lq[2] = lq[3] = 0.f;
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < nt; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    counts[0] = counts[1] = 0;
    for (uint32_t t = 0; t < nt; ++t) { counts[0] += rays[t]; counts[1] += shadows[t]; }
}

void oracle_render(const void* nodes, uint32_t node_count, const float* tri_v, const uint32_t* tri_key,
                   const float* tri_n, const uint32_t* tri_ids, const uint32_t* emitter, const float* materials,
                   uint32_t material_count, const void* lights, uint32_t light_count, const void* fixtures,
                   uint32_t fixture_count, uint32_t light_selection, float scene_radius, const void* frame,
                   const uint32_t* pixels, uint32_t pixel_count, uint32_t threads, float* out_planes,
                   uint64_t* counts) {
    oracle_render_env(nodes, node_count, tri_v, tri_key, tri_n, tri_ids, emitter, materials, material_count, lights,
                      light_count, fixtures, fixture_count, light_selection, scene_radius, frame, pixels, pixel_count,
                      threads, out_planes, counts, nullptr, 0, 0, nullptr);
}

// The environment importance tables the oracle builds: row entries (h),
// column entries (h x w; q, pmf, alias, item) and the integrated luminance.
void oracle_environment_tables(const float* env, uint32_t w, uint32_t h, float* rows_out, float* cols_out,
                               double* integrated) {
    Scene s{};
    s.env = env;
    s.env_w = w;
    s.env_h = h;
    build_environment(s);
    std::memcpy(rows_out, s.env_rows.data(), s.env_rows.size() * 16u);
    std::memcpy(cols_out, s.env_cols.data(), s.env_cols.size() * 16u);
    *integrated = s.env_integrated;
}

// One frame of ReSTIR DI on the CPU: initial RIS + temporal reuse for every
// pixel, then spatial reuse + winner visibility + resolve + direct publish +
// history publish (the GPU's k_restir_temporal / k_restir_spatial).  Inputs:
// the scene's leaf-ordered triangles (traversal), lights, the frame record,
// the ReSTIR parameters, this and the previous frame's GpuPrimarySurfaceV2
// planes and the previous frame's published reservoirs.  Outputs: temporal
// and published reservoirs, direct diffuse / specular (2 x pixels x 4
// floats), rejection reasons, and the 12 statistics counters.
void oracle_restir_frame(const void* nodes, uint32_t node_count, const float* tri_v, const uint32_t* tri_key,
                         const void* lights, uint32_t light_count, const void* fixtures, uint32_t fixture_count,
                         uint32_t light_selection, float scene_radius, const void* frame, const void* params,
                         const void* surf_cur, const void* surf_prev, const void* published_prev, void* temporal_out,
                         void* published_out, float* direct_out, uint32_t* reasons_out, uint32_t* stats_out,
                         uint32_t threads) {
    Scene s{nodes, node_count, tri_v, tri_key, nullptr, nullptr, nullptr, nullptr, 0,
            static_cast<const Light*>(lights), light_count, {}, {}, static_cast<const Fixture*>(fixtures), fixture_count};
    build_distribution(s, light_selection, scene_radius);
    Frame f;
    std::memcpy(&f, frame, sizeof(Frame));
    RParams rp;
    std::memcpy(&rp, params, sizeof(RParams));
    const Surf* cur = static_cast<const Surf*>(surf_cur);
    const Surf* prev = static_cast<const Surf*>(surf_prev);
    const Resv* pub_prev = static_cast<const Resv*>(published_prev);
    Resv* temporal = static_cast<Resv*>(temporal_out);
    Resv* published = static_cast<Resv*>(published_out);
    const uint32_t W = f.width, H = f.height, n = W * H;
    const V3 cam = v3(f.cam_pos[0], f.cam_pos[1], f.cam_pos[2]);
    const uint32_t nt = std::max(1u, threads);
    std::vector<std::array<uint32_t, 12>> st(nt);
    for (auto& a : st) a.fill(0u);
    auto run = [&](auto&& body) {
        std::vector<std::thread> pool;
        for (uint32_t t = 1; t < nt; ++t) pool.emplace_back([&, t] { for (uint32_t p = t; p < n; p += nt) body(p, st[t]); });
        for (uint32_t p = 0; p < n; p += nt) body(p, st[0]);
        for (auto& th : pool) th.join();
    };
    // Pass 1: initial RIS + temporal reuse.
    run([&](uint32_t p, std::array<uint32_t, 12>& cnt) {
        const Surf& sf = cur[p];
        const uint32_t C = rp.candidates;
        Resv r = empty_resv();
        uint32_t n_valid = 0;
        if (surf_valid(sf) && C != 0u) {
            uint32_t rs = rhash(p ^ rp.frame_lo ^ 0xa511e9b3u);
            const uint32_t stream = f.stream ^ 0x52335354u;
            for (uint32_t c = 0; c < C; ++c) {
                const uint32_t smp = f.sample * C + c;
                float u[5];
                for (uint32_t k = 0; k < 5; ++k) u[k] = counter_random(p, smp, k, stream, f.seed_lo, f.seed_hi);
                const LSmp ls = sample_light(s, xyz(sf.pos_depth), u);
                RSample ps = persistent(s, rp, ls, p * C + c);
                ps.source = {p, sf.identity.x, sf.identity.y, sf.identity.z};
                const Cand cd = make_cand(ps, sf, cam, rp.scene_gen, rp.candidate_source, 0u, p);
                if (cand_valid(cd, rp.scene_gen)) ++n_valid;
                update(r, cd, cand_weight(cd, rp.scene_gen), 1u, rrandom(rs), rp.scene_gen);
            }
        }
        clampm(r, rp.max_m);
        finalize(r);
        if (r.state.z & 2u) ++cnt[3];
        cnt[0] += C;
        cnt[1] += n_valid;
        cnt[2] += C - n_valid;
        r.state.y = 0u;
        r.h_surface = {sf.identity.x, sf.identity.y, sf.identity.z, 0u};
        r.h_scene = {rp.scene_gen, rp.light_gen, rp.camera_gen, rp.resolution_gen};
        r.h_frame = {rp.frame_lo, rp.frame_hi, rp.history_gen, 1u};
        r.h_reproj = {p, W, H, 0u};
        uint32_t rej = 0u;
        if (rp.history_enabled != 0u) {
            ++cnt[4];
            float pu = 0.f, pv = 0.f, pdepth = 0.f;
            const bool ok = sf.pos_depth.w > 0.f && prev_uv(rp, xyz(sf.pos_depth), pu, pv, pdepth);
            uint32_t prior = kInv;
            if (!ok) rej = 3u;
            else if (pu < 0.f || pv < 0.f || pu >= 1.f || pv >= 1.f) rej = 2u;
            else {
                const uint32_t px = std::min(uint32_t(pu * float(W)), W - 1u), py = std::min(uint32_t(pv * float(H)), H - 1u);
                prior = py * W + px;
            }
            Resv hs = empty_resv();
            if (prior < n) hs = pub_prev[prior];
            rej = temporal_gate(sf, prior < n ? &prev[prior] : nullptr, hs, rp, rej, pdepth);
            const uint32_t pl = hs.sel.metadata.w;
            if (rej == 0u) {
                RSample rm = hs.sel;
                if (rm.pos_dist.w < 1.0e29f) {
                    const V3 delta = xyz(rm.pos_dist) - xyz(sf.pos_depth);
                    const float dist = std::sqrt(dot(delta, delta));
                    if (std::isfinite(dist) && dist > 1.0e-6f) {
                        rm.pos_dist.w = dist;
                        const V3 dir = delta / dist;
                        rm.dir_pdf.x = dir.x; rm.dir_pdf.y = dir.y; rm.dir_pdf.z = dir.z;
                    } else {
                        rm.metadata.y &= ~1u;
                    }
                }
                rm.metadata.w = pl;
                Cand cd = make_cand(rm, sf, cam, rp.scene_gen, hs.prov.x, 1u, prior);
                cd.t.w = hs.weight.y;
                const float mw = cd.t.x * cd.t.z * hs.weight.y * float(hs.state.x);
                uint32_t rs2 = rhash(p ^ rp.frame_lo ^ 0x63d83595u);
                if (cand_valid(cd, rp.scene_gen) && std::isfinite(mw) && mw >= 0.f) {
                    update(r, cd, mw, hs.state.x, rrandom(rs2), rp.scene_gen);
                    r.state.z |= 4u;
                    r.state.y = std::min(hs.state.y + 1u, rp.max_age);
                    ++cnt[5];
                } else {
                    rej = 1u;
                }
            }
        }
        clampm(r, rp.max_m);
        finalize(r);
        r.state.w = rej;
        r.h_reproj.w = rej;
        reasons_out[p] = rej;
        temporal[p] = r;
    });
    // Pass 2: spatial reuse, winner visibility, resolve, publish.
    run([&](uint32_t p, std::array<uint32_t, 12>& cnt) {
        const Surf& sf = cur[p];
        const Resv& center = temporal[p];
        Resv r;
        if (rp.neighbors == 0u) {
            r = center;
        } else {
            r = empty_resv();
            uint32_t rs = rhash(p ^ rp.frame_lo ^ 0x9e3779b9u);
            uint32_t agg = reasons_out[p];
            Cand cc = make_cand(center.sel, sf, cam, rp.scene_gen, center.prov.x, center.prov.y, p);
            cc.t.w = center.weight.y;
            update(r, cc, cc.t.x * cc.t.z * center.weight.y * float(center.state.x), center.state.x, rrandom(rs),
                   rp.scene_gen);
            r.state.z |= center.state.z & (2u | 4u);
            for (uint32_t k = 0; k < rp.neighbors; ++k) {
                ++cnt[6];
                const uint32_t ni = neighbor(rp, W, H, p, k);
                if (ni >= n) { agg = 2u; continue; }
                const uint32_t rj = validate_pair(sf, cur[ni], rp);
                const Resv& nb = temporal[ni];
                if (rj != 0u || (nb.state.z & 1u) == 0u) { agg = rj != 0u ? rj : 1u; continue; }
                Cand cd = make_cand(nb.sel, sf, cam, rp.scene_gen, nb.prov.x, 2u, ni);
                cd.t.w = nb.weight.y;
                const float mw = cd.t.x * cd.t.z * nb.weight.y * float(nb.state.x);
                if (cand_valid(cd, rp.scene_gen) && std::isfinite(mw) && mw >= 0.f) {
                    update(r, cd, mw, nb.state.x, rrandom(rs), rp.scene_gen);
                    r.state.z |= 8u;
                    ++cnt[7];
                } else {
                    agg = 1u;
                }
            }
            clampm(r, rp.max_m);
            finalize(r);
            r.state.y = center.state.y;
            r.h_surface = center.h_surface;
            r.h_scene = center.h_scene;
            r.h_frame = center.h_frame;
            r.h_reproj = center.h_reproj;
            r.h_reproj.x = p;
            r.h_reproj.w = agg;
            r.state.w = agg;
            reasons_out[p] = agg;
        }
        // Binary visibility of the selected sample from a primary surface
        // (RestirMakeVisibilityRayV3 + RestirBinaryVisibilityV3).
        auto visible_from = [&](const Surf& q, bool& traced) {
            traced = false;
            if (!surf_valid(q)) return false;
            const V3 nrm = normalize(xyz(q.gn_rough));
            V3 dir = normalize(xyz(r.sel.dir_pdf));
            float maxd = 1.0e30f;
            if (std::isfinite(r.sel.pos_dist.w) && r.sel.pos_dist.w > 0.f) {
                const V3 disp = xyz(r.sel.pos_dist) - xyz(q.pos_depth);
                const float dist = std::sqrt(dot(disp, disp));
                if (dist > 2.0e-4f) {
                    dir = disp / dist;
                    maxd = std::fmax(dist - 1.0e-4f, 1.0e-4f);
                }
            }
            const TraceResult h = trace_flat(s.nodes, s.node_count, s.tri_v, s.tri_key, xyz(q.pos_depth) + nrm * 1.0e-4f,
                                             1.0e-4f, dir, maxd, true, true, kInv, kInv, s.alpha);
            traced = true;
            return h.status == 0u && h.tri == kInv;
        };
        // Reference correction (RestirReferenceResolveV3.comp.hlsl): the
        // winner re-weighted with visibility at the centre and every
        // neighbour it could have come from.
        if (rp.estimator == 1u && (r.state.z & 1u) != 0u) {
            float denom = 0.f, sel_t = 0.f, cur_t = 0.f;
            for (uint32_t k = 0; k <= rp.neighbors; ++k) {
                const uint32_t src = k == 0u ? p : neighbor(rp, W, H, p, k - 1u);
                if (src >= n) continue;
                bool traced;
                const float vis = visible_from(cur[src], traced) ? 1.f : 0.f;
                V3 dif, spec;
                const float target = unshadowed(r.sel, cur[src], cam, rp.scene_gen, dif, spec);
                const uint32_t m_src = std::max(temporal[src].state.x, 1u);
                denom += float(m_src) * target * vis;
                if (src == p) cur_t = target;
                if (src == r.prov.z) sel_t = target * vis;
                if (traced) ++cnt[8];
                ++cnt[9];
                if (vis > 0.f) ++cnt[10];
            }
            const float nd = cur_t * denom;
            r.weight.y = nd > 0.f ? r.weight.x * sel_t / nd : 0.f;
            r.terms.w = r.weight.y;
            r.state.z |= 16u;
            if (!(r.weight.y > 0.f) || !std::isfinite(r.weight.y)) r.state.z &= ~1u;
        }
        const bool valid = (r.state.z & 1u) != 0u, dup = (r.state.z & 32u) != 0u;
        bool visible = false;
        if (valid && !dup) {
            bool traced;
            visible = visible_from(sf, traced);
            if (traced) ++cnt[8];
        }
        if (valid && !dup) {
            const float vis = visible ? 1.f : 0.f;
            const float fw = r.weight.y * vis;
            const bool fr = std::isfinite(vis) && vis >= 0.f && vis <= 1.f && std::isfinite(fw) && fw >= 0.f;
            const bool ok = fr && vis > 0.f;
            r.state.z |= 32u;
            r.terms.w = fr ? fw : 0.f;
            if (!fr) { r.state.z &= ~1u; r.state.w = 1u; r.h_reproj.w = 1u; }
            if (ok) r.state.z |= 64u; else r.state.z &= ~64u;
            ++cnt[9];
            if (ok) ++cnt[10];
        }
        if (dup) ++cnt[11];
        V3 dif = splat(0.f), spec = splat(0.f);
        if ((r.state.z & 1u) && (r.state.z & 32u) && (r.state.z & 64u)) {
            unshadowed(r.sel, sf, cam, rp.scene_gen, dif, spec);
            dif = dif * r.terms.w;
            spec = spec * r.terms.w;
        }
        std::memcpy(direct_out + size_t(p) * 4u, &dif, 12);
        direct_out[size_t(p) * 4u + 3] = 0.f;
        std::memcpy(direct_out + (size_t(n) + p) * 4u, &spec, 12);
        direct_out[(size_t(n) + p) * 4u + 3] = 0.f;
        r.h_surface = {sf.identity.x, sf.identity.y, sf.identity.z, 0u};
        r.h_scene.x = rp.scene_gen;
        r.h_scene.y = rp.light_gen;
        const uint32_t hf = (r.state.z & 1u) && (r.state.z & 32u) ? 1u : 2u;
        r.h_frame = {rp.frame_lo, rp.frame_hi, rp.history_gen, hf};
        r.h_reproj = {p, W, H, r.h_reproj.w};
        published[p] = r;
    });
    for (uint32_t k = 0; k < 12; ++k) {
        stats_out[k] = 0;
        for (uint32_t t = 0; t < nt; ++t) stats_out[k] += st[t][k];
    }
}

// Initial RIS over explicit candidate terms (target, proposal pdf, support,
// correction) with explicit random numbers: the float reservoir update of
// RestirProductionV3.hlsli:372-447 on synthetic valid light samples.  Writes
// (weightSum, W) and M; returns the selected candidate or -1.
int oracle_restir_ris(const float* terms, const float* u, uint32_t n, uint32_t max_m, float* out, uint32_t* out_m) {
    Resv r = empty_resv();
    for (uint32_t i = 0; i < n; ++i) {
        Cand c;
        std::memset(&c, 0, sizeof(c));
        c.s.identity = {i, i, 0u, 0u};
        c.s.generation = {1u, 1u, 0u, 0u};
        c.s.metadata = {3u, 1u, 0u, i};
        c.s.dir_pdf = {0.f, 0.f, 1.f, terms[4 * i + 1]};
        c.s.rad_pmf = {1.f, 1.f, 1.f, 1.f};
        c.t = {terms[4 * i], terms[4 * i + 1], terms[4 * i + 2], terms[4 * i + 3]};
        update(r, c, cand_weight(c, 1u), 1u, u[i], 1u);
    }
    clampm(r, max_m);
    finalize(r);
    out[0] = r.weight.x;
    out[1] = r.weight.y;
    *out_m = r.state.x;
    return (r.state.z & 1u) ? int(r.sel.identity.x) : -1;
}

// The spatial pass's neighbour gate (RestirSpatialV3.comp.hlsl:12-112): the
// surface pair, then the neighbour reservoir's valid flag (1).  `rparams` is
// one frame's ReSTIR block (thresholds read from it).
void oracle_restir_spatial_gate(const void* center, const void* neighbor, const uint32_t* neighbor_valid, uint32_t n,
                                const void* rparams, uint32_t* out) {
    const Surf* c = static_cast<const Surf*>(center);
    const Surf* b = static_cast<const Surf*>(neighbor);
    const RParams& rp = *static_cast<const RParams*>(rparams);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t rj = validate_pair(c[i], b[i], rp);
        if (rj == 0u && neighbor_valid[i] == 0u) rj = 1u;
        out[i] = rj;
    }
}

// The temporal pass's history gate (temporal_gate) over arrays: per case the
// current surface, the prior pixel's previous surface, the history
// reservoir, the reprojection result (0, 2 outside, 3 invalid) and the
// reprojected depth; a prior surface with identity.w bit 31 set stands for a
// prior pixel outside the frame.
void oracle_restir_temporal_gate(const void* current, const void* history_surface, const void* history, const uint32_t* reproj,
                                 const float* reprojected_depth, uint32_t n, const void* rparams, uint32_t* out) {
    const Surf* c = static_cast<const Surf*>(current);
    const Surf* h = static_cast<const Surf*>(history_surface);
    const Resv* r = static_cast<const Resv*>(history);
    const RParams& rp = *static_cast<const RParams*>(rparams);
    for (uint32_t i = 0; i < n; ++i)
        out[i] = temporal_gate(c[i], (h[i].identity.w >> 31) ? nullptr : &h[i], r[i], rp, reproj[i], reprojected_depth[i]);
}

// Philox4x32-10 sample (for pinning against the reference's CounterRandomFloat).
float oracle_counter_random(uint32_t pixel, uint32_t sample, uint32_t dim, uint32_t stream, uint32_t seed_lo,
                            uint32_t seed_hi) {
    return counter_random(pixel, sample, dim, stream, seed_lo, seed_hi);
}

// Light alias table of the oracle (entries q, pmf, alias, item).
int oracle_light_distribution(const void* lights, uint32_t n, uint32_t selection, float scene_radius, float* out) {
    Scene s{};
    s.lights = static_cast<const Light*>(lights);
    s.light_count = n;
    build_distribution(s, selection, scene_radius);
    std::memcpy(out, s.alias.data(), s.alias.size() * 16u);
    return int(s.alias.size());
}

// BSDF probe: for each 160-byte query (context, parameters, wo, wi, random
// triple; the layout of re_bsdf_query) evaluates the BSDF at (wo, wi) and
// samples it with the random triple, writing a 128-byte result (the layout of
// re_bsdf_probe_result).  The CPU counterpart of the reference's readback
// probe resources/shaders/integrators/pbr_sampling_probe.hlsl:9-102.
void oracle_bsdf_probe(const float* queries, uint32_t n, float* results) {
    for (uint32_t i = 0; i < n; ++i) {
        const float* q = queries + size_t(i) * 40u;
        auto u32 = [&](int k) { uint32_t v; std::memcpy(&v, q + k, 4); return v; };
        const Ctx c{v3(q[0], q[1], q[2]), q[3], v3(q[4], q[5], q[6]), q[7], v3(q[8], q[9], q[10]), u32(11)};
        const Params p{v3(q[12], q[13], q[14]), q[15], v3(q[16], q[17], q[18]), q[19], v3(q[20], q[21], q[22]),
                       q[23], v3(q[24], q[25], q[26]), u32(27), u32(31), u32(35)};
        const V3 wo = v3(q[28], q[29], q[30]), wi = v3(q[32], q[33], q[34]), u = v3(q[36], q[37], q[38]);
        const Eval e = evaluate(c, p, wo, wi);
        const Smp sm = sample_bsdf(c, p, wo, u);
        float pdf_at = 0.f;
        if (sm.valid && !sm.delta) {
            const Eval e2 = evaluate(c, p, wo, sm.dir);
            pdf_at = (e2.valid && e2.measure == 1) ? e2.pdf : 0.f;
        }
        float* o = results + size_t(i) * 32u;
        auto put = [&](int k, V3 v, float w) { o[k] = v.x; o[k + 1] = v.y; o[k + 2] = v.z; o[k + 3] = w; };
        auto putu = [&](int k, V3 v, uint32_t w) { put(k, v, 0.f); std::memcpy(o + k + 3, &w, 4); };
        put(0, e.value, e.pdf);
        putu(4, e.diff, e.measure);
        putu(8, e.spec, e.lobe);
        put(12, sm.dir, sm.pdf);
        put(16, sm.value, sm.eta);
        putu(20, sm.diff, sm.measure);
        putu(24, sm.spec, sm.lobe);
        const uint32_t flags4[3] = {e.valid ? 1u : 0u, sm.delta ? 1u : 0u, sm.valid ? 1u : 0u};
        std::memcpy(o + 28, flags4, 12);
        o[31] = pdf_at;
    }
}

// sample_vndf on local outgoing directions (3 floats each), alpha and two
// random numbers per query; out: normal xyz + 1/0 validity.
void oracle_ggx_vndf(const float* wo, const float* alpha, const float* u, uint32_t n, float* out) {
    for (uint32_t i = 0; i < n; ++i) {
        V3 m = splat(0);
        const bool ok = sample_vndf(v3(wo[i * 3], wo[i * 3 + 1], wo[i * 3 + 2]), alpha[i], u[i * 2], u[i * 2 + 1], m);
        out[i * 4 + 0] = m.x;
        out[i * 4 + 1] = m.y;
        out[i * 4 + 2] = m.z;
        out[i * 4 + 3] = ok ? 1.f : 0.f;
    }
}

}  // extern "C"
