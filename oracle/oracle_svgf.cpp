// TEST INFRASTRUCTURE ONLY -- CPU restatement of the SVGF / A-Trous
// reconstruction (RenderingEngine reconstruction/src/Svgf.cpp,
// reconstruction/src/History.cpp, reconstruction/src/MotionVectors.cpp) used
// as the checker of the GPU kernels.  Pinned against the reference's own
// SvgfReconstruction (compiled from its sources into oracle/_ref) by
// tests/test_oracle_svgf.py.
//
// Data are kept as flat planes (one float array per channel group) rather
// than the reference's pixel structs; every arithmetic expression keeps the
// reference's operand order so that, compiled without contraction, the
// results are bit-identical to the reference's.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "oracle_common.h"

namespace {

using oracle::V3;
using oracle::finite3;

// Flat records of the C ABI (include/re_b200.h): re_gbuffer_pixel,
// re_signal_pixel, re_svgf_config.
struct GbPix {
    float depth;
    float n[3];
    float dalb[3];
    float salb[3];
    float epd;
    float motion[2];
    uint32_t mat, obj, flags;
};
static_assert(sizeof(GbPix) == 64, "re_gbuffer_pixel");
struct SigPix {
    float d[3];
    float s[3];
};
struct Config {
    float rel_depth, abs_depth, normal_cos;
    uint32_t require_mat, require_obj;
    uint32_t max_history;
    float min_color_alpha, min_moments_alpha;
    uint32_t short_history, radius;
    float min_variance;
    uint32_t iterations;
    float phi_depth, phi_normal, phi_luminance;
    float min_albedo;
    uint32_t demod_specular;
};
struct Outputs {
    float* raw;       // 6 floats per pixel
    float* temporal;
    float* atrous;
    float* svgf;
    uint32_t* history_length;
    float* moments;   // 2 floats per pixel
    float* variance;
    uint32_t* accepted;
    uint32_t* reject;
};

enum : uint32_t {
    NoHistory = 1u << 0, Reset = 1u << 1, ScreenBounds = 1u << 2, InvalidCurrent = 1u << 3,
    InvalidHistory = 1u << 4, NonFinite = 1u << 5, Depth = 1u << 6, Normal = 1u << 7,
    MaterialId = 1u << 8, ObjectId = 1u << 9, InvalidMotion = 1u << 10,
};

V3 vec(const float* p) { return {p[0], p[1], p[2]}; }
float lum_of(V3 d, V3 s) {  // Math.hpp:90-92 of Combined (Svgf.cpp:14-16)
    const V3 c = d + s;
    return 0.2126F * c.x + 0.7152F * c.y + 0.0722F * c.z;
}
V3 unit(V3 v) {  // Math.hpp:78-81
    const float len = std::sqrt(oracle::dot(v, v));
    return len > 1.0e-20F ? v / len : V3{0.0F, 0.0F, 1.0F};
}
bool usable(V3 n) { return finite3(n) && oracle::dot(n, n) > 1.0e-20F; }
float mix(float a, float b, float t) { return a * (1.0F - t) + b * t; }
V3 mix3(V3 a, V3 b, float t) { return a * (1.0F - t) + b * t; }
V3 div3(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }

bool gvalid(const GbPix& g) { return (g.flags & 1u) != 0u; }
bool gmotion(const GbPix& g) { return (g.flags & 2u) != 0u; }
bool geometry_ok(const GbPix& g) {  // Svgf.cpp:37-40
    return std::isfinite(g.depth) && g.depth >= 0.0F && usable(vec(g.n));
}
V3 albedo_floor(const float* a, float minimum) {  // Svgf.cpp:42-50
    const float m = (std::isfinite(minimum) && minimum > 0.0F) ? minimum : 1.0e-3F;
    auto ch = [m](float v) { return std::isfinite(v) ? std::max(v, m) : m; };
    return {ch(a[0]), ch(a[1]), ch(a[2])};
}

// One history generation as planes.
struct Generation {
    std::vector<float> dd, ds, moments, variance, depth, normal;
    std::vector<uint32_t> length, mat, obj;
    std::vector<uint8_t> valid;
    bool published = false;
    uint64_t frame = ~0ull;
    void clear(size_t n) {
        dd.assign(3 * n, 0.0F);
        ds.assign(3 * n, 0.0F);
        moments.assign(2 * n, 0.0F);
        variance.assign(n, 0.0F);
        depth.assign(n, 0.0F);
        normal.assign(3 * n, 0.0F);
        for (size_t i = 0; i < n; ++i) normal[3 * i + 2] = 1.0F;
        length.assign(n, 0u);
        mat.assign(n, 0xffffffffu);
        obj.assign(n, 0xffffffffu);
        valid.assign(n, 0u);
        published = false;
        frame = ~0ull;
    }
};

struct Svgf {
    Config cfg{};
    bool changed = false;
    uint32_t w = 0, h = 0, flights = 1;
    std::vector<Generation> gens;

    size_t slot(uint64_t f) const {  // History.cpp:22-29
        return size_t(((f / flights) & 1ull) * flights + f % flights);
    }
    void reset(uint32_t nw, uint32_t nh) {  // History.cpp:74-84
        w = nw;
        h = nh;
        for (auto& g : gens) g.clear(size_t(w) * h);
    }
};

bool config_ok(const Config& c) {  // Svgf.cpp:52-80
    auto f = [](float v) { return std::isfinite(v); };
    if (!f(c.rel_depth) || c.rel_depth < 0.0F || !f(c.abs_depth) || c.abs_depth < 0.0F || !f(c.normal_cos) ||
        c.normal_cos < -1.0F || c.normal_cos > 1.0F)
        return false;
    if (c.max_history == 0u || !f(c.min_color_alpha) || c.min_color_alpha < 0.0F || c.min_color_alpha > 1.0F ||
        !f(c.min_moments_alpha) || c.min_moments_alpha < 0.0F || c.min_moments_alpha > 1.0F)
        return false;
    if (c.short_history == 0u || c.radius > 64u || !f(c.min_variance) || c.min_variance <= 0.0F) return false;
    if (c.iterations > 16u || !f(c.phi_depth) || c.phi_depth <= 0.0F || !f(c.phi_normal) || c.phi_normal < 0.0F ||
        !f(c.phi_luminance) || c.phi_luminance <= 0.0F || !f(c.min_albedo) || c.min_albedo <= 0.0F)
        return false;
    return true;
}

uint32_t current_reasons(const GbPix& g, bool reset) {  // Svgf.cpp:82-102
    uint32_t r = 0u;
    if (reset) r |= Reset;
    if (!gvalid(g) || !geometry_ok(g)) r |= InvalidCurrent;
    if (!gmotion(g)) r |= InvalidMotion;
    if (!std::isfinite(g.motion[0]) || !std::isfinite(g.motion[1]) || !std::isfinite(g.depth) ||
        !finite3(vec(g.n)) || !std::isfinite(g.epd))
        r |= NonFinite;
    if (gmotion(g) && g.epd < 0.0F) r |= InvalidMotion;
    return r;
}

// ValidateHistory (Svgf.cpp:343-391) against pixel k of generation `p`.
uint32_t history_reasons(const GbPix& cur, const Generation& p, size_t k, const Config& c) {
    uint32_t r = current_reasons(cur, false);
    if (!p.valid[k]) return r | InvalidHistory;
    const V3 pdd = vec(&p.dd[3 * k]), pds = vec(&p.ds[3 * k]), pn = vec(&p.normal[3 * k]);
    if (!std::isfinite(p.depth[k]) || p.depth[k] < 0.0F || !usable(pn) || !finite3(pdd) || !finite3(pds) ||
        !std::isfinite(p.moments[2 * k]) || !std::isfinite(p.moments[2 * k + 1]) || !std::isfinite(p.variance[k]) ||
        p.variance[k] < 0.0F)
        r |= NonFinite;
    if (p.length[k] == 0u || p.length[k] > std::max(c.max_history, 1u)) r |= InvalidHistory;
    const float tol = c.abs_depth + c.rel_depth * std::max(std::abs(cur.epd), std::abs(p.depth[k]));
    if (std::abs(cur.epd - p.depth[k]) > tol) r |= Depth;
    if (oracle::dot(unit(vec(cur.n)), unit(pn)) < c.normal_cos) r |= Normal;
    if (c.require_mat && cur.mat != p.mat[k]) r |= MaterialId;
    if (c.require_obj && cur.obj != p.obj[k]) r |= ObjectId;
    return r;
}

struct Fetched {
    V3 dd{}, ds{};
    float m1 = 0.0F, m2 = 0.0F;
    uint32_t length = 0u;
    uint32_t reasons = 0u;
    bool ok = false;
};

// ReprojectHistory (Svgf.cpp:128-244).
Fetched fetch_history(uint32_t x, uint32_t y, const GbPix& cur, uint32_t W, uint32_t H, const Generation* p,
                      const Config& c, bool reset) {
    Fetched f;
    uint32_t base = current_reasons(cur, reset);
    const float u = (float(x) + 0.5F) / float(W) + cur.motion[0];
    const float v = (float(y) + 0.5F) / float(H) + cur.motion[1];
    if (!std::isfinite(u) || !std::isfinite(v) || u < 0.0F || v < 0.0F || u >= 1.0F || v >= 1.0F)
        base |= ScreenBounds;
    if (p == nullptr) base |= NoHistory;
    if (base != 0u) {
        f.reasons = base;
        return f;
    }
    auto inside = [&](int64_t px, int64_t py) { return px >= 0 && py >= 0 && px < int64_t(W) && py < int64_t(H); };
    const float fxs = u * float(W) - 0.5F, fys = v * float(H) - 0.5F;
    const int64_t x0 = int64_t(std::floor(fxs)), y0 = int64_t(std::floor(fys));
    const float ax = fxs - float(x0), ay = fys - float(y0);
    float total = 0.0F, lengths = 0.0F, m1 = 0.0F, m2 = 0.0F;
    V3 dd{0.0F, 0.0F, 0.0F}, ds{0.0F, 0.0F, 0.0F};
    uint32_t failed = 0u;
    for (int j = 0; j < 2; ++j) {
        for (int i = 0; i < 2; ++i) {
            const float wgt = (i == 0 ? 1.0F - ax : ax) * (j == 0 ? 1.0F - ay : ay);
            if (wgt <= 0.0F) continue;
            const int64_t px = x0 + i, py = y0 + j;
            if (!inside(px, py)) {
                failed |= ScreenBounds;
                continue;
            }
            const size_t k = size_t(py) * W + size_t(px);
            const uint32_t r = history_reasons(cur, *p, k, c);
            if (r != 0u) {
                failed |= r;
                continue;
            }
            dd = dd + vec(&p->dd[3 * k]) * wgt;
            ds = ds + vec(&p->ds[3 * k]) * wgt;
            m1 += p->moments[2 * k] * wgt;
            m2 += p->moments[2 * k + 1] * wgt;
            lengths += float(p->length[k]) * wgt;
            total += wgt;
        }
    }
    if (total > 0.0F) {
        const float inv = 1.0F / total;
        f.dd = dd * inv;
        f.ds = ds * inv;
        f.m1 = m1 * inv;
        f.m2 = m2 * inv;
        f.length = uint32_t(lengths * inv + 0.5F);
        f.ok = true;
        return f;
    }
    const int64_t cx = int64_t(std::floor(u * float(W))), cy = int64_t(std::floor(v * float(H)));
    float nearest = std::numeric_limits<float>::max();
    int64_t pick = -1;
    for (int64_t py = cy - 1; py <= cy + 1; ++py) {
        for (int64_t px = cx - 1; px <= cx + 1; ++px) {
            if (!inside(px, py)) {
                failed |= ScreenBounds;
                continue;
            }
            const size_t k = size_t(py) * W + size_t(px);
            const uint32_t r = history_reasons(cur, *p, k, c);
            if (r != 0u) {
                failed |= r;
                continue;
            }
            const float ex = (float(px) + 0.5F) - u * float(W);
            const float ey = (float(py) + 0.5F) - v * float(H);
            const float d2 = ex * ex + ey * ey;
            if (d2 < nearest) {
                nearest = d2;
                pick = int64_t(k);
            }
        }
    }
    if (pick >= 0) {
        const size_t k = size_t(pick);
        f.dd = vec(&p->dd[3 * k]);
        f.ds = vec(&p->ds[3 * k]);
        f.m1 = p->moments[2 * k];
        f.m2 = p->moments[2 * k + 1];
        f.length = p->length[k];
        f.ok = true;
        return f;
    }
    f.reasons = failed == 0u ? NoHistory : failed;
    return f;
}

// Per-pixel filter inputs shared by the bootstrap and the A-Trous passes.
struct Surface {
    bool filterable;
    float depth;
    V3 n;  // normalised
    uint32_t mat, obj;
};

std::vector<Surface> surfaces(const GbPix* gb, size_t n) {
    std::vector<Surface> s(n);
    for (size_t i = 0; i < n; ++i) {
        s[i].filterable = gvalid(gb[i]) && geometry_ok(gb[i]);
        s[i].depth = gb[i].depth;
        s[i].n = unit(vec(gb[i].n));
        s[i].mat = gb[i].mat;
        s[i].obj = gb[i].obj;
    }
    return s;
}

// BootstrapVariance (Svgf.cpp:584-661); `sig` is 6 floats per pixel.
std::vector<float> bootstrap(const std::vector<float>& sig, const std::vector<Surface>& sf, uint32_t W, uint32_t H,
                             const std::vector<uint32_t>& lengths, const std::vector<float>& temporal,
                             const Config& c) {
    std::vector<float> out(size_t(W) * H);
    const int r = int(c.radius);
    for (uint32_t y = 0; y < H; ++y) {
        for (uint32_t x = 0; x < W; ++x) {
            const size_t i = size_t(y) * W + x;
            const Surface& s0 = sf[i];
            if (!s0.filterable) {
                out[i] = c.min_variance;
                continue;
            }
            float tw = 0.0F, e1 = 0.0F, e2 = 0.0F;
            for (int dy = -r; dy <= r; ++dy) {
                for (int dx = -r; dx <= r; ++dx) {
                    const int64_t px = int64_t(x) + dx, py = int64_t(y) + dy;
                    if (px < 0 || py < 0 || px >= int64_t(W) || py >= int64_t(H)) continue;
                    const size_t j = size_t(py) * W + size_t(px);
                    const Surface& s1 = sf[j];
                    const V3 d = vec(&sig[6 * j]), sp = vec(&sig[6 * j + 3]);
                    if (!s1.filterable || !finite3(d) || !finite3(sp) || s1.mat != s0.mat || s1.obj != s0.obj)
                        continue;
                    const float scale = std::max(0.01F, std::abs(s0.depth) * 0.02F);
                    const float wz = std::exp(-std::abs(s1.depth - s0.depth) / scale);
                    const float wn = std::pow(std::clamp(oracle::dot(s0.n, s1.n), 0.0F, 1.0F), 32.0F);
                    const float wgt = wz * wn;
                    const float l = lum_of(d, sp);
                    const float l2 = l * l;
                    if (!std::isfinite(wgt) || wgt <= 0.0F || !std::isfinite(l) || !std::isfinite(l2)) continue;
                    e1 += l * wgt;
                    e2 += l2 * wgt;
                    tw += wgt;
                }
            }
            const float spatial = (tw > 0.0F && std::isfinite(tw) && std::isfinite(e1) && std::isfinite(e2))
                                      ? std::max(e2 / tw - (e1 / tw) * (e1 / tw), 0.0F)
                                      : 0.0F;
            const float blend =
                std::clamp(float(lengths[i]) / float(std::max(c.short_history, 1u)), 0.0F, 1.0F);
            const float tv = (std::isfinite(temporal[i]) && temporal[i] >= 0.0F) ? temporal[i] : spatial;
            const float b = mix(spatial, tv, blend);
            out[i] = std::isfinite(b) ? std::max(b, c.min_variance) : c.min_variance;
        }
    }
    return out;
}

// FilterATrous (Svgf.cpp:663-752) with EdgeWeight (Svgf.cpp:246-272).
std::vector<float> atrous(std::vector<float> sig, std::vector<float> var, const std::vector<Surface>& sf, uint32_t W,
                          uint32_t H, const Config& c) {
    static const float taps[5] = {1.0F, 4.0F, 6.0F, 4.0F, 1.0F};
    std::vector<float> nsig(sig.size()), nvar(var.size());
    for (uint32_t it = 0; it < c.iterations; ++it) {
        const uint32_t step = 1u << std::min(it, 15u);
        for (uint32_t y = 0; y < H; ++y) {
            for (uint32_t x = 0; x < W; ++x) {
                const size_t i = size_t(y) * W + x;
                V3 cd = vec(&sig[6 * i]), cs = vec(&sig[6 * i + 3]);
                if (!finite3(cd) || !finite3(cs)) cd = cs = V3{0.0F, 0.0F, 0.0F};
                const float cv = (std::isfinite(var[i]) && var[i] >= 0.0F) ? std::max(var[i], c.min_variance)
                                                                           : c.min_variance;
                const Surface& s0 = sf[i];
                V3 od = cd, os = cs;
                float ov = cv;
                if (s0.filterable) {
                    const float cl = lum_of(cd, cs);
                    V3 ad{0.0F, 0.0F, 0.0F}, as{0.0F, 0.0F, 0.0F};
                    float tw = 0.0F, tv = 0.0F;
                    for (int ky = -2; ky <= 2; ++ky) {
                        for (int kx = -2; kx <= 2; ++kx) {
                            const int64_t px = int64_t(x) + int64_t(kx) * step;
                            const int64_t py = int64_t(y) + int64_t(ky) * step;
                            if (px < 0 || py < 0 || px >= int64_t(W) || py >= int64_t(H)) continue;
                            const size_t j = size_t(py) * W + size_t(px);
                            const V3 sd = vec(&sig[6 * j]), ss = vec(&sig[6 * j + 3]);
                            const float sv = var[j];
                            if (!finite3(sd) || !finite3(ss) || !std::isfinite(sv) || sv < 0.0F) continue;
                            const float sl = lum_of(sd, ss);
                            const Surface& s1 = sf[j];
                            float edge = 0.0F;
                            if (s1.filterable && std::isfinite(cl) && std::isfinite(sl) && s0.mat == s1.mat &&
                                s0.obj == s1.obj) {
                                const float scale = std::max(0.01F, std::abs(s0.depth) * 0.01F);
                                const float den = std::max(c.phi_depth * scale * float(step), 1.0e-6F);
                                const float wz = std::exp(-std::abs(s1.depth - s0.depth) / den);
                                const float wn =
                                    std::pow(std::clamp(oracle::dot(s0.n, s1.n), 0.0F, 1.0F), c.phi_normal);
                                const float lden = std::max(c.phi_luminance * std::sqrt(std::max(cv, 0.0F)), 1.0e-4F);
                                const float wl = std::exp(-std::abs(sl - cl) / lden);
                                edge = wz * wn * wl;
                                if (!std::isfinite(edge)) edge = 0.0F;
                            }
                            const float wgt = taps[kx + 2] * taps[ky + 2] * edge;
                            if (!std::isfinite(wgt) || wgt <= 0.0F) continue;
                            ad = ad + sd * wgt;
                            as = as + ss * wgt;
                            tv += sv * wgt * wgt;
                            tw += wgt;
                        }
                    }
                    const bool ok = tw > 0.0F && std::isfinite(tw) && std::isfinite(tv) && finite3(ad) && finite3(as);
                    od = ok ? ad / tw : cd;
                    os = ok ? as / tw : cs;
                    if (!finite3(od) || !finite3(os)) {
                        od = cd;
                        os = cs;
                    }
                    const float fv = ok ? tv / (tw * tw) : cv;
                    ov = std::isfinite(fv) ? std::max(fv, c.min_variance) : cv;
                }
                std::memcpy(&nsig[6 * i], &od, 12);
                std::memcpy(&nsig[6 * i + 3], &os, 12);
                nvar[i] = ov;
            }
        }
        sig.swap(nsig);
        var.swap(nvar);
    }
    return sig;
}

void remodulate_into(float* dst, const float* sig, const GbPix& g, const Config& c) {
    const V3 da = albedo_floor(g.dalb, c.min_albedo), sa = albedo_floor(g.salb, c.min_albedo);
    const V3 d = vec(sig) * da;
    const V3 s = c.demod_specular ? vec(sig + 3) * sa : vec(sig + 3);
    std::memcpy(dst, &d, 12);
    std::memcpy(dst + 3, &s, 12);
}

// SvgfReconstruction::Process (Svgf.cpp:408-582).
int process(Svgf& sv, const GbPix* gb, const SigPix* raw, uint32_t W, uint32_t H, uint64_t frame, uint32_t trigger,
            const Outputs& out) {
    const Config& c = sv.cfg;
    if (W != sv.w || H != sv.h) trigger |= 1u << 2;  // ResetTrigger::Resolution
    if (sv.changed) trigger |= 1u << 6;             // ResetTrigger::ReconstructionParameters
    const bool reset = trigger != 0u;
    if (reset) sv.reset(W, H);  // HistoryPingPong::BeginWrite
    const size_t n = size_t(W) * H;
    Generation& gw = sv.gens[sv.slot(frame)];
    gw.clear(n);
    const Generation* gp = nullptr;
    if (!reset && frame != 0ull) {
        const Generation& cand = sv.gens[sv.slot(frame - 1ull)];
        if (cand.published && cand.frame == frame - 1ull) gp = &cand;
    }
    std::vector<float> cur_sig(6 * n), tmp_sig(6 * n), tvar(n);
    std::vector<uint32_t> lengths(n);
    for (uint32_t y = 0; y < H; ++y) {
        for (uint32_t x = 0; x < W; ++x) {
            const size_t i = size_t(y) * W + x;
            const GbPix& g = gb[i];
            std::memcpy(&out.raw[6 * i], &raw[i], 24);
            const V3 rd = vec(raw[i].d), rs = vec(raw[i].s);
            const V3 da = albedo_floor(g.dalb, c.min_albedo), sa = albedo_floor(g.salb, c.min_albedo);
            const V3 dd = div3(rd, da);
            const V3 ds = c.demod_specular ? div3(rs, sa) : rs;
            const float l0 = lum_of(dd, ds), l0sq = l0 * l0;
            const bool fin = finite3(rd) && finite3(rs) && finite3(dd) && finite3(ds) && std::isfinite(l0) &&
                             std::isfinite(l0sq);
            const V3 zero{0.0F, 0.0F, 0.0F};
            const V3 sd = fin ? dd : zero, ss = fin ? ds : zero;
            const float l = fin ? l0 : 0.0F, lsq = fin ? l0sq : 0.0F;
            std::memcpy(&cur_sig[6 * i], &sd, 12);
            std::memcpy(&cur_sig[6 * i + 3], &ss, 12);

            const Fetched hist = fetch_history(x, y, g, W, H, gp, c, reset);
            uint32_t why = hist.reasons | (fin ? 0u : uint32_t(NonFinite));
            bool took = hist.ok && why == 0u;
            V3 ad = sd, as = ss;
            float m1 = l, m2 = lsq;
            uint32_t len = 1u;
            if (took) {
                const uint32_t cap = std::max(c.max_history, 1u);
                len = std::min(hist.length, cap - 1u) + 1u;
                const float inv = 1.0F / float(len);
                const float ca = std::max(c.min_color_alpha, inv), ma = std::max(c.min_moments_alpha, inv);
                ad = mix3(hist.dd, sd, ca);
                as = mix3(hist.ds, ss, ca);
                m1 = mix(hist.m1, l, ma);
                m2 = mix(hist.m2, lsq, ma);
            }
            float rv = m2 - m1 * m1;
            if (!finite3(ad) || !finite3(as) || !std::isfinite(m1) || !std::isfinite(m2) || !std::isfinite(rv)) {
                why |= NonFinite;
                took = false;
                ad = sd;
                as = ss;
                m1 = l;
                m2 = lsq;
                len = 1u;
                rv = m2 - m1 * m1;
            }
            const float var = std::max(rv, 0.0F);
            std::memcpy(&gw.dd[3 * i], &ad, 12);
            std::memcpy(&gw.ds[3 * i], &as, 12);
            gw.moments[2 * i] = m1;
            gw.moments[2 * i + 1] = m2;
            gw.variance[i] = var;
            gw.depth[i] = (std::isfinite(g.depth) && g.depth >= 0.0F) ? g.depth : 0.0F;
            const V3 nn = usable(vec(g.n)) ? unit(vec(g.n)) : V3{0.0F, 0.0F, 1.0F};
            std::memcpy(&gw.normal[3 * i], &nn, 12);
            gw.length[i] = len;
            gw.mat[i] = g.mat;
            gw.obj[i] = g.obj;
            gw.valid[i] = fin && gvalid(g) && geometry_ok(g) && finite3(ad) && finite3(as) && std::isfinite(m1) &&
                          std::isfinite(m2) && std::isfinite(var);
            std::memcpy(&tmp_sig[6 * i], &ad, 12);
            std::memcpy(&tmp_sig[6 * i + 3], &as, 12);
            remodulate_into(&out.temporal[6 * i], &tmp_sig[6 * i], g, c);
            out.history_length[i] = len;
            lengths[i] = len;
            out.moments[2 * i] = m1;
            out.moments[2 * i + 1] = m2;
            tvar[i] = var;
            out.accepted[i] = took ? 1u : 0u;
            out.reject[i] = why;
        }
    }
    const std::vector<Surface> sf = surfaces(gb, n);
    const std::vector<float> var = bootstrap(tmp_sig, sf, W, H, lengths, tvar, c);
    for (size_t i = 0; i < n; ++i) {
        out.variance[i] = var[i];
        gw.variance[i] = var[i];
    }
    const std::vector<float> raw_var =
        bootstrap(cur_sig, sf, W, H, std::vector<uint32_t>(n, 1u), std::vector<float>(n, 0.0F), c);
    const std::vector<float> a_only = atrous(cur_sig, raw_var, sf, W, H, c);
    const std::vector<float> full = atrous(tmp_sig, var, sf, W, H, c);
    for (size_t i = 0; i < n; ++i) {
        remodulate_into(&out.atrous[6 * i], &a_only[6 * i], gb[i], c);
        remodulate_into(&out.svgf[6 * i], &full[6 * i], gb[i], c);
    }
    gw.published = true;  // HistoryPingPong::Publish
    gw.frame = frame;
    sv.changed = false;
    return 0;
}

}  // namespace

extern "C" {

void* oracle_svgf_create(uint32_t w, uint32_t h, uint32_t flights, const Config* cfg) {
    if (w == 0 || h == 0 || flights == 0 || cfg == nullptr || !config_ok(*cfg)) return nullptr;
    auto* s = new Svgf();
    s->cfg = *cfg;
    s->flights = flights;
    s->gens.resize(2 * size_t(flights));
    s->reset(w, h);
    return s;
}

void oracle_svgf_destroy(void* h) { delete static_cast<Svgf*>(h); }

int oracle_svgf_set_config(void* h, const Config* cfg) {
    if (cfg == nullptr || !config_ok(*cfg)) return 1;
    auto* s = static_cast<Svgf*>(h);
    s->cfg = *cfg;
    s->changed = true;
    return 0;
}

int oracle_svgf_process(void* h, const GbPix* gb, const SigPix* raw, uint32_t w, uint32_t hgt, uint64_t frame,
                        uint32_t trigger, const Outputs* out) {
    if (h == nullptr || gb == nullptr || raw == nullptr || out == nullptr || w == 0 || hgt == 0) return 1;
    return process(*static_cast<Svgf*>(h), gb, raw, w, hgt, frame, trigger, *out);
}

// ComputeRmse (Svgf.cpp:824-833) over 3-float pixels.
float oracle_image_rmse(const float* a, const float* b, uint64_t n) {
    double acc = 0.0;
    for (uint64_t i = 0; i < n; ++i) {
        const V3 d{a[3 * i] - b[3 * i], a[3 * i + 1] - b[3 * i + 1], a[3 * i + 2] - b[3 * i + 2]};
        acc += double(oracle::dot(d, d));
    }
    return float(std::sqrt(acc / (double(n) * 3.0)));
}

// ComputeMotionVector (reconstruction/src/MotionVectors.cpp:37-67) for a
// static object: matrices are row-major 4x4, applied to column vectors.
// out = (currentUv.xy, previousUv.xy, motion.xy, expectedPreviousDepth, valid).
void oracle_motion_vector(const float* position, const float* cur_view_proj, const float* prev_view_proj,
                          const float* prev_world_to_view, const float* cur_jitter, const float* prev_jitter,
                          float* out) {
    auto xf = [](const float* m, const float* v, float* r) {
        for (int row = 0; row < 4; ++row)
            r[row] = m[4 * row] * v[0] + m[4 * row + 1] * v[1] + m[4 * row + 2] * v[2] + m[4 * row + 3] * v[3];
    };
    auto fin4 = [](const float* v) {
        return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]) && std::isfinite(v[3]);
    };
    const float obj[4] = {position[0], position[1], position[2], 1.0F};
    auto project = [&](const float* vp, const float* jit, float* uv) {
        float clip[4];
        xf(vp, obj, clip);
        if (!fin4(obj) || !fin4(clip) || clip[3] <= 1.0e-8F) return false;
        const float rw = 1.0F / clip[3];
        const float nx = clip[0] * rw, ny = clip[1] * rw;
        uv[0] = nx * 0.5F + 0.5F + jit[0];
        uv[1] = 0.5F - ny * 0.5F + jit[1];
        return std::isfinite(uv[0]) && std::isfinite(uv[1]);
    };
    float cu[2] = {0.0F, 0.0F}, pu[2] = {0.0F, 0.0F};
    const bool cv = project(cur_view_proj, cur_jitter, cu);
    const bool pv = project(prev_view_proj, prev_jitter, pu);
    float view[4];
    xf(prev_world_to_view, obj, view);
    const float depth = -view[2];
    const bool dv = fin4(obj) && fin4(view) && std::isfinite(depth) && depth >= 0.0F;
    const bool ok = cv && pv && dv;
    out[0] = cu[0];
    out[1] = cu[1];
    out[2] = pu[0];
    out[3] = pu[1];
    out[4] = ok ? pu[0] - cu[0] : 0.0F;
    out[5] = ok ? pu[1] - cu[1] : 0.0F;
    out[6] = ok ? depth : 0.0F;
    out[7] = ok ? 1.0F : 0.0F;
}

}  // extern "C"
