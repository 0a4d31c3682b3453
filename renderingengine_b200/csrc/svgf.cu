// SVGF / A-Trous reconstruction on sm_100a.
//
// Restates SvgfReconstruction::Process (reconstruction/src/Svgf.cpp:393-582)
// as one pass per data dependency instead of the reference's per-image loops:
//
//   k_temporal   demodulate + ReprojectHistory (Svgf.cpp:128-244) + temporal
//                accumulation of signal and luminance moments; writes the next
//                history generation, the frame planes, the edge records and the
//                two A-Trous chains' first inputs (temporal signal, raw signal)
//   k_bootstrap  BootstrapVariance (Svgf.cpp:584-661) for both chains at once
//                (the depth / normal weights of a 7x7 tap are shared)
//   k_atrous     one FilterATrous iteration (Svgf.cpp:663-752) for both chains
//                at once; the last iteration remodulates (Svgf.cpp:561-577)
//   k_compose    remodulation when the iteration count is 0
//
// Every floating-point expression keeps the reference's operation order and
// rounding (no contraction: the library is built with --fmad=false and IEEE
// division / square root), so everything except expf / powf results is
// bit-identical to the reference's CPU code; history lengths, acceptance and
// reject reasons are exact.
//
// HBM layout, per pixel of the W x H extent:
//   history generation (2 x framesInFlight of them): 4 float4 planes
//     A = (demodDiffuse.xyz, demodSpecular.x)   B = (demodSpecular.yz, moments)
//     C = (variance, linearDepth, normal.xy)    D = (normal.z bits,
//         historyLength | valid << 31, materialId, objectId)
//   A-Trous chains (svgf over the temporal signal, atrous over the raw
//   signal), ping-pong: float4 (diffuse.xyz, variance), float4 (specular.xyz,
//   luminance of the pair)
//   edge records: float4 (normalised normal, linear depth or -1 where the
//   surface is not filterable), uint2 (materialId, objectId)
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "runtime.h"

namespace re {
namespace {

constexpr uint32_t kNoHistory = RE_REJECT_NO_HISTORY;
constexpr uint32_t kReset = RE_REJECT_RESET;
constexpr uint32_t kScreenBounds = RE_REJECT_SCREEN_BOUNDS;
constexpr uint32_t kInvalidCurrent = RE_REJECT_INVALID_CURRENT;
constexpr uint32_t kInvalidHistory = RE_REJECT_INVALID_HISTORY;
constexpr uint32_t kNonFinite = RE_REJECT_NON_FINITE;
constexpr uint32_t kDepth = RE_REJECT_DEPTH;
constexpr uint32_t kNormal = RE_REJECT_NORMAL;
constexpr uint32_t kMaterialId = RE_REJECT_MATERIAL_ID;
constexpr uint32_t kObjectId = RE_REJECT_OBJECT_ID;
constexpr uint32_t kInvalidMotion = RE_REJECT_INVALID_MOTION;
constexpr uint32_t kValidBit = 0x80000000u;

struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ bool finite3(V3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }
// std::max / std::clamp semantics (the first argument wins on NaN).
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float sclamp(float v, float lo, float hi) {
    return (v < lo) ? lo : ((hi < v) ? hi : v);
}
__device__ __forceinline__ V3 lerp3(V3 a, V3 b, float t) { return a * (1.0F - t) + b * t; }
__device__ __forceinline__ float lerp1(float a, float b, float t) { return a * (1.0F - t) + b * t; }
// Luminance(Combined(signal)) (reconstruction/include/reconstruction/Math.hpp:90-92).
__device__ __forceinline__ float luminance(V3 d, V3 s) {
    const V3 c = d + s;
    return 0.2126F * c.x + 0.7152F * c.y + 0.0722F * c.z;
}
// Normalize (Math.hpp:78-81): v / |v| with a +Z fallback.
__device__ __forceinline__ V3 normalize_safe(V3 v) {
    const float len = sqrtf(dot(v, v));
    return len > 1.0e-20F ? v / len : V3{0.0F, 0.0F, 1.0F};
}
__device__ __forceinline__ bool usable_normal(V3 n) { return finite3(n) && dot(n, n) > 1.0e-20F; }

struct Gbuf {
    float depth;
    V3 n;
    V3 dalb, salb;
    float epd;  // expected previous linear depth
    float mx, my;
    uint32_t mat, obj, flags;
};

__device__ __forceinline__ Gbuf load_gbuf(const re_gbuffer_pixel* g, size_t i) {
    const float4* p = reinterpret_cast<const float4*>(g + i);
    const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
    Gbuf r;
    r.depth = a.x;
    r.n = {a.y, a.z, a.w};
    r.dalb = {b.x, b.y, b.z};
    r.salb = {b.w, c.x, c.y};
    r.epd = c.z;
    r.mx = c.w;
    r.my = d.x;
    r.mat = __float_as_uint(d.y);
    r.obj = __float_as_uint(d.z);
    r.flags = __float_as_uint(d.w);
    return r;
}

__device__ __forceinline__ bool gb_valid(const Gbuf& g) { return (g.flags & RE_GBUFFER_VALID) != 0u; }
__device__ __forceinline__ bool gb_motion_valid(const Gbuf& g) { return (g.flags & RE_GBUFFER_MOTION_VALID) != 0u; }
// IsFiniteGeometry (Svgf.cpp:37-40).
__device__ __forceinline__ bool finite_geometry(const Gbuf& g) {
    return isfinite(g.depth) && g.depth >= 0.0F && usable_normal(g.n);
}

struct Sig {
    V3 d, s;
};
__device__ __forceinline__ Sig load_sig(const re_signal_pixel* p, size_t i) {
    const float2* q = reinterpret_cast<const float2*>(p + i);
    const float2 a = q[0], b = q[1], c = q[2];
    return {{a.x, a.y, b.x}, {b.y, c.x, c.y}};
}
__device__ __forceinline__ void store_sig(re_signal_pixel* p, size_t i, V3 d, V3 s) {
    float2* q = reinterpret_cast<float2*>(p + i);
    q[0] = make_float2(d.x, d.y);
    q[1] = make_float2(d.z, s.x);
    q[2] = make_float2(s.y, s.z);
}
__device__ __forceinline__ bool sig_finite(V3 d, V3 s) { return finite3(d) && finite3(s); }

struct Cfg {
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

// SafeAlbedo (Svgf.cpp:42-50).
__device__ __forceinline__ V3 safe_albedo(V3 a, float minimum) {
    const float m = (isfinite(minimum) && minimum > 0.0F) ? minimum : 1.0e-3F;
    return {isfinite(a.x) ? smax(a.x, m) : m, isfinite(a.y) ? smax(a.y, m) : m,
            isfinite(a.z) ? smax(a.z, m) : m};
}
__device__ __forceinline__ Sig remodulate(V3 d, V3 s, const Gbuf& g, const Cfg& c) {
    const V3 da = safe_albedo(g.dalb, c.min_albedo);
    const V3 sa = safe_albedo(g.salb, c.min_albedo);
    return {d * da, c.demod_specular ? s * sa : s};
}

// ValidateCurrentState (Svgf.cpp:82-102).
__device__ __forceinline__ uint32_t validate_current(const Gbuf& g, bool reset) {
    uint32_t r = 0u;
    if (reset) r |= kReset;
    if (!gb_valid(g) || !finite_geometry(g)) r |= kInvalidCurrent;
    if (!gb_motion_valid(g)) r |= kInvalidMotion;
    if (!isfinite(g.mx) || !isfinite(g.my) || !isfinite(g.depth) || !finite3(g.n) || !isfinite(g.epd))
        r |= kNonFinite;
    if (gb_motion_valid(g) && g.epd < 0.0F) r |= kInvalidMotion;
    return r;
}

struct HistView {
    float4* a;
    float4* b;
    float4* c;
    uint4* d;
};

struct Tap {
    V3 dd, ds;
    float m1, m2, var, depth;
    V3 n;
    uint32_t hlen, mat, obj;
    bool valid;
};

__device__ __forceinline__ Tap load_tap(const HistView& h, size_t i) {
    const float4 a = __ldg(h.a + i), b = __ldg(h.b + i), c = __ldg(h.c + i);
    const uint4 d = __ldg(h.d + i);
    Tap t;
    t.dd = {a.x, a.y, a.z};
    t.ds = {a.w, b.x, b.y};
    t.m1 = b.z;
    t.m2 = b.w;
    t.var = c.x;
    t.depth = c.y;
    t.n = {c.z, c.w, __uint_as_float(d.x)};
    t.hlen = d.y & ~kValidBit;
    t.valid = (d.y & kValidBit) != 0u;
    t.mat = d.z;
    t.obj = d.w;
    return t;
}

// ValidateHistory (Svgf.cpp:343-391) for a tap of an existing generation,
// called after the current-state checks passed (they contribute nothing).
__device__ __forceinline__ uint32_t validate_tap(const Gbuf& cur, const Tap& t, const Cfg& c) {
    if (!t.valid) return kInvalidHistory;
    uint32_t r = 0u;
    if (!isfinite(t.depth) || t.depth < 0.0F || !usable_normal(t.n) || !finite3(t.dd) || !finite3(t.ds) ||
        !isfinite(t.m1) || !isfinite(t.m2) || !isfinite(t.var) || t.var < 0.0F)
        r |= kNonFinite;
    const uint32_t max_len = c.max_history < 1u ? 1u : c.max_history;
    if (t.hlen == 0u || t.hlen > max_len) r |= kInvalidHistory;
    const float tol = c.abs_depth + c.rel_depth * smax(fabsf(cur.epd), fabsf(t.depth));
    if (fabsf(cur.epd - t.depth) > tol) r |= kDepth;
    if (dot(normalize_safe(cur.n), normalize_safe(t.n)) < c.normal_cos) r |= kNormal;
    if (c.require_mat && cur.mat != t.mat) r |= kMaterialId;
    if (c.require_obj && cur.obj != t.obj) r |= kObjectId;
    return r;
}

struct Reprojected {
    V3 dd, ds;
    float m1, m2;
    uint32_t hlen;
    uint32_t reasons;
    bool accepted;
};

// ReprojectHistory (Svgf.cpp:128-244): validated bilinear footprint with
// normalised surviving weights, else the nearest valid tap of the 3x3
// neighbourhood of the reprojected pixel.
__device__ Reprojected reproject(uint32_t x, uint32_t y, const Gbuf& cur, uint32_t W, uint32_t H,
                                 const HistView prev, bool has_prev, const Cfg& c, bool reset) {
    Reprojected out{};
    uint32_t base = validate_current(cur, reset);
    const float u = (float(x) + 0.5F) / float(W) + cur.mx;
    const float v = (float(y) + 0.5F) / float(H) + cur.my;
    if (!isfinite(u) || !isfinite(v) || u < 0.0F || v < 0.0F || u >= 1.0F || v >= 1.0F) base |= kScreenBounds;
    if (!has_prev) base |= kNoHistory;
    if (base != 0u) {
        out.reasons = base;
        return out;
    }
    const float sx = u * float(W) - 0.5F;
    const float sy = v * float(H) - 0.5F;
    const long long bx = static_cast<long long>(floorf(sx));
    const long long by = static_cast<long long>(floorf(sy));
    const float fx = sx - float(bx);
    const float fy = sy - float(by);
    float wsum = 0.0F, whl = 0.0F;
    V3 sdd{0.0F, 0.0F, 0.0F}, sds{0.0F, 0.0F, 0.0F};
    float sm1 = 0.0F, sm2 = 0.0F;
    uint32_t failed = 0u;
#pragma unroll
    for (int ty = 0; ty < 2; ++ty) {
#pragma unroll
        for (int tx = 0; tx < 2; ++tx) {
            const long long px = bx + tx, py = by + ty;
            const float wx = tx == 0 ? 1.0F - fx : fx;
            const float wy = ty == 0 ? 1.0F - fy : fy;
            const float w = wx * wy;
            if (w <= 0.0F) continue;
            if (px < 0 || py < 0 || px >= W || py >= H) {
                failed |= kScreenBounds;
                continue;
            }
            const Tap t = load_tap(prev, size_t(py) * W + size_t(px));
            const uint32_t r = validate_tap(cur, t, c);
            if (r != 0u) {
                failed |= r;
                continue;
            }
            sdd = sdd + t.dd * w;
            sds = sds + t.ds * w;
            sm1 += t.m1 * w;
            sm2 += t.m2 * w;
            whl += float(t.hlen) * w;
            wsum += w;
        }
    }
    if (wsum > 0.0F) {
        const float rw = 1.0F / wsum;
        out.dd = sdd * rw;
        out.ds = sds * rw;
        out.m1 = sm1 * rw;
        out.m2 = sm2 * rw;
        out.hlen = static_cast<uint32_t>(whl * rw + 0.5F);
        out.accepted = true;
        return out;
    }
    const long long cx = static_cast<long long>(floorf(u * float(W)));
    const long long cy = static_cast<long long>(floorf(v * float(H)));
    float best_d = FLT_MAX;
    long long best = -1;
    for (int oy = -1; oy <= 1; ++oy) {
        for (int ox = -1; ox <= 1; ++ox) {
            const long long px = cx + ox, py = cy + oy;
            if (px < 0 || py < 0 || px >= W || py >= H) {
                failed |= kScreenBounds;
                continue;
            }
            const size_t idx = size_t(py) * W + size_t(px);
            const uint32_t r = validate_tap(cur, load_tap(prev, idx), c);
            if (r != 0u) {
                failed |= r;
                continue;
            }
            const float dx = (float(px) + 0.5F) - u * float(W);
            const float dy = (float(py) + 0.5F) - v * float(H);
            const float d2 = dx * dx + dy * dy;
            if (d2 < best_d) {
                best_d = d2;
                best = static_cast<long long>(idx);
            }
        }
    }
    if (best >= 0) {
        const Tap t = load_tap(prev, size_t(best));
        out.dd = t.dd;
        out.ds = t.ds;
        out.m1 = t.m1;
        out.m2 = t.m2;
        out.hlen = t.hlen;
        out.accepted = true;
        return out;
    }
    out.reasons = failed == 0u ? kNoHistory : failed;
    return out;
}

struct Planes {
    re_signal_pixel* raw;
    re_signal_pixel* temporal;
    re_signal_pixel* atrous;
    re_signal_pixel* svgf;
    uint32_t* hlen;
    float2* moments;
    float* variance;   // bootstrapped temporal variance (ReconstructionFrame::variance)
    float* var_raw;    // bootstrapped variance of the raw chain
    uint32_t* accepted;
    uint32_t* reject;
    float4* edge;
    uint2* ids;
    float4* chain[2][2][2];  // [svgf=0 / atrous=1][ping][A / B]
};

struct TemporalArgs {
    const re_gbuffer_pixel* gb;
    const re_signal_pixel* raw;
    uint32_t W, H;
    bool reset;
    bool has_prev;
    HistView prev;
    HistView write;
    Planes pl;
    Cfg c;
};

__global__ void __launch_bounds__(256) k_temporal(TemporalArgs a) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.W || y >= a.H) return;
    const size_t i = size_t(y) * a.W + x;
    const Cfg& c = a.c;
    const Gbuf g = load_gbuf(a.gb, i);
    const Sig raw = load_sig(a.raw, i);
    store_sig(a.pl.raw, i, raw.d, raw.s);

    // Demodulate (Svgf.cpp:316-328).
    const V3 da = safe_albedo(g.dalb, c.min_albedo);
    const V3 sa = safe_albedo(g.salb, c.min_albedo);
    const V3 cd = raw.d / da;
    const V3 cs = c.demod_specular ? raw.s / sa : raw.s;
    const float lum0 = luminance(cd, cs);
    const float lum0_sq = lum0 * lum0;
    const bool cur_finite = sig_finite(raw.d, raw.s) && sig_finite(cd, cs) && isfinite(lum0) && isfinite(lum0_sq);
    const V3 zero{0.0F, 0.0F, 0.0F};
    const V3 safe_d = cur_finite ? cd : zero;
    const V3 safe_s = cur_finite ? cs : zero;
    const float lum = cur_finite ? lum0 : 0.0F;
    const float lum_sq = cur_finite ? lum0_sq : 0.0F;

    const Reprojected rp = reproject(x, y, g, a.W, a.H, a.prev, a.has_prev, c, a.reset);
    uint32_t reject = rp.reasons;
    if (!cur_finite) reject |= kNonFinite;
    bool accepted = rp.accepted && reject == 0u;
    V3 acc_d = safe_d, acc_s = safe_s;
    float m1 = lum, m2 = lum_sq;
    uint32_t hlen = 1u;
    if (accepted) {
        const uint32_t max_len = c.max_history < 1u ? 1u : c.max_history;
        hlen = (rp.hlen < max_len - 1u ? rp.hlen : max_len - 1u) + 1u;
        const float rh = 1.0F / float(hlen);
        const float ca = smax(c.min_color_alpha, rh);
        const float ma = smax(c.min_moments_alpha, rh);
        acc_d = lerp3(rp.dd, safe_d, ca);
        acc_s = lerp3(rp.ds, safe_s, ca);
        m1 = lerp1(rp.m1, lum, ma);
        m2 = lerp1(rp.m2, lum_sq, ma);
    }
    float raw_var = m2 - m1 * m1;
    if (!sig_finite(acc_d, acc_s) || !isfinite(m1) || !isfinite(m2) || !isfinite(raw_var)) {
        reject |= kNonFinite;
        accepted = false;
        acc_d = safe_d;
        acc_s = safe_s;
        m1 = lum;
        m2 = lum_sq;
        hlen = 1u;
        raw_var = m2 - m1 * m1;
    }
    const float tvar = smax(raw_var, 0.0F);

    // Next history generation (Svgf.cpp:513-529); the variance word is
    // replaced by the bootstrapped variance in k_bootstrap.
    const bool geom = finite_geometry(g);
    const float depth_out = (isfinite(g.depth) && g.depth >= 0.0F) ? g.depth : 0.0F;
    const V3 n_out = usable_normal(g.n) ? normalize_safe(g.n) : V3{0.0F, 0.0F, 1.0F};
    const bool valid_out = cur_finite && gb_valid(g) && geom && sig_finite(acc_d, acc_s) && isfinite(m1) &&
                           isfinite(m2) && isfinite(tvar);
    a.write.a[i] = make_float4(acc_d.x, acc_d.y, acc_d.z, acc_s.x);
    a.write.b[i] = make_float4(acc_s.y, acc_s.z, m1, m2);
    a.write.c[i] = make_float4(tvar, depth_out, n_out.x, n_out.y);
    a.write.d[i] = make_uint4(__float_as_uint(n_out.z), hlen | (valid_out ? kValidBit : 0u), g.mat, g.obj);

    const Sig t = remodulate(acc_d, acc_s, g, c);
    store_sig(a.pl.temporal, i, t.d, t.s);
    a.pl.hlen[i] = hlen;
    a.pl.moments[i] = make_float2(m1, m2);
    a.pl.accepted[i] = accepted ? 1u : 0u;
    a.pl.reject[i] = reject;

    // Edge record shared by the bootstrap and every A-Trous iteration.
    const bool filterable = gb_valid(g) && geom;
    const V3 nn = normalize_safe(g.n);
    a.pl.edge[i] = make_float4(nn.x, nn.y, nn.z, filterable ? g.depth : -1.0F);
    a.pl.ids[i] = make_uint2(g.mat, g.obj);
    // First inputs of the two chains: the temporal signal (SVGF) and the
    // current signal (A-Trous only); .w of A = pre-bootstrap variance.
    a.pl.chain[0][0][0][i] = make_float4(acc_d.x, acc_d.y, acc_d.z, tvar);
    a.pl.chain[0][0][1][i] = make_float4(acc_s.x, acc_s.y, acc_s.z, luminance(acc_d, acc_s));
    a.pl.chain[1][0][0][i] = make_float4(safe_d.x, safe_d.y, safe_d.z, 0.0F);
    a.pl.chain[1][0][1][i] = make_float4(safe_s.x, safe_s.y, safe_s.z, luminance(safe_d, safe_s));
}

struct FilterArgs {
    uint32_t W, H;
    Planes pl;
    Cfg c;
    float* history_variance;  // C plane of the written generation, stride 4 floats
    const re_gbuffer_pixel* gb;
};

// BootstrapVariance (Svgf.cpp:584-661) of both chains: the temporal chain
// with its history lengths and temporal variance, the raw chain with history
// length 1 and variance 0.
__global__ void __launch_bounds__(256) k_bootstrap(FilterArgs a) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.W || y >= a.H) return;
    const size_t i = size_t(y) * a.W + x;
    const Cfg& c = a.c;
    const float4 ce = __ldg(a.pl.edge + i);
    float out_t = c.min_variance, out_r = c.min_variance;
    if (ce.w >= 0.0F) {
        const uint2 cid = __ldg(a.pl.ids + i);
        const V3 cn{ce.x, ce.y, ce.z};
        const float depth_scale = smax(0.01F, fabsf(ce.w) * 0.02F);
        float w_t = 0.0F, f_t = 0.0F, s_t = 0.0F;
        float w_r = 0.0F, f_r = 0.0F, s_r = 0.0F;
        const int r = int(c.radius);
        for (int oy = -r; oy <= r; ++oy) {
            const long long py = (long long)y + oy;
            if (py < 0 || py >= a.H) continue;
            for (int ox = -r; ox <= r; ++ox) {
                const long long px = (long long)x + ox;
                if (px < 0 || px >= a.W) continue;
                const size_t j = size_t(py) * a.W + size_t(px);
                const float4 se = __ldg(a.pl.edge + j);
                if (!(se.w >= 0.0F)) continue;
                const uint2 sid = __ldg(a.pl.ids + j);
                if (sid.x != cid.x || sid.y != cid.y) continue;
                const float dw = expf(-fabsf(se.w - ce.w) / depth_scale);
                const float nw = powf(sclamp(dot(cn, V3{se.x, se.y, se.z}), 0.0F, 1.0F), 32.0F);
                const float w = dw * nw;
                if (!isfinite(w) || w <= 0.0F) continue;
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const float4 sa = __ldg(a.pl.chain[k][0][0] + j);
                    const float4 sb = __ldg(a.pl.chain[k][0][1] + j);
                    if (!sig_finite(V3{sa.x, sa.y, sa.z}, V3{sb.x, sb.y, sb.z})) continue;
                    const float l = sb.w;
                    const float l2 = l * l;
                    if (!isfinite(l) || !isfinite(l2)) continue;
                    if (k == 0) {
                        f_t += l * w;
                        s_t += l2 * w;
                        w_t += w;
                    } else {
                        f_r += l * w;
                        s_r += l2 * w;
                        w_r += w;
                    }
                }
            }
        }
        const float short_len = float(c.short_history < 1u ? 1u : c.short_history);
        {
            const float sv = (w_t > 0.0F && isfinite(w_t) && isfinite(f_t) && isfinite(s_t))
                                 ? smax(s_t / w_t - (f_t / w_t) * (f_t / w_t), 0.0F)
                                 : 0.0F;
            const float blend = sclamp(float(__ldg(a.pl.hlen + i)) / short_len, 0.0F, 1.0F);
            const float tv = __ldg(a.pl.chain[0][0][0] + i).w;
            const float safe_tv = (isfinite(tv) && tv >= 0.0F) ? tv : sv;
            const float b = lerp1(sv, safe_tv, blend);
            out_t = isfinite(b) ? smax(b, c.min_variance) : c.min_variance;
        }
        {
            const float sv = (w_r > 0.0F && isfinite(w_r) && isfinite(f_r) && isfinite(s_r))
                                 ? smax(s_r / w_r - (f_r / w_r) * (f_r / w_r), 0.0F)
                                 : 0.0F;
            const float blend = sclamp(1.0F / short_len, 0.0F, 1.0F);
            const float b = lerp1(sv, 0.0F, blend);
            out_r = isfinite(b) ? smax(b, c.min_variance) : c.min_variance;
        }
    }
    a.pl.variance[i] = out_t;
    a.pl.var_raw[i] = out_r;
    a.history_variance[4 * i] = out_t;
}

// One FilterATrous iteration (Svgf.cpp:677-749) for both chains.  FIRST reads
// the per-pixel variance from the bootstrap planes, later iterations from .w
// of the chain; LAST remodulates into the frame's atrous / svgf planes.
template <bool FIRST, bool LAST>
__global__ void __launch_bounds__(256) k_atrous(FilterArgs a, uint32_t step, int ping) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.W || y >= a.H) return;
    const size_t i = size_t(y) * a.W + x;
    const Cfg& c = a.c;
    const float* var0[2] = {a.pl.variance, a.pl.var_raw};
    const float4* in_a[2] = {a.pl.chain[0][ping][0], a.pl.chain[1][ping][0]};
    const float4* in_b[2] = {a.pl.chain[0][ping][1], a.pl.chain[1][ping][1]};

    V3 safe_d[2], safe_s[2];
    float safe_var[2], c_lum[2], lum_den[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const float4 ca = __ldg(in_a[k] + i);
        const float4 cb = __ldg(in_b[k] + i);
        const V3 d{ca.x, ca.y, ca.z}, s{cb.x, cb.y, cb.z};
        const bool fin = sig_finite(d, s);
        safe_d[k] = fin ? d : V3{0.0F, 0.0F, 0.0F};
        safe_s[k] = fin ? s : V3{0.0F, 0.0F, 0.0F};
        const float v = FIRST ? __ldg(var0[k] + i) : ca.w;
        safe_var[k] = (isfinite(v) && v >= 0.0F) ? smax(v, c.min_variance) : c.min_variance;
        c_lum[k] = fin ? cb.w : luminance(safe_d[k], safe_s[k]);
        lum_den[k] = smax(c.phi_luminance * sqrtf(smax(safe_var[k], 0.0F)), 1.0e-4F);
    }
    V3 out_d[2] = {safe_d[0], safe_d[1]}, out_s[2] = {safe_s[0], safe_s[1]};
    float out_var[2] = {safe_var[0], safe_var[1]};

    const float4 ce = __ldg(a.pl.edge + i);
    if (ce.w >= 0.0F) {
        const uint2 cid = __ldg(a.pl.ids + i);
        const V3 cn{ce.x, ce.y, ce.z};
        const float depth_scale = smax(0.01F, fabsf(ce.w) * 0.01F);
        const float depth_den = smax(c.phi_depth * depth_scale * float(step), 1.0e-6F);
        const float kernel[5] = {1.0F, 4.0F, 6.0F, 4.0F, 1.0F};
        V3 sd[2] = {{0.0F, 0.0F, 0.0F}, {0.0F, 0.0F, 0.0F}};
        V3 ss[2] = {{0.0F, 0.0F, 0.0F}, {0.0F, 0.0F, 0.0F}};
        float ws[2] = {0.0F, 0.0F}, wv[2] = {0.0F, 0.0F};
#pragma unroll
        for (int ky = -2; ky <= 2; ++ky) {
            const long long py = (long long)y + (long long)ky * step;
            if (py < 0 || py >= a.H) continue;
#pragma unroll
            for (int kx = -2; kx <= 2; ++kx) {
                const long long px = (long long)x + (long long)kx * step;
                if (px < 0 || px >= a.W) continue;
                const size_t j = size_t(py) * a.W + size_t(px);
                const float4 se = __ldg(a.pl.edge + j);
                if (!(se.w >= 0.0F)) continue;  // EdgeWeight == 0
                const uint2 sid = __ldg(a.pl.ids + j);
                if (sid.x != cid.x || sid.y != cid.y) continue;
                // EdgeWeight (Svgf.cpp:246-272): the depth and normal terms
                // are shared by both chains.
                const float dw = expf(-fabsf(se.w - ce.w) / depth_den);
                const float nw = powf(sclamp(dot(cn, V3{se.x, se.y, se.z}), 0.0F, 1.0F), c.phi_normal);
                const float dn = dw * nw;
                const float spatial = kernel[kx + 2] * kernel[ky + 2];
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const float4 sa = __ldg(in_a[k] + j);
                    const float4 sb = __ldg(in_b[k] + j);
                    const V3 d{sa.x, sa.y, sa.z}, s{sb.x, sb.y, sb.z};
                    const float sv = FIRST ? __ldg(var0[k] + j) : sa.w;
                    if (!sig_finite(d, s) || !isfinite(sv) || sv < 0.0F) continue;
                    const float sl = sb.w;
                    float ew = 0.0F;
                    if (isfinite(c_lum[k]) && isfinite(sl)) {
                        const float lw = expf(-fabsf(sl - c_lum[k]) / lum_den[k]);
                        ew = dn * lw;
                        if (!isfinite(ew)) ew = 0.0F;
                    }
                    const float w = spatial * ew;
                    if (!isfinite(w) || w <= 0.0F) continue;
                    sd[k] = sd[k] + d * w;
                    ss[k] = ss[k] + s * w;
                    wv[k] += sv * w * w;
                    ws[k] += w;
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const bool ok = ws[k] > 0.0F && isfinite(ws[k]) && isfinite(wv[k]) && sig_finite(sd[k], ss[k]);
            V3 fd = ok ? sd[k] / ws[k] : safe_d[k];
            V3 fs = ok ? ss[k] / ws[k] : safe_s[k];
            if (!sig_finite(fd, fs)) {
                fd = safe_d[k];
                fs = safe_s[k];
            }
            out_d[k] = fd;
            out_s[k] = fs;
            const float fv = ok ? wv[k] / (ws[k] * ws[k]) : safe_var[k];
            out_var[k] = isfinite(fv) ? smax(fv, c.min_variance) : safe_var[k];
        }
    }
    if (LAST) {
        const Gbuf g = load_gbuf(a.gb, i);
        const Sig s0 = remodulate(out_d[0], out_s[0], g, c);
        const Sig s1 = remodulate(out_d[1], out_s[1], g, c);
        store_sig(a.pl.svgf, i, s0.d, s0.s);
        store_sig(a.pl.atrous, i, s1.d, s1.s);
    } else {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            a.pl.chain[k][ping ^ 1][0][i] = make_float4(out_d[k].x, out_d[k].y, out_d[k].z, out_var[k]);
            a.pl.chain[k][ping ^ 1][1][i] =
                make_float4(out_s[k].x, out_s[k].y, out_s[k].z, luminance(out_d[k], out_s[k]));
        }
    }
}

// Zero A-Trous iterations: FilterATrous returns its input unchanged.
__global__ void __launch_bounds__(256) k_compose(FilterArgs a) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.W || y >= a.H) return;
    const size_t i = size_t(y) * a.W + x;
    const Gbuf g = load_gbuf(a.gb, i);
    for (int k = 0; k < 2; ++k) {
        const float4 ca = a.pl.chain[k][0][0][i];
        const float4 cb = a.pl.chain[k][0][1][i];
        const Sig s = remodulate(V3{ca.x, ca.y, ca.z}, V3{cb.x, cb.y, cb.z}, g, a.c);
        store_sig(k == 0 ? a.pl.svgf : a.pl.atrous, i, s.d, s.s);
    }
}

// RejectReasonColor (Svgf.cpp:274-308).
__device__ __forceinline__ V3 reject_color(uint32_t r) {
    if (r == 0u) return {0.0F, 1.0F, 0.0F};
    if (r & kReset) return {1.0F, 1.0F, 0.0F};
    if (r & kScreenBounds) return {1.0F, 0.0F, 1.0F};
    if (r & kDepth) return {0.0F, 0.25F, 1.0F};
    if (r & kNormal) return {0.0F, 1.0F, 1.0F};
    if (r & kMaterialId) return {0.0F, 0.6F, 0.0F};
    if (r & kObjectId) return {0.6F, 0.0F, 1.0F};
    if (r & kInvalidMotion) return {1.0F, 0.2F, 0.2F};
    if (r & kNonFinite) return {1.0F, 0.4F, 0.0F};
    if ((r & kInvalidCurrent) || (r & kInvalidHistory)) return {1.0F, 0.0F, 0.0F};
    return {0.35F, 0.35F, 0.35F};
}

// SelectOutput (Svgf.cpp:754-822).
__global__ void __launch_bounds__(256) k_select(Planes pl, const re_gbuffer_pixel* gb, uint32_t output,
                                                uint32_t max_history, size_t count, float* dst) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    V3 v{0.0F, 0.0F, 0.0F};
    switch (output) {
        case RE_SVGF_OUTPUT_RAW:
        case RE_SVGF_OUTPUT_TEMPORAL:
        case RE_SVGF_OUTPUT_ATROUS:
        case RE_SVGF_OUTPUT_SVGF: {
            const re_signal_pixel* p = output == RE_SVGF_OUTPUT_RAW        ? pl.raw
                                       : output == RE_SVGF_OUTPUT_TEMPORAL ? pl.temporal
                                       : output == RE_SVGF_OUTPUT_ATROUS   ? pl.atrous
                                                                           : pl.svgf;
            const Sig s = load_sig(p, i);
            v = s.d + s.s;
            break;
        }
        case RE_SVGF_OUTPUT_MOTION: {
            const Gbuf g = load_gbuf(gb, i);
            v = {0.5F + g.mx * 16.0F, 0.5F + g.my * 16.0F, 0.5F};
            break;
        }
        case RE_SVGF_OUTPUT_HISTORY_LENGTH: {
            const float n = float(pl.hlen[i]) / float(max_history < 1u ? 1u : max_history);
            v = {n, n, n};
            break;
        }
        case RE_SVGF_OUTPUT_MOMENTS:
            v = {pl.moments[i].x, pl.moments[i].y, 0.0F};
            break;
        case RE_SVGF_OUTPUT_VARIANCE: {
            const float sd = sqrtf(smax(pl.variance[i], 0.0F));
            v = {sd, sd, sd};
            break;
        }
        case RE_SVGF_OUTPUT_HISTORY_ACCEPTANCE:
            v = pl.accepted[i] != 0u ? V3{0.0F, 1.0F, 0.0F} : V3{1.0F, 0.0F, 0.0F};
            break;
        case RE_SVGF_OUTPUT_REJECT_REASONS:
            v = reject_color(pl.reject[i]);
            break;
        default:
            break;
    }
    dst[3 * i + 0] = v.x;
    dst[3 * i + 1] = v.y;
    dst[3 * i + 2] = v.z;
}

// ComputeRmse (Svgf.cpp:824-833): per-pixel Dot(d, d) in float, summed in
// double.
__global__ void __launch_bounds__(256) k_sqerr(const float* a, const float* b, size_t count, double* acc) {
    double local = 0.0;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x) {
        const V3 d{a[3 * i] - b[3 * i], a[3 * i + 1] - b[3 * i + 1], a[3 * i + 2] - b[3 * i + 2]};
        local += double(dot(d, d));
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
    __shared__ double part[8];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) s += part[w];
        atomicAdd(acc, s);
    }
}

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

}  // namespace
}  // namespace re

using namespace re;

struct re_svgf {
    int device = 0;
    re_svgf_config cfg{};
    bool params_changed = false;
    uint32_t width = 0, height = 0, flights = 1;
    size_t capacity = 0;  // pixels the arena is carved for
    struct Generation {
        HistView view{};
        bool published = false;
        uint64_t frame = ~0ull;
    };
    std::vector<Generation> gens;
    Planes pl{};
    re_gbuffer_pixel* stage_gb = nullptr;
    re_signal_pixel* stage_sig = nullptr;
    DeviceBuffer arena;
    bool has_frame = false;
    uint32_t frame_w = 0, frame_h = 0;
};

namespace {

re_status validate_config(const re_svgf_config& c) {
    auto fin = [](float v) { return std::isfinite(v); };
    if (!fin(c.relative_depth_threshold) || c.relative_depth_threshold < 0.0F || !fin(c.absolute_depth_threshold) ||
        c.absolute_depth_threshold < 0.0F || !fin(c.normal_cosine_threshold) || c.normal_cosine_threshold < -1.0F ||
        c.normal_cosine_threshold > 1.0F)
        return set_error(RE_INVALID_ARGUMENT, "SVGF history-validation parameters are invalid");
    if (c.max_history_length == 0u || c.max_history_length > 0x7fffffffu || !fin(c.minimum_color_alpha) ||
        c.minimum_color_alpha < 0.0F || c.minimum_color_alpha > 1.0F || !fin(c.minimum_moments_alpha) ||
        c.minimum_moments_alpha < 0.0F || c.minimum_moments_alpha > 1.0F)
        return set_error(RE_INVALID_ARGUMENT, "SVGF temporal parameters are invalid");
    if (c.short_history_length == 0u || c.spatial_radius > 64u || !fin(c.minimum_variance) ||
        c.minimum_variance <= 0.0F)
        return set_error(RE_INVALID_ARGUMENT, "SVGF variance parameters are invalid");
    if (c.atrous_iterations > 16u || !fin(c.phi_depth) || c.phi_depth <= 0.0F || !fin(c.phi_normal) ||
        c.phi_normal < 0.0F || !fin(c.phi_luminance) || c.phi_luminance <= 0.0F || !fin(c.minimum_albedo) ||
        c.minimum_albedo <= 0.0F)
        return set_error(RE_INVALID_ARGUMENT, "SVGF spatial/demodulation parameters are invalid");
    return RE_SUCCESS;
}

Cfg device_cfg(const re_svgf_config& s) {
    Cfg c;
    c.rel_depth = s.relative_depth_threshold;
    c.abs_depth = s.absolute_depth_threshold;
    c.normal_cos = s.normal_cosine_threshold;
    c.require_mat = s.require_material_id;
    c.require_obj = s.require_object_id;
    c.max_history = s.max_history_length;
    c.min_color_alpha = s.minimum_color_alpha;
    c.min_moments_alpha = s.minimum_moments_alpha;
    c.short_history = s.short_history_length;
    c.radius = s.spatial_radius;
    c.min_variance = s.minimum_variance;
    c.iterations = s.atrous_iterations;
    c.phi_depth = s.phi_depth;
    c.phi_normal = s.phi_normal;
    c.phi_luminance = s.phi_luminance;
    c.min_albedo = s.minimum_albedo;
    c.demod_specular = s.demodulate_specular;
    return c;
}

// Carves every plane out of one allocation sized for `pixels`.
re_status carve(re_svgf* s, size_t pixels) {
    const size_t P = pixels;
    const size_t gens = 2 * size_t(s->flights);
    size_t total = 0;
    auto slot = [&](size_t bytes) {
        const size_t off = total;
        total += align_up(bytes, 256);
        return off;
    };
    std::vector<size_t> hist_off;
    for (size_t g = 0; g < gens * 4; ++g) hist_off.push_back(slot(16 * P));
    const size_t o_raw = slot(24 * P), o_tmp = slot(24 * P), o_atr = slot(24 * P), o_svgf = slot(24 * P);
    const size_t o_hlen = slot(4 * P), o_mom = slot(8 * P), o_var = slot(4 * P), o_varr = slot(4 * P);
    const size_t o_acc = slot(4 * P), o_rej = slot(4 * P), o_edge = slot(16 * P), o_ids = slot(8 * P);
    size_t o_chain[2][2][2];
    for (int k = 0; k < 2; ++k)
        for (int p = 0; p < 2; ++p)
            for (int h = 0; h < 2; ++h) o_chain[k][p][h] = slot(16 * P);
    const size_t o_sgb = slot(64 * P), o_ssig = slot(24 * P);
    RE_CUDA_TRY(s->arena.reserve(total));
    char* base = static_cast<char*>(s->arena.ptr);
    s->gens.assign(gens, {});
    for (size_t g = 0; g < gens; ++g) {
        s->gens[g].view.a = reinterpret_cast<float4*>(base + hist_off[4 * g + 0]);
        s->gens[g].view.b = reinterpret_cast<float4*>(base + hist_off[4 * g + 1]);
        s->gens[g].view.c = reinterpret_cast<float4*>(base + hist_off[4 * g + 2]);
        s->gens[g].view.d = reinterpret_cast<uint4*>(base + hist_off[4 * g + 3]);
    }
    Planes& pl = s->pl;
    pl.raw = reinterpret_cast<re_signal_pixel*>(base + o_raw);
    pl.temporal = reinterpret_cast<re_signal_pixel*>(base + o_tmp);
    pl.atrous = reinterpret_cast<re_signal_pixel*>(base + o_atr);
    pl.svgf = reinterpret_cast<re_signal_pixel*>(base + o_svgf);
    pl.hlen = reinterpret_cast<uint32_t*>(base + o_hlen);
    pl.moments = reinterpret_cast<float2*>(base + o_mom);
    pl.variance = reinterpret_cast<float*>(base + o_var);
    pl.var_raw = reinterpret_cast<float*>(base + o_varr);
    pl.accepted = reinterpret_cast<uint32_t*>(base + o_acc);
    pl.reject = reinterpret_cast<uint32_t*>(base + o_rej);
    pl.edge = reinterpret_cast<float4*>(base + o_edge);
    pl.ids = reinterpret_cast<uint2*>(base + o_ids);
    for (int k = 0; k < 2; ++k)
        for (int p = 0; p < 2; ++p)
            for (int h = 0; h < 2; ++h) pl.chain[k][p][h] = reinterpret_cast<float4*>(base + o_chain[k][p][h]);
    s->stage_gb = reinterpret_cast<re_gbuffer_pixel*>(base + o_sgb);
    s->stage_sig = reinterpret_cast<re_signal_pixel*>(base + o_ssig);
    s->capacity = P;
    return RE_SUCCESS;
}

// HistoryPingPong::Reset (History.cpp:74-84): new extent, nothing published.
re_status reset_history(re_svgf* s, uint32_t w, uint32_t h) {
    if (w == 0 || h == 0) return set_error(RE_INVALID_ARGUMENT, "History extent must be non-zero");
    const size_t P = size_t(w) * h;
    if (P > s->capacity) {  // every plane is carved for `capacity` pixels
        re_status st = carve(s, P);
        if (st != RE_SUCCESS) return st;
    }
    s->width = w;
    s->height = h;
    for (auto& g : s->gens) {
        g.published = false;
        g.frame = ~0ull;
    }
    s->has_frame = false;
    return RE_SUCCESS;
}

// HistoryPingPong::ResourceIndex (History.cpp:22-29).
size_t resource_index(const re_svgf* s, uint64_t frame) {
    const uint64_t gen = (frame / s->flights) & 1ull;
    const uint64_t slot = frame % s->flights;
    return size_t(gen * s->flights + slot);
}

size_t plane_bytes(uint32_t plane, size_t P) {
    switch (plane) {
        case RE_SVGF_PLANE_RAW:
        case RE_SVGF_PLANE_TEMPORAL:
        case RE_SVGF_PLANE_ATROUS:
        case RE_SVGF_PLANE_SVGF: return 24 * P;
        case RE_SVGF_PLANE_MOMENTS: return 8 * P;
        case RE_SVGF_PLANE_HISTORY_LENGTH:
        case RE_SVGF_PLANE_VARIANCE:
        case RE_SVGF_PLANE_ACCEPTED:
        case RE_SVGF_PLANE_REJECT_REASONS: return 4 * P;
        default: return 0;
    }
}

void* plane_ptr(re_svgf* s, uint32_t plane) {
    switch (plane) {
        case RE_SVGF_PLANE_RAW: return s->pl.raw;
        case RE_SVGF_PLANE_TEMPORAL: return s->pl.temporal;
        case RE_SVGF_PLANE_ATROUS: return s->pl.atrous;
        case RE_SVGF_PLANE_SVGF: return s->pl.svgf;
        case RE_SVGF_PLANE_HISTORY_LENGTH: return s->pl.hlen;
        case RE_SVGF_PLANE_MOMENTS: return s->pl.moments;
        case RE_SVGF_PLANE_VARIANCE: return s->pl.variance;
        case RE_SVGF_PLANE_ACCEPTED: return s->pl.accepted;
        case RE_SVGF_PLANE_REJECT_REASONS: return s->pl.reject;
        default: return nullptr;
    }
}

}  // namespace

extern "C" {

RE_API re_status re_svgf_default_config(re_svgf_config* out) {
    if (out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null config");
    *out = re_svgf_config{};
    out->relative_depth_threshold = 0.02F;
    out->absolute_depth_threshold = 0.01F;
    out->normal_cosine_threshold = 0.9063078F;
    out->require_material_id = 1;
    out->require_object_id = 1;
    out->max_history_length = 32;
    out->minimum_color_alpha = 0.05F;
    out->minimum_moments_alpha = 0.10F;
    out->short_history_length = 4;
    out->spatial_radius = 3;
    out->minimum_variance = 1.0e-6F;
    out->atrous_iterations = 4;
    out->phi_depth = 1.0F;
    out->phi_normal = 64.0F;
    out->phi_luminance = 4.0F;
    out->minimum_albedo = 1.0e-3F;
    out->demodulate_specular = 1;
    return clear_error();
}

RE_API re_status re_svgf_create(uint32_t width, uint32_t height, uint32_t frames_in_flight,
                                const re_svgf_config* config, uint32_t device, re_svgf** out) {
    if (out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null output handle");
    *out = nullptr;
    if (width == 0 || height == 0) return set_error(RE_INVALID_ARGUMENT, "History extent must be non-zero");
    if (frames_in_flight == 0) return set_error(RE_INVALID_ARGUMENT, "framesInFlight must be at least one");
    re_svgf_config cfg;
    if (config != nullptr) {
        cfg = *config;
    } else {
        re_svgf_default_config(&cfg);
    }
    re_status st = validate_config(cfg);
    if (st != RE_SUCCESS) return st;
    RE_CUDA_TRY(cudaSetDevice(int(device)));
    auto* s = new re_svgf();
    s->device = int(device);
    s->cfg = cfg;
    s->flights = frames_in_flight;
    st = carve(s, size_t(width) * height);
    if (st == RE_SUCCESS) st = reset_history(s, width, height);
    if (st != RE_SUCCESS) {
        delete s;
        return st;
    }
    *out = s;
    return clear_error();
}

RE_API re_status re_svgf_destroy(re_svgf* s) {
    if (s == nullptr) return clear_error();
    cudaSetDevice(s->device);
    cudaDeviceSynchronize();
    delete s;
    return clear_error();
}

RE_API re_status re_svgf_set_config(re_svgf* s, const re_svgf_config* config) {
    if (s == nullptr || config == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    re_status st = validate_config(*config);
    if (st != RE_SUCCESS) return st;
    s->cfg = *config;
    s->params_changed = true;
    return clear_error();
}

RE_API re_status re_svgf_get_config(const re_svgf* s, re_svgf_config* out) {
    if (s == nullptr || out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    *out = s->cfg;
    return clear_error();
}

RE_API re_status re_svgf_reset(re_svgf* s, uint32_t width, uint32_t height) {
    if (s == nullptr) return set_error(RE_INVALID_ARGUMENT, "null svgf");
    RE_CUDA_TRY(cudaSetDevice(s->device));
    RE_CUDA_TRY(cudaDeviceSynchronize());
    re_status st = reset_history(s, width, height);
    if (st != RE_SUCCESS) return st;
    s->params_changed = false;
    return clear_error();
}

RE_API re_status re_svgf_process(re_svgf* s, const re_svgf_frame_inputs* in, void* stream) {
    if (s == nullptr || in == nullptr || in->gbuffer == nullptr || in->raw_signal == nullptr)
        return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (in->width == 0 || in->height == 0) return set_error(RE_INVALID_ARGUMENT, "Image extent must be non-zero");
    if (in->memory != RE_MEMORY_HOST && in->memory != RE_MEMORY_DEVICE)
        return set_error(RE_INVALID_ARGUMENT, "unknown memory kind");
    if (in->memory == RE_MEMORY_DEVICE &&
        ((reinterpret_cast<uintptr_t>(in->gbuffer) | reinterpret_cast<uintptr_t>(in->raw_signal)) & 15u) != 0)
        return set_error(RE_INVALID_ARGUMENT, "device input arrays must be 16-byte aligned");
    RE_CUDA_TRY(cudaSetDevice(s->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t W = in->width, H = in->height;
    const size_t P = size_t(W) * H;

    uint32_t trigger = in->reset_trigger;
    if (W != s->width || H != s->height) trigger |= RE_RESET_RESOLUTION;
    if (s->params_changed) trigger |= RE_RESET_RECONSTRUCTION_PARAMS;
    const bool reset = trigger != 0u;
    if (reset) {
        // HistoryPingPong::BeginWrite resets every generation; planes in use
        // by earlier work on other streams must be idle before a re-carve.
        if (W != s->width || H != s->height) RE_CUDA_TRY(cudaDeviceSynchronize());
        re_status r = reset_history(s, W, H);
        if (r != RE_SUCCESS) return r;
    }
    const size_t wi = resource_index(s, in->frame_index);
    s->gens[wi].published = false;
    s->gens[wi].frame = ~0ull;
    const HistView* prev = nullptr;
    if (!reset && in->frame_index != 0ull) {
        const size_t ri = resource_index(s, in->frame_index - 1ull);
        if (s->gens[ri].published && s->gens[ri].frame == in->frame_index - 1ull) prev = &s->gens[ri].view;
    }

    const re_gbuffer_pixel* gb = in->gbuffer;
    const re_signal_pixel* raw = in->raw_signal;
    if (in->memory == RE_MEMORY_HOST) {
        RE_CUDA_TRY(cudaMemcpyAsync(s->stage_gb, gb, 64 * P, cudaMemcpyHostToDevice, st));
        RE_CUDA_TRY(cudaMemcpyAsync(s->stage_sig, raw, 24 * P, cudaMemcpyHostToDevice, st));
        gb = s->stage_gb;
        raw = s->stage_sig;
    }

    const dim3 block(32, 8);
    const dim3 grid((W + 31) / 32, (H + 7) / 8);
    TemporalArgs ta{};
    ta.gb = gb;
    ta.raw = raw;
    ta.W = W;
    ta.H = H;
    ta.reset = reset;
    ta.has_prev = prev != nullptr;
    if (prev != nullptr) ta.prev = *prev;
    ta.write = s->gens[wi].view;
    ta.pl = s->pl;
    ta.c = device_cfg(s->cfg);
    k_temporal<<<grid, block, 0, st>>>(ta);
    RE_CUDA_TRY(cudaGetLastError());

    FilterArgs fa{};
    fa.W = W;
    fa.H = H;
    fa.pl = s->pl;
    fa.c = ta.c;
    fa.history_variance = reinterpret_cast<float*>(s->gens[wi].view.c);
    fa.gb = gb;
    k_bootstrap<<<grid, block, 0, st>>>(fa);
    RE_CUDA_TRY(cudaGetLastError());
    const uint32_t n = s->cfg.atrous_iterations;
    if (n == 0u) {
        k_compose<<<grid, block, 0, st>>>(fa);
    } else {
        int ping = 0;
        for (uint32_t it = 0; it < n; ++it) {
            const uint32_t step = 1u << (it < 15u ? it : 15u);
            const bool first = it == 0, last = it + 1 == n;
            if (first && last) k_atrous<true, true><<<grid, block, 0, st>>>(fa, step, ping);
            else if (first) k_atrous<true, false><<<grid, block, 0, st>>>(fa, step, ping);
            else if (last) k_atrous<false, true><<<grid, block, 0, st>>>(fa, step, ping);
            else k_atrous<false, false><<<grid, block, 0, st>>>(fa, step, ping);
            ping ^= 1;
        }
    }
    RE_CUDA_TRY(cudaGetLastError());
    // HistoryPingPong::Publish (History.cpp:68-72).
    s->gens[wi].published = true;
    s->gens[wi].frame = in->frame_index;
    s->params_changed = false;
    s->has_frame = true;
    s->frame_w = W;
    s->frame_h = H;
    return clear_error();
}

RE_API re_status re_svgf_read(re_svgf* s, uint32_t plane, void* dst, uint64_t bytes, uint32_t memory,
                              void* stream) {
    if (s == nullptr || dst == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (!s->has_frame) return set_error(RE_NOT_READY, "no frame has been processed");
    const size_t need = plane_bytes(plane, size_t(s->frame_w) * s->frame_h);
    if (need == 0) return set_error(RE_INVALID_ARGUMENT, "unknown plane");
    if (bytes < need) return set_error(RE_INVALID_ARGUMENT, "destination is smaller than the plane");
    RE_CUDA_TRY(cudaSetDevice(s->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    RE_CUDA_TRY(cudaMemcpyAsync(dst, plane_ptr(s, plane), need,
                                memory == RE_MEMORY_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, st));
    if (memory == RE_MEMORY_HOST) RE_CUDA_TRY(cudaStreamSynchronize(st));
    return clear_error();
}

RE_API re_status re_svgf_plane_pointer(re_svgf* s, uint32_t plane, void** out) {
    if (s == nullptr || out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    *out = plane_ptr(s, plane);
    if (*out == nullptr) return set_error(RE_INVALID_ARGUMENT, "unknown plane");
    return clear_error();
}

RE_API re_status re_svgf_select_output(re_svgf* s, const re_gbuffer_pixel* gbuffer, uint32_t gbuffer_memory,
                                       uint32_t output, float* dst, uint32_t dst_memory, void* stream) {
    if (s == nullptr || dst == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (!s->has_frame) return set_error(RE_NOT_READY, "no frame has been processed");
    if (output > RE_SVGF_OUTPUT_REJECT_REASONS) return set_error(RE_INVALID_ARGUMENT, "unknown output");
    if (output == RE_SVGF_OUTPUT_MOTION && gbuffer == nullptr)
        return set_error(RE_INVALID_ARGUMENT, "the motion output needs the gbuffer");
    RE_CUDA_TRY(cudaSetDevice(s->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t P = size_t(s->frame_w) * s->frame_h;
    const re_gbuffer_pixel* gb = gbuffer;
    if (gb != nullptr && gbuffer_memory == RE_MEMORY_HOST) {
        RE_CUDA_TRY(cudaMemcpyAsync(s->stage_gb, gb, 64 * P, cudaMemcpyHostToDevice, st));
        gb = s->stage_gb;
    }
    float* out = dst;
    DeviceBuffer tmp;
    if (dst_memory == RE_MEMORY_HOST) {
        RE_CUDA_TRY(tmp.reserve(12 * P));
        out = static_cast<float*>(tmp.ptr);
    }
    const unsigned blocks = unsigned((P + 255) / 256);
    k_select<<<blocks, 256, 0, st>>>(s->pl, gb, output, s->cfg.max_history_length, P, out);
    RE_CUDA_TRY(cudaGetLastError());
    if (dst_memory == RE_MEMORY_HOST) {
        RE_CUDA_TRY(cudaMemcpyAsync(dst, out, 12 * P, cudaMemcpyDeviceToHost, st));
        RE_CUDA_TRY(cudaStreamSynchronize(st));
    }
    return clear_error();
}

RE_API re_status re_image_rmse(const float* candidate, const float* reference, uint64_t pixel_count,
                               float* out_rmse, void* stream) {
    if (candidate == nullptr || reference == nullptr || out_rmse == nullptr || pixel_count == 0)
        return set_error(RE_INVALID_ARGUMENT, "null argument or empty image");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DeviceBuffer acc;
    RE_CUDA_TRY(acc.reserve(sizeof(double)));
    RE_CUDA_TRY(cudaMemsetAsync(acc.ptr, 0, sizeof(double), st));
    const size_t blocks = std::min<size_t>((pixel_count + 255) / 256, 148 * 8);
    k_sqerr<<<unsigned(blocks), 256, 0, st>>>(candidate, reference, pixel_count, static_cast<double*>(acc.ptr));
    RE_CUDA_TRY(cudaGetLastError());
    double sum = 0.0;
    RE_CUDA_TRY(cudaMemcpyAsync(&sum, acc.ptr, sizeof(double), cudaMemcpyDeviceToHost, st));
    RE_CUDA_TRY(cudaStreamSynchronize(st));
    *out_rmse = static_cast<float>(std::sqrt(sum / (double(pixel_count) * 3.0)));
    return clear_error();
}

}  // extern "C"
