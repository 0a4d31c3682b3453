// Closest-hit and any-hit traversal of the child-pair BVH (device side).
//
// Semantics follow the reference's flattened-SAH traversal:
//   - ray validity: SoftwareRayIsValid (software_common.hlsli:69-75)
//   - slab test with a per-ray reciprocal: SoftwareIntersectBounds (:77-118)
//   - Moller-Trumbore test: SoftwareIntersectTriangle (:120-172), evaluated in
//     the same order as the CPU mirror (SoftwareGpu.cpp:661-703) with explicit
//     round-to-nearest operations, so t/u/v are bit-identical to the oracle
//   - culling, casts-shadow and ignored-(instance, primitive) rules and the
//     equal-distance lower-(instance, primitive) tie rule of
//     PbrTraceSoftwareIgnoringL6 (pbr_software_traversal.hlsli:288-535)
//   - near-first DFS with near pruning (`near > limit` once a hit exists,
//     `near >= limit` before): SoftwareGpu::Trace (SoftwareGpu.cpp:1529-1700)
// The closest hit is independent of visiting order (ties resolve by key), so
// the result equals the reference traversal; only near-ties at the 1-ulp level
// of the node slab arithmetic can prune differently.
#pragma once

#include "device_math.cuh"
#include "sah_builder.h"

namespace re {

// Alpha-mask data of a scene (re_scene_set_alpha_masks), read only for
// triangles flagged kTriAlphaMask: per leaf-ordered triangle its texture
// coordinates and material (tc0.xy, tc1.xy | tc2.xy, material, -), per
// material (alpha factor, cutoff, alpha layer, sampler id), and the alpha
// atlas, layers x height x width floats.
struct AlphaView {
    const float4* tc;
    const float4* materials;
    const float* atlas;
    uint32_t material_count;
    uint32_t width, height, layers;
    uint32_t sampler_id;     // the only sampler id a textured mapping may name
};

struct TraceSceneView {
    const float4* nodes;     // DeviceNode as 4 x float4
    const float4* tris;      // DeviceTriangle as 4 x float4
    uint32_t node_count;
    uint32_t tri_count;
    float root_lo[3];        // root box, tested first as the reference does
    float root_hi[3];
    const float4* wide;      // WideNode as 8 x float4 (null until built)
    uint32_t wide_count;
    uint32_t wide_stack;     // most stack entries a wide traversal holds
    const AlphaView* alpha;  // device copy; null when no alpha masks are set
    const float4* eight;     // Wide8Node as 16 x float4 (null until built)
    const float4* eightq;    // Wide8QNode as 6 x float4 (null until built)
    uint32_t eight_count;
    uint32_t eight_stack;    // most stack entries an eight-wide traversal holds
};

struct TraceRay {
    f3 o;
    f3 d;
    float tmin;
    float tmax;
};

struct TraceHit {
    float t;
    float u;
    float v;
    uint32_t tri;      // leaf-ordered triangle index, 0xffffffff on miss
    uint32_t front;
    uint32_t status;   // 0 ok, 1 invalid ray, 2 stack overflow, 3 malformed
};

struct TraceCounters {
    uint32_t node_tests;
    uint32_t tri_tests;
    uint32_t leaf_visits;
    uint32_t leaf_prims;
    uint32_t max_leaf;
    uint32_t max_stack;
    uint32_t node_bytes;  // node records fetched (64 B child pairs or 128 B wide nodes)
};

__device__ __forceinline__ bool ray_is_valid(const TraceRay& r) {
    const float len2 = dot(r.d, r.d);
    return finite3(r.o) && finite3(r.d) && isfinite(len2) && fabsf(len2 - 1.0f) <= 1.0e-4f &&
           !isnan(r.tmin) && !isnan(r.tmax) && r.tmin < r.tmax;
}

// Per-ray slab-test state.  inv = 1 / d per axis, so a zero component gives
// +inf or -inf; neg_* select which plane of an axis is entered first.
struct SlabRay {
    f3 o;
    f3 inv;
    bool neg_x, neg_y, neg_z;
    float tmin;
    float tmax;
};

__device__ __forceinline__ SlabRay make_slab_ray(const TraceRay& r) {
    SlabRay s;
    s.o = r.o;
    s.inv = mk(1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z);
    s.neg_x = signbit(s.inv.x);
    s.neg_y = signbit(s.inv.y);
    s.neg_z = signbit(s.inv.z);
    s.tmin = r.tmin;
    s.tmax = r.tmax;
    return s;
}

// Returns true when the box is entered inside the ray interval and within the
// current distance limit; near is clipped to tmin.
//
// Same distances as the reference's form (both plane distances, swapped when
// near > far; a zero direction component tested as inside / outside the slab,
// SoftwareGpu.cpp:610-640): for a box with lo <= hi the entry plane of an axis
// is lo when 1/d >= 0 and hi otherwise, and (plane - o) * inv is the value the
// swap would keep, rounding included.  For a zero component inv is +-inf:
// inside the slab the distances are -inf / +inf or NaN (origin on the plane),
// which the NaN-ignoring max / min leave out, as the reference's
// (-inf, +inf) does; outside, one distance is +inf (entry) or -inf (exit),
// a miss as in the reference.  slab_test_planes takes each axis's entry and
// exit planes already chosen; slab_test chooses them by the direction signs.
__device__ __forceinline__ bool slab_test_planes(const SlabRay& r, float xn, float xf, float yn, float yf,
                                                 float zn, float zf, float limit_cmp, float& near_out) {
    const float nx = __fmul_rn(__fsub_rn(xn, r.o.x), r.inv.x);
    const float fx = __fmul_rn(__fsub_rn(xf, r.o.x), r.inv.x);
    const float ny = __fmul_rn(__fsub_rn(yn, r.o.y), r.inv.y);
    const float fy = __fmul_rn(__fsub_rn(yf, r.o.y), r.inv.y);
    const float nz = __fmul_rn(__fsub_rn(zn, r.o.z), r.inv.z);
    const float fz = __fmul_rn(__fsub_rn(zf, r.o.z), r.inv.z);
    // Three-input max / min (sm_100), NaN inputs ignored as by fmaxf / fminf.
    // A NaN distance needs a zero direction component, so for a valid ray
    // (|d| = 1) at most two of a triple are NaN and these equal the chains
    // seeded with -inf / +inf.
    float tn, tf;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(tn) : "f"(nx), "f"(ny), "f"(nz));
    asm("min.f32 %0, %1, %2, %3;" : "=f"(tf) : "f"(fx), "f"(fy), "f"(fz));
    // tn < tMax, the reference's third condition, follows from the limit
    // test: the limit starts at tMax and only takes hit distances below it.
    // limit_cmp folds the reference's two forms into one compare: the limit
    // itself before a hit (near < limit), the next float above it after one
    // (near <= limit), see next_up.
    const bool within_limit = tn < limit_cmp;
    const bool hit = !(tf < tn) && tf > r.tmin && within_limit;
    near_out = fmaxf(tn, r.tmin);
    return hit;
}

__device__ __forceinline__ bool slab_test(const SlabRay& r, float x0, float x1, float y0, float y1,
                                          float z0, float z1, float limit_cmp, float& near_out) {
    return slab_test_planes(r, r.neg_x ? x1 : x0, r.neg_x ? x0 : x1, r.neg_y ? y1 : y0, r.neg_y ? y0 : y1,
                            r.neg_z ? z1 : z0, r.neg_z ? z0 : z1, limit_cmp, near_out);
}

// Conservative slab test (traversal modes 7 and 8): each plane distance is
// one fused multiply-add, plane * inv - o * inv, with o * inv precomputed
// per ray and axis, instead of the reference's (plane - o) * inv (two
// roundings, two instructions).  On axis a the fused form differs from the
// reference's value by at most 3 * 2^-24 |t| (the fma's rounding against
// the reference's two) + 2^-24 |o_a * inv_a| (the rounding of the product):
// a shift of the ray origin by under an ulp of o_a.  The test enters every
// box the reference enters by moving each entry plane's constant up and
// each exit plane's constant down by |o_a * inv_a| * 2^-22 + 2^-126 (per
// axis: a global bound would inflate every axis by the worst one, and a
// ray with a near-zero direction component would enter half the scene), and
// by widening what the distances are compared against, rounded upward:
//   - the exit distance by |exit| * 2^-21;
//   - the distance limit by |limit| * 2^-21 + 2^-126 (widen_limit).
// A zero direction component makes o * inv infinite or NaN; its plane
// distances are then NaN or -inf (entry) / +inf (exit), which the
// NaN-ignoring max / min and the compares treat as "no constraint": such
// rays may enter boxes the reference rejects, never the reverse.  Rays must
// have tmin >= 0 (every wavefront ray does).  Entering extra boxes only adds
// node visits and triangle tests, whose arithmetic is the reference's, so
// closest hits and visibility are the reference's except where the
// reference's own rounding rejects a box the ray enters (a ray clipping a
// box corner within a few ulps at the triangle it hits).
struct SlabRayC {
    f3 inv;
    f3 oin;  // o * inv per axis, moved up: entry planes
    f3 oif;  // o * inv per axis, moved down: exit planes
    float tmin;
    bool neg_x, neg_y, neg_z;
};

__device__ __forceinline__ void slab_constants(float o, float inv, float& on, float& of) {
    const float oi = __fmul_rn(o, inv);
    const float m = __fmaf_ru(fabsf(oi), 0x1p-22f, 0x1p-126f);
    on = __fadd_ru(oi, m);
    of = __fadd_rd(oi, -m);
}

__device__ __forceinline__ SlabRayC make_slab_ray_c(const TraceRay& r) {
    SlabRayC s;
    s.inv = mk(1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z);
    slab_constants(r.o.x, s.inv.x, s.oin.x, s.oif.x);
    slab_constants(r.o.y, s.inv.y, s.oin.y, s.oif.y);
    slab_constants(r.o.z, s.inv.z, s.oin.z, s.oif.z);
    s.neg_x = signbit(s.inv.x);
    s.neg_y = signbit(s.inv.y);
    s.neg_z = signbit(s.inv.z);
    s.tmin = r.tmin;
    return s;
}

// The limit a conservative near distance is compared against: the exact
// compare limit (tMax, or next_up of the closest hit) widened upward.
__device__ __forceinline__ float widen_limit(float limit_cmp) {
    return __fadd_ru(__fmaf_ru(fabsf(limit_cmp), 0x1p-21f, limit_cmp), 0x1p-126f);
}

__device__ __forceinline__ bool slab_test_planes_c(const SlabRayC& r, float xn, float xf, float yn, float yf,
                                                   float zn, float zf, float limit_c, float& near_out) {
    const float nx = __fmaf_rn(xn, r.inv.x, -r.oin.x);
    const float fx = __fmaf_rn(xf, r.inv.x, -r.oif.x);
    const float ny = __fmaf_rn(yn, r.inv.y, -r.oin.y);
    const float fy = __fmaf_rn(yf, r.inv.y, -r.oif.y);
    const float nz = __fmaf_rn(zn, r.inv.z, -r.oin.z);
    const float fz = __fmaf_rn(zf, r.inv.z, -r.oif.z);
    float tn, tf;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(tn) : "f"(nx), "f"(ny), "f"(nz));
    asm("min.f32 %0, %1, %2, %3;" : "=f"(tf) : "f"(fx), "f"(fy), "f"(fz));
    const float tfw = __fmaf_ru(fabsf(tf), 0x1p-21f, tf);
    near_out = fmaxf(tn, r.tmin);
    return tfw >= near_out && near_out < limit_c;
}

__device__ __forceinline__ bool slab_test_c(const SlabRayC& r, float x0, float x1, float y0, float y1, float z0,
                                            float z1, float limit_c, float& near_out) {
    return slab_test_planes_c(r, r.neg_x ? x1 : x0, r.neg_x ? x0 : x1, r.neg_y ? y1 : y0, r.neg_y ? y0 : y1,
                              r.neg_z ? z1 : z0, r.neg_z ? z0 : z1, limit_c, near_out);
}

// The slab form of a loop: exact (the reference's arithmetic) or
// conservative (C).
template <bool C>
struct SlabOf {
    using Ray = SlabRay;
    static __device__ __forceinline__ Ray make(const TraceRay& r) { return make_slab_ray(r); }
    static __device__ __forceinline__ float limit(float limit_cmp, const Ray&) { return limit_cmp; }
    static __device__ __forceinline__ bool planes(const Ray& r, float xn, float xf, float yn, float yf, float zn,
                                                  float zf, float lim, float& near_out) {
        return slab_test_planes(r, xn, xf, yn, yf, zn, zf, lim, near_out);
    }
    static __device__ __forceinline__ bool box(const Ray& r, float x0, float x1, float y0, float y1, float z0,
                                               float z1, float lim, float& near_out) {
        return slab_test(r, x0, x1, y0, y1, z0, z1, lim, near_out);
    }
};
template <>
struct SlabOf<true> {
    using Ray = SlabRayC;
    static __device__ __forceinline__ Ray make(const TraceRay& r) { return make_slab_ray_c(r); }
    static __device__ __forceinline__ float limit(float limit_cmp, const Ray&) { return widen_limit(limit_cmp); }
    static __device__ __forceinline__ bool planes(const Ray& r, float xn, float xf, float yn, float yf, float zn,
                                                  float zf, float lim, float& near_out) {
        return slab_test_planes_c(r, xn, xf, yn, yf, zn, zf, lim, near_out);
    }
    static __device__ __forceinline__ bool box(const Ray& r, float x0, float x1, float y0, float y1, float z0,
                                               float z1, float lim, float& near_out) {
        return slab_test_c(r, x0, x1, y0, y1, z0, z1, lim, near_out);
    }
};

// The six plane vectors of a four-wide node (WideNode: lo / hi per axis for
// the four children), loaded as entry and exit planes for this ray: the
// direction signs pick which vector of each axis is loaded as which, so the
// per-child slab tests need no selects.
struct WidePlanes {
    float4 xn, xf, yn, yf, zn, zf;
};

template <class R>
__device__ __forceinline__ WidePlanes load_wide_planes(const float4* w, const R& r) {
    const int sx = r.neg_x ? 1 : 0, sy = r.neg_y ? 1 : 0, sz = r.neg_z ? 1 : 0;
    WidePlanes p;
    p.xn = __ldg(w + sx);
    p.xf = __ldg(w + (1 - sx));
    p.yn = __ldg(w + (2 + sy));
    p.yf = __ldg(w + (3 - sy));
    p.zn = __ldg(w + (4 + sz));
    p.zf = __ldg(w + (5 - sz));
    return p;
}

// The next float above a finite x (for either zero the smallest positive
// subnormal): `y <= x` is `y < next_up(x)` for every finite y, so a
// traversal keeps one compare limit -- tMax before its first hit (`< tMax`),
// next_up(t) after it (`<= t`) -- instead of choosing a compare per test.
__device__ __forceinline__ float next_up(float x) {
    const uint32_t u = __float_as_uint(x);
    return x >= 0.0f ? __uint_as_float((u & 0x7fffffffu) + 1u) : __uint_as_float(u - 1u);
}

// Moller-Trumbore in the CPU mirror's exact operation order.
__device__ __forceinline__ bool tri_test(const TraceRay& r, float4 p0, float4 e1v, float4 e2v,
                                         float limit_cmp, float& t_out, float& u_out,
                                         float& v_out, bool& front) {
    const float e1x = e1v.x, e1y = e1v.y, e1z = e1v.z;
    const float e2x = e2v.x, e2y = e2v.y, e2z = e2v.z;
    // p = cross(d, e2)
    const float px = __fsub_rn(__fmul_rn(r.d.y, e2z), __fmul_rn(r.d.z, e2y));
    const float py = __fsub_rn(__fmul_rn(r.d.z, e2x), __fmul_rn(r.d.x, e2z));
    const float pz = __fsub_rn(__fmul_rn(r.d.x, e2y), __fmul_rn(r.d.y, e2x));
    const float det = __fadd_rn(__fadd_rn(__fmul_rn(e1x, px), __fmul_rn(e1y, py)), __fmul_rn(e1z, pz));
    if (det == 0.0f || !isfinite(det)) return false;
    const float inv = __frcp_rn(det);
    const float tx = __fsub_rn(r.o.x, p0.x), ty = __fsub_rn(r.o.y, p0.y), tz = __fsub_rn(r.o.z, p0.z);
    const float u = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(tx, px), __fmul_rn(ty, py)), __fmul_rn(tz, pz)), inv);
    if (!(u >= 0.0f && u <= 1.0f)) return false;
    // q = cross(tvec, e1)
    const float qx = __fsub_rn(__fmul_rn(ty, e1z), __fmul_rn(tz, e1y));
    const float qy = __fsub_rn(__fmul_rn(tz, e1x), __fmul_rn(tx, e1z));
    const float qz = __fsub_rn(__fmul_rn(tx, e1y), __fmul_rn(ty, e1x));
    const float v = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(r.d.x, qx), __fmul_rn(r.d.y, qy)), __fmul_rn(r.d.z, qz)), inv);
    if (!(v >= 0.0f && __fadd_rn(u, v) <= 1.0f)) return false;
    const float t = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(e2x, qx), __fmul_rn(e2y, qy)), __fmul_rn(e2z, qz)), inv);
    const bool within_limit = t < limit_cmp;
    if (!(isfinite(t) && t > r.tmin && t < r.tmax && within_limit)) return false;
    t_out = t;
    u_out = u;
    v_out = v;
    front = det > 0.0f;
    return true;
}

// Alpha-masked candidate acceptance (pbr_software_traversal.hlsli:207-240,
// 430-470): 1 keeps the candidate, 0 skips it (alpha below the material's
// cutoff), -1 is an invalid mapping (material out of range, an unknown alpha
// layer or sampler), which ends the traversal as malformed.  alpha = the
// material's alpha factor, times the atlas texel at the interpolated
// texture coordinate (nearest, clamped to the edge) when the material names
// an alpha layer.  Out of line: only masked triangles call it.
static __device__ __noinline__ int alpha_accept(const AlphaView* a, uint32_t ti, float u, float v) {
    if (a == nullptr) return -1;
    const float4 t0 = __ldg(a->tc + size_t(ti) * 2u), t1 = __ldg(a->tc + size_t(ti) * 2u + 1u);
    const uint32_t mat = __float_as_uint(t1.z);
    if (mat >= a->material_count) return -1;
    const float4 m = __ldg(a->materials + mat);
    const uint32_t layer = __float_as_uint(m.z), sampler = __float_as_uint(m.w);
    float alpha = m.x;
    if (layer == 0xffffffffu) {
        if (sampler != 0xffffffffu) return -1;
    } else if (layer >= a->layers || sampler != a->sampler_id) {
        return -1;
    } else {
        const float w0 = __fsub_rn(__fsub_rn(1.0f, u), v);
        const float su = __fadd_rn(__fadd_rn(__fmul_rn(w0, t0.x), __fmul_rn(u, t0.z)), __fmul_rn(v, t1.x));
        const float sv = __fadd_rn(__fadd_rn(__fmul_rn(w0, t0.y), __fmul_rn(u, t0.w)), __fmul_rn(v, t1.y));
        const int i = min(max(int(floorf(__fmul_rn(su, float(a->width)))), 0), int(a->width) - 1);
        const int j = min(max(int(floorf(__fmul_rn(sv, float(a->height)))), 0), int(a->height) - 1);
        alpha = __fmul_rn(alpha, __ldg(a->atlas + (size_t(layer) * a->height + size_t(j)) * a->width + size_t(i)));
    }
    return alpha < m.y ? 0 : 1;
}

// Stack entry: ref | (leaf count << 28); near distance as float bits.
constexpr uint32_t kLeafShift = 28u;
constexpr uint32_t kRefMask = (1u << kLeafShift) - 1u;
static_assert(kLeafShift == kWideLeafShift, "wide node entries are stack entries");

struct TraceOptions {
    uint32_t ignore_instance;   // 0xffffffff: none
    uint32_t ignore_primitive;
    bool shadow;                // any-hit visibility query (casts-shadow rule)
};

template <bool ANY, bool COUNT, int STACK>
__device__ __forceinline__ TraceHit trace(const TraceSceneView& s, const TraceRay& ray,
                                          const TraceOptions& opt, TraceCounters* cnt) {
    TraceHit h;
    h.t = ray.tmax;
    h.u = 0.0f;
    h.v = 0.0f;
    h.tri = 0xffffffffu;
    h.front = 0u;
    h.status = 0u;
    if (!ray_is_valid(ray)) {
        h.status = 1u;
        return h;
    }
    if (s.node_count == 0u) return h;
    const SlabRay sr = make_slab_ray(ray);
    uint2 stack[STACK];
    int sp = 0;
    bool found = false;
    float limit = ray.tmax;
    float limit_cmp = ray.tmax;  // see next_up
    uint32_t best_i = 0xffffffffu, best_p = 0xffffffffu;
    uint32_t cur = 0u;         // interior node 0 = root
    uint32_t cur_count = 0u;   // 0: interior, >0: leaf with that many triangles
    // The reference tests the root box first (SoftwareGpu.cpp:1569-1580); a
    // ray that misses it never fetches a node.
    if (COUNT) cnt->node_tests += 1u;
    {
        float root_near;
        if (!slab_test(sr, s.root_lo[0], s.root_hi[0], s.root_lo[1], s.root_hi[1], s.root_lo[2], s.root_hi[2],
                       ray.tmax, root_near))
            return h;
    }
    uint32_t steps = 0u;
    const uint32_t max_steps = s.node_count * 4u + 8u;
    while (true) {
        if (++steps > max_steps) {  // malformed (cyclic) tree guard
            h.status = 3u;
            h.tri = 0xffffffffu;
            return h;
        }
        if (cur_count == 0u) {
            const float4* n = s.nodes + size_t(cur) * 4u;
            const float4 a = __ldg(n + 0);
            const float4 b = __ldg(n + 1);
            const float4 c = __ldg(n + 2);
            const uint4 d = __ldg(reinterpret_cast<const uint4*>(n + 3));
            float nl, nr;
            const bool hl = slab_test(sr, a.x, a.y, a.z, a.w, b.x, b.y, limit_cmp, nl);
            const bool hr = slab_test(sr, b.z, b.w, c.x, c.y, c.z, c.w, limit_cmp, nr);
            if (COUNT) {
                cnt->node_tests += 2u;
                cnt->node_bytes += uint32_t(sizeof(DeviceNode));
            }
            if (hl && hr) {
                // Near first; equal near -> left (lower pre-order index) first.
                const bool left_first = nl < nr || !(nr < nl);
                const uint32_t far_ref = left_first ? (d.y | (d.w << kLeafShift)) : (d.x | (d.z << kLeafShift));
                const float far_near = left_first ? nr : nl;
                if (sp >= STACK) {
                    h.status = 2u;
                    h.tri = 0xffffffffu;
                    return h;
                }
                stack[sp++] = make_uint2(far_ref, __float_as_uint(far_near));
                if (COUNT) cnt->max_stack = max(cnt->max_stack, uint32_t(sp));
                cur = left_first ? d.x : d.y;
                cur_count = left_first ? d.z : d.w;
                continue;
            }
            if (hl) { cur = d.x; cur_count = d.z; continue; }
            if (hr) { cur = d.y; cur_count = d.w; continue; }
        } else {
            if (COUNT) {
                cnt->leaf_visits += 1u;
                cnt->leaf_prims += cur_count;
                cnt->max_leaf = max(cnt->max_leaf, cur_count);
            }
            for (uint32_t k = 0; k < cur_count; ++k) {
                const uint32_t ti = cur + k;
                const float4* tp = s.tris + size_t(ti) * 4u;
                const float4 p0 = __ldg(tp + 0), e1 = __ldg(tp + 1), e2 = __ldg(tp + 2);
                const uint2 key = make_uint2(__float_as_uint(e1.w), __float_as_uint(e2.w));
                if (key.x == opt.ignore_instance && key.y == opt.ignore_primitive) continue;
                const uint32_t flags = __float_as_uint(p0.w);
                if (opt.shadow && (flags & kTriCastsShadow) == 0u) continue;
                if (COUNT) cnt->tri_tests += 1u;
                float t, u, v;
                bool front;
                if (!tri_test(ray, p0, e1, e2, limit_cmp, t, u, v, front)) continue;
                if (!front && (flags & kTriDoubleSided) == 0u) continue;
                if ((flags & kTriAlphaMask) != 0u) {
                    const int acc = alpha_accept(s.alpha, ti, u, v);
                    if (acc < 0) {
                        h.status = 3u;
                        h.tri = 0xffffffffu;
                        return h;
                    }
                    if (acc == 0) continue;
                }
                if (ANY) {
                    h.t = t; h.u = u; h.v = v; h.tri = ti; h.front = front ? 1u : 0u;
                    return h;
                }
                const bool lower_key = t == limit && (key.x < best_i || (key.x == best_i && key.y < best_p));
                if (!found || t < limit || lower_key) {
                    found = true;
                    limit = t;
                    limit_cmp = next_up(t);
                    h.t = t; h.u = u; h.v = v; h.tri = ti; h.front = front ? 1u : 0u;
                    best_i = key.x;
                    best_p = key.y;
                }
            }
        }
        // Pop the next entry that is still within the distance limit.
        bool next = false;
        while (sp > 0) {
            const uint2 e = stack[--sp];
            const float nn = __uint_as_float(e.y);
            if (nn >= limit_cmp) continue;
            cur = e.x & kRefMask;
            cur_count = e.x >> kLeafShift;
            next = true;
            break;
        }
        if (!next) break;
    }
    return h;
}

// While-while traversal with postponed leaves (Aila and Laine, "Understanding
// the Efficiency of Ray Traversal on GPUs", HPG 2009).  A lane that reaches a
// leaf parks it and keeps descending interior nodes until every active lane
// of its warp holds a leaf; the warp then tests triangles together, so node
// fetches and triangle tests each run with most lanes busy instead of
// alternating between two half-empty branches.  Each ray still visits nodes
// near-first with the same slab and triangle arithmetic; a parked leaf's hits
// shorten the distance limit later than in `trace`, so a ray may visit more
// nodes, and the closest hit (ties by key) is `trace`'s.  For any-hit rays
// the occluder reported may differ from `trace`'s; visibility does not.  The
// warp votes use the lanes active at the vote, so divergent callers work.
template <bool ANY, int STACK>
__device__ __forceinline__ TraceHit trace_ww(const TraceSceneView& s, const TraceRay& ray, const TraceOptions& opt) {
    TraceHit h;
    h.t = ray.tmax;
    h.u = 0.0f;
    h.v = 0.0f;
    h.tri = 0xffffffffu;
    h.front = 0u;
    h.status = 0u;
    if (!ray_is_valid(ray)) {
        h.status = 1u;
        return h;
    }
    if (s.node_count == 0u) return h;
    const SlabRay sr = make_slab_ray(ray);
    {
        float root_near;
        if (!slab_test(sr, s.root_lo[0], s.root_hi[0], s.root_lo[1], s.root_hi[1], s.root_lo[2], s.root_hi[2],
                       ray.tmax, root_near))
            return h;
    }
    uint2 stack[STACK];
    int sp = 0;
    bool found = false;
    float limit = ray.tmax;
    float limit_cmp = ray.tmax;  // see next_up
    uint32_t best_i = 0xffffffffu, best_p = 0xffffffffu;
    uint32_t cur = 0u, cur_count = 0u;  // next node to visit (leaf when cur_count > 0)
    bool has_cur = true;
    uint32_t leaf = 0u, leaf_count = 0u;  // parked leaf (none when leaf_count == 0)
    uint32_t steps = 0u;
    const uint32_t max_steps = s.node_count * 4u + 8u;
    // Next stack entry still within the distance limit.
    auto pop = [&]() {
        while (sp > 0) {
            const uint2 e = stack[--sp];
            const float nn = __uint_as_float(e.y);
            if (nn >= limit_cmp) continue;
            cur = e.x & kRefMask;
            cur_count = e.x >> kLeafShift;
            return true;
        }
        return false;
    };
    while (has_cur || leaf_count != 0u) {
        // Interior nodes, parking the first leaf met.
        while (has_cur && cur_count == 0u) {
            if (++steps > max_steps) {  // malformed (cyclic) tree guard
                h.status = 3u;
                h.tri = 0xffffffffu;
                return h;
            }
            const float4* n = s.nodes + size_t(cur) * 4u;
            const float4 a = __ldg(n + 0);
            const float4 b = __ldg(n + 1);
            const float4 c = __ldg(n + 2);
            const uint4 d = __ldg(reinterpret_cast<const uint4*>(n + 3));
            float nl, nr;
            const bool hl = slab_test(sr, a.x, a.y, a.z, a.w, b.x, b.y, limit_cmp, nl);
            const bool hr = slab_test(sr, b.z, b.w, c.x, c.y, c.z, c.w, limit_cmp, nr);
            if (hl && hr) {
                const bool left_first = nl < nr || !(nr < nl);
                if (sp >= STACK) {
                    h.status = 2u;
                    h.tri = 0xffffffffu;
                    return h;
                }
                stack[sp++] = make_uint2(left_first ? (d.y | (d.w << kLeafShift)) : (d.x | (d.z << kLeafShift)),
                                         __float_as_uint(left_first ? nr : nl));
                cur = left_first ? d.x : d.y;
                cur_count = left_first ? d.z : d.w;
            } else if (hl) {
                cur = d.x;
                cur_count = d.z;
            } else if (hr) {
                cur = d.y;
                cur_count = d.w;
            } else {
                has_cur = pop();
            }
            if (has_cur && cur_count != 0u && leaf_count == 0u) {
                leaf = cur;
                leaf_count = cur_count;
                has_cur = pop();
            }
            if (!__any_sync(__activemask(), leaf_count == 0u)) break;
        }
        // Leaves: the parked one, then the next node while it is a leaf.
        while (true) {
            if (leaf_count == 0u) {
                if (!(has_cur && cur_count != 0u)) break;
                leaf = cur;
                leaf_count = cur_count;
                has_cur = pop();
            }
            for (uint32_t k = 0; k < leaf_count; ++k) {
                const uint32_t ti = leaf + k;
                const float4* tp = s.tris + size_t(ti) * 4u;
                const float4 p0 = __ldg(tp + 0), e1 = __ldg(tp + 1), e2 = __ldg(tp + 2);
                const uint2 key = make_uint2(__float_as_uint(e1.w), __float_as_uint(e2.w));
                if (key.x == opt.ignore_instance && key.y == opt.ignore_primitive) continue;
                const uint32_t flags = __float_as_uint(p0.w);
                if (opt.shadow && (flags & kTriCastsShadow) == 0u) continue;
                float t, u, v;
                bool front;
                if (!tri_test(ray, p0, e1, e2, limit_cmp, t, u, v, front)) continue;
                if (!front && (flags & kTriDoubleSided) == 0u) continue;
                if ((flags & kTriAlphaMask) != 0u) {
                    const int acc = alpha_accept(s.alpha, ti, u, v);
                    if (acc < 0) {
                        h.status = 3u;
                        h.tri = 0xffffffffu;
                        return h;
                    }
                    if (acc == 0) continue;
                }
                if (ANY) {
                    h.t = t; h.u = u; h.v = v; h.tri = ti; h.front = front ? 1u : 0u;
                    return h;
                }
                const bool lower_key = t == limit && (key.x < best_i || (key.x == best_i && key.y < best_p));
                if (!found || t < limit || lower_key) {
                    found = true;
                    limit = t;
                    limit_cmp = next_up(t);
                    h.t = t; h.u = u; h.v = v; h.tri = ti; h.front = front ? 1u : 0u;
                    best_i = key.x;
                    best_p = key.y;
                }
            }
            leaf_count = 0u;
        }
    }
    return h;
}

// Compare-exchange of two (near, entry) pairs: nearer first.
__device__ __forceinline__ void order_pair(float& na, uint32_t& ea, float& nb, uint32_t& eb) {
    if (nb < na) {
        const float tn = na;
        na = nb;
        nb = tn;
        const uint32_t te = ea;
        ea = eb;
        eb = te;
    }
}

// Descent from a four-wide node whose entered children carry finite near
// distances (the others +inf): the children ordered near-first by a
// five-comparator network, the nearest visited next (cur / cur_count), the
// others pushed farthest first.  Returns 1 after a descent, 0 when no child
// was entered, -1 when the stack would overflow.  (Any-hit rays take the
// same order: pushing them unsorted was measured slower.)
template <int STACK>
__device__ __forceinline__ int wide_descend(float n0, uint32_t e0, float n1, uint32_t e1, float n2, uint32_t e2,
                                            float n3, uint32_t e3, uint2 (&stack)[STACK], int& sp, uint32_t& cur,
                                            uint32_t& cur_count) {
    order_pair(n0, e0, n1, e1);
    order_pair(n2, e2, n3, e3);
    order_pair(n0, e0, n2, e2);
    order_pair(n1, e1, n3, e3);
    order_pair(n1, e1, n2, e2);
    if (n0 == INFINITY) return 0;
    const int pushes = (n1 != INFINITY) + (n2 != INFINITY) + (n3 != INFINITY);
    if (sp + pushes > STACK) return -1;
    if (n3 != INFINITY) stack[sp++] = make_uint2(e3, __float_as_uint(n3));
    if (n2 != INFINITY) stack[sp++] = make_uint2(e2, __float_as_uint(n2));
    if (n1 != INFINITY) stack[sp++] = make_uint2(e1, __float_as_uint(n1));
    cur = e0 & kRefMask;
    cur_count = e0 >> kLeafShift;
    return 1;
}

// Four-wide traversal (WideNode).  One fetch of 128 bytes tests up to four
// child boxes with the reference's slab arithmetic; the entered children are
// ordered near-first (wide_descend), so every ray still
// visits boxes near-first with the same pruning rule (`near > limit` once a
// hit exists, `near >= limit` before) and tests the same triangles with the
// same arithmetic.  The closest hit (ties by key) is `trace`'s; for any-hit
// rays the occluder reported may differ, visibility does not.  Half as many
// dependent node fetches per ray as the child-pair layout, each twice as
// wide.
template <bool ANY, bool COUNT, int STACK, bool C = false>
__device__ __forceinline__ TraceHit trace_wide(const TraceSceneView& s, const TraceRay& ray,
                                               const TraceOptions& opt, TraceCounters* cnt) {
    TraceHit h;
    h.t = ray.tmax;
    h.u = 0.0f;
    h.v = 0.0f;
    h.tri = 0xffffffffu;
    h.front = 0u;
    h.status = 0u;
    if (!ray_is_valid(ray)) {
        h.status = 1u;
        return h;
    }
    if (s.wide_count == 0u) return h;
    using S = SlabOf<C>;
    const typename S::Ray sr = S::make(ray);
    if (COUNT) cnt->node_tests += 1u;
    {
        float root_near;
        if (!S::box(sr, s.root_lo[0], s.root_hi[0], s.root_lo[1], s.root_hi[1], s.root_lo[2], s.root_hi[2],
                    S::limit(ray.tmax, sr), root_near))
            return h;
    }
    uint2 stack[STACK];
    int sp = 0;
    bool found = false;
    float limit = ray.tmax;
    float limit_cmp = ray.tmax;  // see next_up
    float lim = S::limit(ray.tmax, sr);  // what box near distances are compared against
    uint32_t best_i = 0xffffffffu, best_p = 0xffffffffu;
    uint32_t cur = 0u, cur_count = 0u;
    uint32_t steps = 0u;
    const uint32_t max_steps = s.wide_count * 5u + 8u;
    while (true) {
        if (++steps > max_steps) {  // malformed (cyclic) tree guard
            h.status = 3u;
            h.tri = 0xffffffffu;
            return h;
        }
        bool next = false;
        if (cur_count == 0u) {
            const float4* w = s.wide + size_t(cur) * 8u;
            const WidePlanes pl = load_wide_planes(w, sr);
            const uint4 ent = __ldg(reinterpret_cast<const uint4*>(w + 6));
            if (COUNT) cnt->node_bytes += uint32_t(sizeof(WideNode));
            float n0 = INFINITY, n1 = INFINITY, n2 = INFINITY, n3 = INFINITY;
            // A child's entry matters only when it is entered (finite near):
            // the others sort last and are neither visited nor pushed.
            const uint32_t e0 = ent.x, e1 = ent.y, e2 = ent.z, e3 = ent.w;
            float nn;
            if (!COUNT || ent.x != kWideEmpty) {  // an empty slot's +inf box is never entered
                if (COUNT) cnt->node_tests += 1u;
                if (S::planes(sr, pl.xn.x, pl.xf.x, pl.yn.x, pl.yf.x, pl.zn.x, pl.zf.x, lim, nn)) {
                    n0 = nn;
                }
            }
            if (!COUNT || ent.y != kWideEmpty) {  // an empty slot's +inf box is never entered
                if (COUNT) cnt->node_tests += 1u;
                if (S::planes(sr, pl.xn.y, pl.xf.y, pl.yn.y, pl.yf.y, pl.zn.y, pl.zf.y, lim, nn)) {
                    n1 = nn;
                }
            }
            if (!COUNT || ent.z != kWideEmpty) {  // an empty slot's +inf box is never entered
                if (COUNT) cnt->node_tests += 1u;
                if (S::planes(sr, pl.xn.z, pl.xf.z, pl.yn.z, pl.yf.z, pl.zn.z, pl.zf.z, lim, nn)) {
                    n2 = nn;
                }
            }
            if (!COUNT || ent.w != kWideEmpty) {  // an empty slot's +inf box is never entered
                if (COUNT) cnt->node_tests += 1u;
                if (S::planes(sr, pl.xn.w, pl.xf.w, pl.yn.w, pl.yf.w, pl.zn.w, pl.zf.w, lim, nn)) {
                    n3 = nn;
                }
            }
            // Entered children have finite near distances (near < tMax);
            // the others sort last at +inf.
            const int down = wide_descend<STACK>(n0, e0, n1, e1, n2, e2, n3, e3, stack, sp, cur, cur_count);
            if (down < 0) {
                h.status = 2u;
                h.tri = 0xffffffffu;
                return h;
            }
            if (down > 0) {
                if (COUNT) cnt->max_stack = max(cnt->max_stack, uint32_t(sp));
                next = true;
            }
        } else {
            if (COUNT) {
                cnt->leaf_visits += 1u;
                cnt->leaf_prims += cur_count;
                cnt->max_leaf = max(cnt->max_leaf, cur_count);
            }
            for (uint32_t k = 0; k < cur_count; ++k) {
                const uint32_t ti = cur + k;
                const float4* tp = s.tris + size_t(ti) * 4u;
                const float4 p0 = __ldg(tp + 0), e1 = __ldg(tp + 1), e2 = __ldg(tp + 2);
                const uint2 key = make_uint2(__float_as_uint(e1.w), __float_as_uint(e2.w));
                if (key.x == opt.ignore_instance && key.y == opt.ignore_primitive) continue;
                const uint32_t flags = __float_as_uint(p0.w);
                if (opt.shadow && (flags & kTriCastsShadow) == 0u) continue;
                if (COUNT) cnt->tri_tests += 1u;
                float t, u, v;
                bool front;
                if (!tri_test(ray, p0, e1, e2, limit_cmp, t, u, v, front)) continue;
                if (!front && (flags & kTriDoubleSided) == 0u) continue;
                if ((flags & kTriAlphaMask) != 0u) {
                    const int acc = alpha_accept(s.alpha, ti, u, v);
                    if (acc < 0) {
                        h.status = 3u;
                        h.tri = 0xffffffffu;
                        return h;
                    }
                    if (acc == 0) continue;
                }
                if (ANY) {
                    h.t = t; h.u = u; h.v = v; h.tri = ti; h.front = front ? 1u : 0u;
                    return h;
                }
                const bool lower_key = t == limit && (key.x < best_i || (key.x == best_i && key.y < best_p));
                if (!found || t < limit || lower_key) {
                    found = true;
                    limit = t;
                    limit_cmp = next_up(t);
                    lim = S::limit(limit_cmp, sr);
                    h.t = t; h.u = u; h.v = v; h.tri = ti; h.front = front ? 1u : 0u;
                    best_i = key.x;
                    best_p = key.y;
                }
            }
        }
        if (next) continue;
        // Pop the next entry that is still within the distance limit.
        while (sp > 0) {
            const uint2 e = stack[--sp];
            const float pn = __uint_as_float(e.y);
            if (pn >= lim) continue;
            cur = e.x & kRefMask;
            cur_count = e.x >> kLeafShift;
            next = true;
            break;
        }
        if (!next) break;
    }
    return h;
}

// ---------------------------------------------------------------------------
// Eight-wide traversal (Wide8Node, or Wide8QNode with Q): one node fetch
// tests up to eight child boxes -- the plain form reads the exact boxes (14
// aligned 16-byte loads), the compressed form six 16-byte loads and decodes
// each bound as origin + q * 2^e added with rounding toward -inf (lower
// bounds) or +inf (upper bounds), so every decoded box contains the exact
// one.  The entered children are ordered near-first by Batcher's odd-even
// merge network (19 comparators); the nearest is visited next, the others
// pushed farthest first.  The slab and triangle arithmetic are the
// reference's, so the closest hit (ties by key) and any-hit visibility are
// trace's; conservative boxes can only add node visits.
// ---------------------------------------------------------------------------
struct Eight {
    float n[8];
    uint32_t e[8];
};

__device__ __forceinline__ void ce8(Eight& s, int a, int b) {
    if (s.n[b] < s.n[a]) {
        const float tn = s.n[a];
        s.n[a] = s.n[b];
        s.n[b] = tn;
        const uint32_t te = s.e[a];
        s.e[a] = s.e[b];
        s.e[b] = te;
    }
}

__device__ __forceinline__ void sort8(Eight& s) {
    ce8(s, 0, 1); ce8(s, 2, 3); ce8(s, 4, 5); ce8(s, 6, 7);
    ce8(s, 0, 2); ce8(s, 1, 3); ce8(s, 4, 6); ce8(s, 5, 7);
    ce8(s, 1, 2); ce8(s, 5, 6);
    ce8(s, 0, 4); ce8(s, 1, 5); ce8(s, 2, 6); ce8(s, 3, 7);
    ce8(s, 2, 4); ce8(s, 3, 5);
    ce8(s, 1, 2); ce8(s, 3, 4); ce8(s, 5, 6);
}

// Byte k (0..7) of the 8-byte run held in two words.
__device__ __forceinline__ float qbyte(uint32_t lo4, uint32_t hi4, int k) {
    const uint32_t w = k < 4 ? lo4 : hi4;
    return __uint2float_rn((w >> (8 * (k & 3))) & 0xffu);
}

template <bool ANY, bool COUNT, int STACK, bool Q>
__device__ __forceinline__ TraceHit trace_eight(const TraceSceneView& s, const TraceRay& ray, const TraceOptions& opt,
                                                TraceCounters* cnt) {
    TraceHit h;
    h.t = ray.tmax;
    h.u = 0.0f;
    h.v = 0.0f;
    h.tri = 0xffffffffu;
    h.front = 0u;
    h.status = 0u;
    if (!ray_is_valid(ray)) {
        h.status = 1u;
        return h;
    }
    if (s.eight_count == 0u) return h;
    const SlabRay sr = make_slab_ray(ray);
    if (COUNT) cnt->node_tests += 1u;
    {
        float root_near;
        if (!slab_test(sr, s.root_lo[0], s.root_hi[0], s.root_lo[1], s.root_hi[1], s.root_lo[2], s.root_hi[2],
                       ray.tmax, root_near))
            return h;
    }
    uint2 stack[STACK];
    int sp = 0;
    bool found = false;
    float limit = ray.tmax;
    float limit_cmp = ray.tmax;
    uint32_t best_i = 0xffffffffu, best_p = 0xffffffffu;
    uint32_t cur = 0u, cur_count = 0u;
    uint32_t steps = 0u;
    const uint32_t max_steps = s.eight_count * 9u + 8u;
    while (true) {
        if (++steps > max_steps) {  // malformed (cyclic) tree guard
            h.status = 3u;
            h.tri = 0xffffffffu;
            return h;
        }
        bool next = false;
        if (cur_count == 0u) {
            Eight c;
            uint4 ea, eb;
            if (Q) {
                const float4* w = s.eightq + size_t(cur) * 6u;
                const float4 hd = __ldg(w);
                const uint4 ax = __ldg(reinterpret_cast<const uint4*>(w + 1));
                const uint4 ay = __ldg(reinterpret_cast<const uint4*>(w + 2));
                const uint4 az = __ldg(reinterpret_cast<const uint4*>(w + 3));
                ea = __ldg(reinterpret_cast<const uint4*>(w + 4));
                eb = __ldg(reinterpret_cast<const uint4*>(w + 5));
                const uint32_t ex = __float_as_uint(hd.w);
                const float scx = __uint_as_float((ex & 0xffu) << 23);
                const float scy = __uint_as_float(((ex >> 8) & 0xffu) << 23);
                const float scz = __uint_as_float(((ex >> 16) & 0xffu) << 23);
                if (COUNT) cnt->node_bytes += uint32_t(sizeof(Wide8QNode));
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const float lx = __fadd_rd(hd.x, __fmul_rn(qbyte(ax.x, ax.y, k), scx));
                    const float hx = __fadd_ru(hd.x, __fmul_rn(qbyte(ax.z, ax.w, k), scx));
                    const float ly = __fadd_rd(hd.y, __fmul_rn(qbyte(ay.x, ay.y, k), scy));
                    const float hy = __fadd_ru(hd.y, __fmul_rn(qbyte(ay.z, ay.w, k), scy));
                    const float lz = __fadd_rd(hd.z, __fmul_rn(qbyte(az.x, az.y, k), scz));
                    const float hz = __fadd_ru(hd.z, __fmul_rn(qbyte(az.z, az.w, k), scz));
                    float nn;
                    c.n[k] = slab_test(sr, lx, hx, ly, hy, lz, hz, limit_cmp, nn) ? nn : INFINITY;
                }
            } else {
                const float4* w = s.eight + size_t(cur) * 16u;
                const int sx = sr.neg_x ? 2 : 0, sy = sr.neg_y ? 2 : 0, sz = sr.neg_z ? 2 : 0;
                const float4 xn0 = __ldg(w + sx), xn1 = __ldg(w + sx + 1);
                const float4 xf0 = __ldg(w + 2 - sx), xf1 = __ldg(w + 3 - sx);
                const float4 yn0 = __ldg(w + 4 + sy), yn1 = __ldg(w + 5 + sy);
                const float4 yf0 = __ldg(w + 6 - sy), yf1 = __ldg(w + 7 - sy);
                const float4 zn0 = __ldg(w + 8 + sz), zn1 = __ldg(w + 9 + sz);
                const float4 zf0 = __ldg(w + 10 - sz), zf1 = __ldg(w + 11 - sz);
                ea = __ldg(reinterpret_cast<const uint4*>(w + 12));
                eb = __ldg(reinterpret_cast<const uint4*>(w + 13));
                if (COUNT) cnt->node_bytes += 224u;
                float nn;
#define RE_EIGHT_CHILD(K, F0, F1, L)                                                                     \
    c.n[K] = slab_test_planes(sr, (L ? xn1 : xn0).F0, (L ? xf1 : xf0).F0, (L ? yn1 : yn0).F0,           \
                              (L ? yf1 : yf0).F0, (L ? zn1 : zn0).F0, (L ? zf1 : zf0).F0, limit_cmp, nn) \
                 ? nn                                                                                    \
                 : INFINITY
                RE_EIGHT_CHILD(0, x, x, 0);
                RE_EIGHT_CHILD(1, y, y, 0);
                RE_EIGHT_CHILD(2, z, z, 0);
                RE_EIGHT_CHILD(3, w, w, 0);
                RE_EIGHT_CHILD(4, x, x, 1);
                RE_EIGHT_CHILD(5, y, y, 1);
                RE_EIGHT_CHILD(6, z, z, 1);
                RE_EIGHT_CHILD(7, w, w, 1);
#undef RE_EIGHT_CHILD
            }
            c.e[0] = ea.x; c.e[1] = ea.y; c.e[2] = ea.z; c.e[3] = ea.w;
            c.e[4] = eb.x; c.e[5] = eb.y; c.e[6] = eb.z; c.e[7] = eb.w;
            if (COUNT) {
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    if (c.e[k] == kWideEmpty) c.n[k] = INFINITY;  // an empty slot is never entered
                    else cnt->node_tests += 1u;
                }
            }
            sort8(c);
            if (c.n[0] != INFINITY) {
                int pushes = 0;
#pragma unroll
                for (int k = 1; k < 8; ++k) pushes += c.n[k] != INFINITY ? 1 : 0;
                if (sp + pushes > STACK) {
                    h.status = 2u;
                    h.tri = 0xffffffffu;
                    return h;
                }
#pragma unroll
                for (int k = 7; k >= 1; --k)
                    if (c.n[k] != INFINITY) stack[sp++] = make_uint2(c.e[k], __float_as_uint(c.n[k]));
                cur = c.e[0] & kRefMask;
                cur_count = c.e[0] >> kLeafShift;
                if (COUNT) cnt->max_stack = max(cnt->max_stack, uint32_t(sp));
                next = true;
            }
        } else {
            if (COUNT) {
                cnt->leaf_visits += 1u;
                cnt->leaf_prims += cur_count;
                cnt->max_leaf = max(cnt->max_leaf, cur_count);
            }
            for (uint32_t k = 0; k < cur_count; ++k) {
                const uint32_t ti = cur + k;
                const float4* tp = s.tris + size_t(ti) * 4u;
                const float4 p0 = __ldg(tp + 0), e1 = __ldg(tp + 1), e2 = __ldg(tp + 2);
                const uint2 key = make_uint2(__float_as_uint(e1.w), __float_as_uint(e2.w));
                if (key.x == opt.ignore_instance && key.y == opt.ignore_primitive) continue;
                const uint32_t flags = __float_as_uint(p0.w);
                if (opt.shadow && (flags & kTriCastsShadow) == 0u) continue;
                if (COUNT) cnt->tri_tests += 1u;
                float t, u, v;
                bool front;
                if (!tri_test(ray, p0, e1, e2, limit_cmp, t, u, v, front)) continue;
                if (!front && (flags & kTriDoubleSided) == 0u) continue;
                if ((flags & kTriAlphaMask) != 0u) {
                    const int acc = alpha_accept(s.alpha, ti, u, v);
                    if (acc < 0) {
                        h.status = 3u;
                        h.tri = 0xffffffffu;
                        return h;
                    }
                    if (acc == 0) continue;
                }
                if (ANY) {
                    h.t = t; h.u = u; h.v = v; h.tri = ti; h.front = front ? 1u : 0u;
                    return h;
                }
                const bool lower_key = t == limit && (key.x < best_i || (key.x == best_i && key.y < best_p));
                if (!found || t < limit || lower_key) {
                    found = true;
                    limit = t;
                    limit_cmp = next_up(t);
                    h.t = t; h.u = u; h.v = v; h.tri = ti; h.front = front ? 1u : 0u;
                    best_i = key.x;
                    best_p = key.y;
                }
            }
        }
        if (next) continue;
        while (sp > 0) {
            const uint2 e = stack[--sp];
            const float pn = __uint_as_float(e.y);
            if (pn >= limit_cmp) continue;
            cur = e.x & kRefMask;
            cur_count = e.x >> kLeafShift;
            next = true;
            break;
        }
        if (!next) break;
    }
    return h;
}

// Four-wide traversal with postponed leaves: trace_wide's node visits and
// triangle tests, in the while-while form of trace_ww (a lane that reaches
// a leaf parks it and keeps descending until every active lane of its warp
// holds one; the warp then tests triangles together).  Same closest hit and
// visibility as trace_wide.
template <bool ANY, int STACK, bool C = false>
__device__ __forceinline__ TraceHit trace_wide_ww(const TraceSceneView& s, const TraceRay& ray,
                                                  const TraceOptions& opt) {
    TraceHit h;
    h.t = ray.tmax;
    h.u = 0.0f;
    h.v = 0.0f;
    h.tri = 0xffffffffu;
    h.front = 0u;
    h.status = 0u;
    if (!ray_is_valid(ray)) {
        h.status = 1u;
        return h;
    }
    if (s.wide_count == 0u) return h;
    using S = SlabOf<C>;
    const typename S::Ray sr = S::make(ray);
    {
        float root_near;
        if (!S::box(sr, s.root_lo[0], s.root_hi[0], s.root_lo[1], s.root_hi[1], s.root_lo[2], s.root_hi[2],
                    S::limit(ray.tmax, sr), root_near))
            return h;
    }
    uint2 stack[STACK];
    int sp = 0;
    bool found = false;
    float limit = ray.tmax;
    float limit_cmp = ray.tmax;  // see next_up
    float lim = S::limit(ray.tmax, sr);  // what box near distances are compared against
    uint32_t best_i = 0xffffffffu, best_p = 0xffffffffu;
    uint32_t cur = 0u, cur_count = 0u;
    bool has_cur = true;
    uint32_t leaf = 0u, leaf_count = 0u;
    uint32_t steps = 0u;
    const uint32_t max_steps = s.wide_count * 5u + 8u;
    auto pop = [&]() {
        while (sp > 0) {
            const uint2 e = stack[--sp];
            const float pn = __uint_as_float(e.y);
            if (pn >= lim) continue;
            cur = e.x & kRefMask;
            cur_count = e.x >> kLeafShift;
            return true;
        }
        return false;
    };
    while (has_cur || leaf_count != 0u) {
        while (has_cur && cur_count == 0u) {
            if (++steps > max_steps) {  // malformed (cyclic) tree guard
                h.status = 3u;
                h.tri = 0xffffffffu;
                return h;
            }
            const float4* w = s.wide + size_t(cur) * 8u;
            const WidePlanes pl = load_wide_planes(w, sr);
            const uint4 ent = __ldg(reinterpret_cast<const uint4*>(w + 6));
            float n0 = INFINITY, n1 = INFINITY, n2 = INFINITY, n3 = INFINITY;
            // A child's entry matters only when it is entered (finite near):
            // the others sort last and are neither visited nor pushed.
            const uint32_t e0 = ent.x, e1 = ent.y, e2 = ent.z, e3 = ent.w;
            float nn;
            // An empty slot's +inf box is never entered.
            if (S::planes(sr, pl.xn.x, pl.xf.x, pl.yn.x, pl.yf.x, pl.zn.x, pl.zf.x, lim, nn)) {
                n0 = nn;
            }
            if (S::planes(sr, pl.xn.y, pl.xf.y, pl.yn.y, pl.yf.y, pl.zn.y, pl.zf.y, lim, nn)) {
                n1 = nn;
            }
            if (S::planes(sr, pl.xn.z, pl.xf.z, pl.yn.z, pl.yf.z, pl.zn.z, pl.zf.z, lim, nn)) {
                n2 = nn;
            }
            if (S::planes(sr, pl.xn.w, pl.xf.w, pl.yn.w, pl.yf.w, pl.zn.w, pl.zf.w, lim, nn)) {
                n3 = nn;
            }
            const int down = wide_descend<STACK>(n0, e0, n1, e1, n2, e2, n3, e3, stack, sp, cur, cur_count);
            if (down < 0) {
                h.status = 2u;
                h.tri = 0xffffffffu;
                return h;
            }
            if (down == 0) has_cur = pop();
            if (has_cur && cur_count != 0u && leaf_count == 0u) {
                leaf = cur;
                leaf_count = cur_count;
                has_cur = pop();
            }
            if (!__any_sync(__activemask(), leaf_count == 0u)) break;
        }
        while (true) {
            if (leaf_count == 0u) {
                if (!(has_cur && cur_count != 0u)) break;
                leaf = cur;
                leaf_count = cur_count;
                has_cur = pop();
            }
            for (uint32_t k = 0; k < leaf_count; ++k) {
                const uint32_t ti = leaf + k;
                const float4* tp = s.tris + size_t(ti) * 4u;
                const float4 p0 = __ldg(tp + 0), e1 = __ldg(tp + 1), e2 = __ldg(tp + 2);
                const uint2 key = make_uint2(__float_as_uint(e1.w), __float_as_uint(e2.w));
                if (key.x == opt.ignore_instance && key.y == opt.ignore_primitive) continue;
                const uint32_t flags = __float_as_uint(p0.w);
                if (opt.shadow && (flags & kTriCastsShadow) == 0u) continue;
                float t, u, v;
                bool front;
                if (!tri_test(ray, p0, e1, e2, limit_cmp, t, u, v, front)) continue;
                if (!front && (flags & kTriDoubleSided) == 0u) continue;
                if ((flags & kTriAlphaMask) != 0u) {
                    const int acc = alpha_accept(s.alpha, ti, u, v);
                    if (acc < 0) {
                        h.status = 3u;
                        h.tri = 0xffffffffu;
                        return h;
                    }
                    if (acc == 0) continue;
                }
                if (ANY) {
                    h.t = t; h.u = u; h.v = v; h.tri = ti; h.front = front ? 1u : 0u;
                    return h;
                }
                const bool lower_key = t == limit && (key.x < best_i || (key.x == best_i && key.y < best_p));
                if (!found || t < limit || lower_key) {
                    found = true;
                    limit = t;
                    limit_cmp = next_up(t);
                    lim = S::limit(limit_cmp, sr);
                    h.t = t; h.u = u; h.v = v; h.tri = ti; h.front = front ? 1u : 0u;
                    best_i = key.x;
                    best_p = key.y;
                }
            }
            leaf_count = 0u;
        }
    }
    return h;
}

// Resumable form of `trace` for persistent kernels that refill idle lanes
// with new rays: the same visiting order and the same results, one node or
// one leaf per step() call.
template <bool ANY, int STACK>
struct Traverser {
    TraceRay ray;
    SlabRay sr;
    TraceOptions opt;
    TraceHit h;
    uint2 stack[STACK];
    int sp;
    uint32_t cur, cur_count;
    bool found;
    float limit, limit_cmp;
    uint32_t bi, bp;
    uint32_t steps, max_steps;

    // Returns false when the ray is already finished (invalid or misses the root box).
    __device__ __forceinline__ bool init(const TraceSceneView& s, const TraceRay& r, const TraceOptions& o) {
        ray = r;
        opt = o;
        h.t = r.tmax;
        h.u = 0.f;
        h.v = 0.f;
        h.tri = 0xffffffffu;
        h.front = 0u;
        h.status = 0u;
        if (!ray_is_valid(r)) {
            h.status = 1u;
            return false;
        }
        if (s.node_count == 0u) return false;
        sr = make_slab_ray(r);
        float root_near;
        if (!slab_test(sr, s.root_lo[0], s.root_hi[0], s.root_lo[1], s.root_hi[1], s.root_lo[2], s.root_hi[2], r.tmax,
                       root_near))
            return false;
        sp = 0;
        cur = 0u;
        cur_count = 0u;
        found = false;
        limit = r.tmax;
        limit_cmp = r.tmax;
        bi = bp = 0xffffffffu;
        steps = 0u;
        max_steps = s.node_count * 4u + 8u;
        return true;
    }

    // Processes one interior node or one leaf; returns false when finished.
    __device__ __forceinline__ bool step(const TraceSceneView& s) {
        if (++steps > max_steps) {
            h.status = 3u;
            h.tri = 0xffffffffu;
            return false;
        }
        if (cur_count == 0u) {
            const float4* n = s.nodes + size_t(cur) * 4u;
            const float4 a = __ldg(n + 0);
            const float4 b = __ldg(n + 1);
            const float4 c = __ldg(n + 2);
            const uint4 d = __ldg(reinterpret_cast<const uint4*>(n + 3));
            float nl, nr;
            const bool hl = slab_test(sr, a.x, a.y, a.z, a.w, b.x, b.y, limit_cmp, nl);
            const bool hr = slab_test(sr, b.z, b.w, c.x, c.y, c.z, c.w, limit_cmp, nr);
            if (hl && hr) {
                const bool left_first = nl < nr || !(nr < nl);
                if (sp >= STACK) {
                    h.status = 2u;
                    h.tri = 0xffffffffu;
                    return false;
                }
                stack[sp++] = make_uint2(left_first ? (d.y | (d.w << kLeafShift)) : (d.x | (d.z << kLeafShift)),
                                         __float_as_uint(left_first ? nr : nl));
                cur = left_first ? d.x : d.y;
                cur_count = left_first ? d.z : d.w;
                return true;
            }
            if (hl) { cur = d.x; cur_count = d.z; return true; }
            if (hr) { cur = d.y; cur_count = d.w; return true; }
        } else {
            for (uint32_t k = 0; k < cur_count; ++k) {
                const uint32_t ti = cur + k;
                const float4* tp = s.tris + size_t(ti) * 4u;
                const float4 p0 = __ldg(tp + 0), e1 = __ldg(tp + 1), e2 = __ldg(tp + 2);
                const uint2 key = make_uint2(__float_as_uint(e1.w), __float_as_uint(e2.w));
                if (key.x == opt.ignore_instance && key.y == opt.ignore_primitive) continue;
                const uint32_t flags = __float_as_uint(p0.w);
                if (opt.shadow && (flags & kTriCastsShadow) == 0u) continue;
                float t, u, v;
                bool front;
                if (!tri_test(ray, p0, e1, e2, limit_cmp, t, u, v, front)) continue;
                if (!front && (flags & kTriDoubleSided) == 0u) continue;
                if ((flags & kTriAlphaMask) != 0u) {
                    const int acc = alpha_accept(s.alpha, ti, u, v);
                    if (acc < 0) {
                        h.status = 3u;
                        h.tri = 0xffffffffu;
                        return false;
                    }
                    if (acc == 0) continue;
                }
                if (ANY) {
                    h.t = t; h.u = u; h.v = v; h.tri = ti; h.front = front ? 1u : 0u;
                    return false;
                }
                const bool lower_key = t == limit && (key.x < bi || (key.x == bi && key.y < bp));
                if (!found || t < limit || lower_key) {
                    found = true;
                    limit = t;
                    limit_cmp = next_up(t);
                    h.t = t; h.u = u; h.v = v; h.tri = ti; h.front = front ? 1u : 0u;
                    bi = key.x;
                    bp = key.y;
                }
            }
        }
        while (sp > 0) {
            const uint2 e = stack[--sp];
            const float nn = __uint_as_float(e.y);
            if (nn >= limit_cmp) continue;
            cur = e.x & kRefMask;
            cur_count = e.x >> kLeafShift;
            return true;
        }
        return false;
    }
};

// trace_wide as a step machine (one four-wide node or one leaf per step), for
// the lane-refill kernels: the same node visits, tests and pruning, so the
// same closest hit and visibility as trace_wide.
template <bool ANY, int STACK>
struct WideTraverser {
    TraceRay ray;
    SlabRay sr;
    TraceOptions opt;
    TraceHit h;
    uint2 stack[STACK];
    int sp;
    uint32_t cur, cur_count;
    bool found;
    float limit, limit_cmp;
    uint32_t bi, bp;
    uint32_t steps, max_steps;

    // Returns false when the ray is already finished (invalid or misses the root box).
    __device__ __forceinline__ bool init(const TraceSceneView& s, const TraceRay& r, const TraceOptions& o) {
        ray = r;
        opt = o;
        h.t = r.tmax;
        h.u = 0.f;
        h.v = 0.f;
        h.tri = 0xffffffffu;
        h.front = 0u;
        h.status = 0u;
        if (!ray_is_valid(r)) {
            h.status = 1u;
            return false;
        }
        if (s.wide_count == 0u) return false;
        sr = make_slab_ray(r);
        float root_near;
        if (!slab_test(sr, s.root_lo[0], s.root_hi[0], s.root_lo[1], s.root_hi[1], s.root_lo[2], s.root_hi[2], r.tmax,
                       root_near))
            return false;
        sp = 0;
        cur = 0u;
        cur_count = 0u;
        found = false;
        limit = r.tmax;
        limit_cmp = r.tmax;
        bi = bp = 0xffffffffu;
        steps = 0u;
        max_steps = s.wide_count * 5u + 8u;
        return true;
    }

    // Processes one wide node or one leaf; returns false when finished.
    __device__ __forceinline__ bool step(const TraceSceneView& s) {
        if (++steps > max_steps) {  // malformed (cyclic) tree guard
            h.status = 3u;
            h.tri = 0xffffffffu;
            return false;
        }
        if (cur_count == 0u) {
            const float4* w = s.wide + size_t(cur) * 8u;
            const WidePlanes pl = load_wide_planes(w, sr);
            const uint4 ent = __ldg(reinterpret_cast<const uint4*>(w + 6));
            float n0 = INFINITY, n1 = INFINITY, n2 = INFINITY, n3 = INFINITY;
            uint32_t e0 = 0u, e1 = 0u, e2 = 0u, e3 = 0u;
            float nn;
            // An empty slot's +inf box is never entered.
            if (slab_test_planes(sr, pl.xn.x, pl.xf.x, pl.yn.x, pl.yf.x, pl.zn.x, pl.zf.x, limit_cmp, nn)) {
                n0 = nn;
                e0 = ent.x;
            }
            if (slab_test_planes(sr, pl.xn.y, pl.xf.y, pl.yn.y, pl.yf.y, pl.zn.y, pl.zf.y, limit_cmp, nn)) {
                n1 = nn;
                e1 = ent.y;
            }
            if (slab_test_planes(sr, pl.xn.z, pl.xf.z, pl.yn.z, pl.yf.z, pl.zn.z, pl.zf.z, limit_cmp, nn)) {
                n2 = nn;
                e2 = ent.z;
            }
            if (slab_test_planes(sr, pl.xn.w, pl.xf.w, pl.yn.w, pl.yf.w, pl.zn.w, pl.zf.w, limit_cmp, nn)) {
                n3 = nn;
                e3 = ent.w;
            }
            const int down = wide_descend<STACK>(n0, e0, n1, e1, n2, e2, n3, e3, stack, sp, cur, cur_count);
            if (down < 0) {
                h.status = 2u;
                h.tri = 0xffffffffu;
                return false;
            }
            if (down > 0) return true;
        } else {
            for (uint32_t k = 0; k < cur_count; ++k) {
                const uint32_t ti = cur + k;
                const float4* tp = s.tris + size_t(ti) * 4u;
                const float4 p0 = __ldg(tp + 0), e1 = __ldg(tp + 1), e2 = __ldg(tp + 2);
                const uint2 key = make_uint2(__float_as_uint(e1.w), __float_as_uint(e2.w));
                if (key.x == opt.ignore_instance && key.y == opt.ignore_primitive) continue;
                const uint32_t flags = __float_as_uint(p0.w);
                if (opt.shadow && (flags & kTriCastsShadow) == 0u) continue;
                float t, u, v;
                bool front;
                if (!tri_test(ray, p0, e1, e2, limit_cmp, t, u, v, front)) continue;
                if (!front && (flags & kTriDoubleSided) == 0u) continue;
                if ((flags & kTriAlphaMask) != 0u) {
                    const int acc = alpha_accept(s.alpha, ti, u, v);
                    if (acc < 0) {
                        h.status = 3u;
                        h.tri = 0xffffffffu;
                        return false;
                    }
                    if (acc == 0) continue;
                }
                if (ANY) {
                    h.t = t; h.u = u; h.v = v; h.tri = ti; h.front = front ? 1u : 0u;
                    return false;
                }
                const bool lower_key = t == limit && (key.x < bi || (key.x == bi && key.y < bp));
                if (!found || t < limit || lower_key) {
                    found = true;
                    limit = t;
                    limit_cmp = next_up(t);
                    h.t = t; h.u = u; h.v = v; h.tri = ti; h.front = front ? 1u : 0u;
                    bi = key.x;
                    bp = key.y;
                }
            }
        }
        while (sp > 0) {
            const uint2 e = stack[--sp];
            const float pn = __uint_as_float(e.y);
            if (pn >= limit_cmp) continue;
            cur = e.x & kRefMask;
            cur_count = e.x >> kLeafShift;
            return true;
        }
        return false;
    }
};

}  // namespace re

struct re_scene;
namespace re {
// Device view (buffers + root box) of a resident scene.
TraceSceneView scene_view(const re_scene* sc);
}  // namespace re
