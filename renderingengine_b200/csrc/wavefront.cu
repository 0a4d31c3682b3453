// Wavefront path tracer for sm_100a: RayGen -> (Intersect -> Shade ->
// TraceShadow) x depth -> Resolve, the stage sequence of the reference
// wavefront integrator (integrators/wavefront/shaders/*.hlsl, schedule in
// WavefrontSchedule.cpp:43-331) with these B200 choices:
//   - persistent kernels: every warp pulls 32 queue entries at a time from a
//     global work counter, so queue lengths never round-trip to the host and
//     the whole frame replays as one CUDA graph;
//   - warp-ballot + popc compaction with one atomic per warp per queue in
//     place of the three-pass Blelloch scan (Scan.hlsl/AddOffsets/Scatter);
//   - SoA path state and queues with 128-bit accesses;
//   - an optional fused Intersect+Shade kernel (autotuned split point).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "runtime.h"
#include "wavefront.cuh"

namespace re {
namespace {

constexpr uint32_t kInv = 0xffffffffu;

__device__ __forceinline__ uint32_t* slot(const WfDevice& d, uint32_t b, uint32_t k) {
    return d.counters + b * kSlotsPerBounce + k;
}

__device__ __forceinline__ void set_fatal(const WfDevice& d, uint32_t bit) { atomicOr(d.counters + kSlotFatal, bit); }

// Warp-wide fetch of the next 32 queue entries; returns false when drained.
__device__ __forceinline__ bool fetch(uint32_t* work, uint32_t count, uint32_t& base) {
    uint32_t b = 0;
    if ((threadIdx.x & 31) == 0) b = atomicAdd(work, 32u);
    base = __shfl_sync(0xffffffffu, b, 0);
    return base < count;
}

// Warp-aggregated append: returns this lane's slot (valid when flag set).
__device__ __forceinline__ uint32_t warp_append(uint32_t* count, bool flag) {
    const uint32_t mask = __ballot_sync(0xffffffffu, flag);
    const uint32_t lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == 0 && mask != 0u) base = atomicAdd(count, uint32_t(__popc(mask)));
    base = __shfl_sync(0xffffffffu, base, 0);
    return base + uint32_t(__popc(mask & ((1u << lane) - 1u)));
}

__device__ __forceinline__ void warp_count(uint32_t* counter, bool flag) {
    const uint32_t mask = __ballot_sync(0xffffffffu, flag);
    if ((threadIdx.x & 31) == 0 && mask != 0u) atomicAdd(counter, uint32_t(__popc(mask)));
}

// ---------------------------------------------------------------------------
// RayGen (RayGen.hlsl:10-93): one camera ray per pixel, dense in queue 0.
// ---------------------------------------------------------------------------
// Pixel of launch index `local` within a width x height view, so that the 32
// lanes of a warp take an 8 x 4 pixel tile: the full tiles first (row-major
// over tiles), then the pixels right of them in the tiled rows, then the rows
// below, each row-major -- a bijection onto the view's pixels.  A path's
// pixel (and its random streams, film and history) does not depend on it;
// only the queue order does, and with it the coherence of a warp's rays.
__device__ __forceinline__ uint32_t tiled_pixel(uint32_t local, uint32_t width, uint32_t height) {
    const uint32_t w8 = width & ~7u, h4 = height & ~3u;
    const uint32_t tiled = w8 * h4;
    uint32_t x, y;
    if (local < tiled) {
        const uint32_t tile = local >> 5, within = local & 31u, per_row = w8 >> 3;
        x = (tile % per_row) * 8u + (within & 7u);
        y = (tile / per_row) * 4u + (within >> 3);
    } else {
        const uint32_t b = local - tiled, side = width - w8;
        if (b < side * h4) {
            y = b / side;
            x = w8 + b % side;
        } else {
            const uint32_t b2 = b - side * h4;
            y = h4 + b2 / width;
            x = b2 % width;
        }
    }
    return y * width + x;
}

__global__ void k_raygen(WfDevice d) {
    const BatchParams bp = *d.batch;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < bp.pixel_total; base += stride) {
        const uint32_t c = base + threadIdx.x;
        const bool live = c < bp.pixel_total;
        const uint32_t q = warp_append(slot(d, 0, kSlotRays), live);
        if (!live) continue;
        const uint32_t v = launch_view(d.views, bp.view_count, c);
        const FrameParams& fp = d.views[v];
        const uint32_t pix = tiled_pixel(c - fp.pixel_base, fp.width, fp.height);
        const uint32_t i = fp.path_offset + pix;
        d.path_view[i] = v;
        const uint32_t x = pix % fp.width, y = pix / fp.width;
        const float jx = counter_random(pix, fp.sample, kDimCameraJitterX, fp.stream, fp.seed_lo, fp.seed_hi);
        const float jy = counter_random(pix, fp.sample, kDimCameraJitterY, fp.stream, fp.seed_lo, fp.seed_hi);
        float sx = (float(x) + jx) / float(fp.width);
        float sy = (float(y) + jy) / float(fp.height);
        sx = sx * 2.f - 1.f;
        sy = sy * 2.f - 1.f;
        sy = -sy;
        const f3 dir = normalize3(fp.cam_fwd + fp.cam_right * (sx * fp.aspect * fp.tan_half_fov) +
                                  fp.cam_up * (sy * fp.tan_half_fov));
        if (q < d.capacity) {
            d.ray_o[0][q] = to4(fp.cam_pos, fp.eps);
            d.ray_d[0][q] = to4(dir, 1.0e30f);
            d.ray_path[0][q] = pack_path(i, fp.scene_slot);
        }
        const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
        d.beta[i] = make_float4(1.f, 1.f, 1.f, 1.f);
        d.beta_d[i] = z;
        d.beta_s[i] = z;
        d.acc_cam[i] = z;
        d.acc_dd[i] = z;
        d.acc_ds[i] = z;
        d.acc_id[i] = z;
        d.acc_is[i] = z;
        d.prev_pos_pdf[i] = z;
        d.prev_ng[i] = z;
        d.prev_ns[i] = z;
        d.ident[i] = make_uint4(pix, fp.sample, 0u, kPathActive | kPathPrevDelta);
        d.gb_pos[i] = z;
        d.gb_nrm[i] = make_float4(0.f, 0.f, 0.f, __uint_as_float(kInv));
        d.gb_alb[i] = z;
        d.gb_id[i] = make_uint4(kInv, kInv, kInv, 0u);
        if (fp.rs.enabled != 0u) {  // PbrClearReconstructionInputsV2: a miss publishes an invalid surface
            float4* pr = d.prim[fp.rs.parity] + size_t(i) * 6u;
#pragma unroll
            for (int k = 0; k < 6; ++k) pr[k] = z;
        }
    }
}

// ---------------------------------------------------------------------------
// Intersect (Intersect.hlsl:4-39)
// ---------------------------------------------------------------------------
// Traversal loop of the wavefront stages (same closest hit in every mode):
// 0 = one child-pair node or leaf per step, the reference's loop; 1 =
// while-while with postponed leaves; 2 = four-wide nodes, postponed leaves;
// 4 = four-wide nodes, one node or leaf per step (and the counting form of 2).
template <bool ANY, bool COUNT, int STACK, int MODE>
__device__ __forceinline__ TraceHit trace_mode(const TraceSceneView& s, const TraceRay& ray, const TraceOptions& opt,
                                               TraceCounters* cnt) {
    if (MODE == 5) return trace_eight<ANY, COUNT, STACK, false>(s, ray, opt, cnt);
    if (MODE == 6) return trace_eight<ANY, COUNT, STACK, true>(s, ray, opt, cnt);
    if (MODE == 2 && !COUNT) return trace_wide_ww<ANY, STACK>(s, ray, opt);
    if (MODE == 2 || MODE == 4) return trace_wide<ANY, COUNT, STACK>(s, ray, opt, cnt);
    if (MODE == 8 && !COUNT) return trace_wide_ww<ANY, STACK, true>(s, ray, opt);
    if (MODE == 7 || MODE == 8) return trace_wide<ANY, COUNT, STACK, true>(s, ray, opt, cnt);
    if (MODE == 1 && !COUNT) return trace_ww<ANY, STACK>(s, ray, opt);
    return trace<ANY, COUNT, STACK>(s, ray, opt, cnt);
}

template <int STACK, int MODE = 0>
__device__ __forceinline__ float4 intersect_one(const SceneSlot& sc, float4 o, float4 dir) {
    TraceRay ray{from4(o), from4(dir), o.w, dir.w};
    TraceOptions opt{kInv, kInv, false};
    const TraceHit h = trace_mode<false, false, STACK, MODE>(sc.scene, ray, opt, nullptr);
    uint32_t code = h.tri;
    if (h.status != 0u) code = 0xfffffffeu;  // invalid ray / malformed: error hit
    else if (h.tri != kInv) code = h.tri | (h.front ? 0x80000000u : 0u);
    return make_float4(h.t, h.u, h.v, __uint_as_float(code));
}

// 1024 threads per SM (at most 64 registers): traversal is issue-bound and
// wants every warp the register file allows.  The CTA size (128, 256 or 512
// threads, the autotuner's block-size axis) only changes how those warps are
// grouped: the kernel is persistent and each warp fetches 32 rays at a time.
template <int STACK, int MODE, int BLOCK = 128>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) k_intersect(WfDevice d, uint32_t bounce) {
    const uint32_t q = bounce & 1u;
    const uint32_t count = *slot(d, bounce, kSlotRays);
    uint32_t base;
    while (fetch(slot(d, bounce, kSlotWorkIntersect), count, base)) {
        const uint32_t i = base + (threadIdx.x & 31);
        if (i < count)
            d.hit[i] = intersect_one<STACK, MODE>(d.scenes[d.ray_path[q][i] >> kPathBits], d.ray_o[q][i],
                                                  d.ray_d[q][i]);
    }
}

// Warp-reduced accumulation of node tests, triangle tests and node bytes
// fetched (profiling only): three counters per bounce.
__device__ __forceinline__ void add_tests(unsigned long long* dst, const TraceCounters& c) {
    unsigned long long a = c.node_tests, b = c.tri_tests, n = c.node_bytes;
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        n += __shfl_xor_sync(0xffffffffu, n, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(dst, a);
        atomicAdd(dst + 1, b);
        atomicAdd(dst + 2, n);
    }
}

// Counting variant of Intersect: same hits, plus node / triangle tests.
template <int STACK, int MODE>
__global__ void __launch_bounds__(128) k_intersect_counted(WfDevice d, uint32_t bounce, unsigned long long* cnt) {
    const uint32_t q = bounce & 1u;
    const uint32_t count = *slot(d, bounce, kSlotRays);
    uint32_t base;
    while (fetch(slot(d, bounce, kSlotWorkIntersect), count, base)) {
        const uint32_t i = base + (threadIdx.x & 31);
        TraceCounters c{};
        if (i < count) {
            const float4 o = d.ray_o[q][i], dir = d.ray_d[q][i];
            TraceRay ray{from4(o), from4(dir), o.w, dir.w};
            TraceOptions opt{kInv, kInv, false};
            const TraceHit h =
                trace_mode<false, true, STACK, MODE>(d.scenes[d.ray_path[q][i] >> kPathBits].scene, ray, opt, &c);
            uint32_t code = h.tri;
            if (h.status != 0u) code = 0xfffffffeu;
            else if (h.tri != kInv) code = h.tri | (h.front ? 0x80000000u : 0u);
            d.hit[i] = make_float4(h.t, h.u, h.v, __uint_as_float(code));
        }
        add_tests(cnt + bounce * 3u, c);
    }
}

__device__ __forceinline__ float4 encode_hit(const TraceHit& h) {
    uint32_t code = h.tri;
    if (h.status != 0u) code = 0xfffffffeu;
    else if (h.tri != kInv) code = h.tri | (h.front ? 0x80000000u : 0u);
    return make_float4(h.t, h.u, h.v, __uint_as_float(code));
}

// Persistent Intersect with per-lane refill: a lane whose ray finished takes
// a new ray as soon as at least `refill` lanes of its warp are idle, instead
// of waiting for the slowest ray of a 32-ray packet.  Same hits as
// k_intersect (the traversal of each ray is unchanged).  WIDE walks the
// four-wide nodes one node or leaf per step, otherwise the child pairs.
template <int STACK, bool WIDE>
__global__ void __launch_bounds__(128, 8) k_intersect_refill(WfDevice d, uint32_t bounce, uint32_t refill) {
    const uint32_t q = bounce & 1u;
    const uint32_t count = *slot(d, bounce, kSlotRays);
    uint32_t* work = slot(d, bounce, kSlotWorkIntersect);
    const uint32_t lane = threadIdx.x & 31;
    std::conditional_t<WIDE, WideTraverser<false, STACK>, Traverser<false, STACK>> tr;
    bool active = false, drained = false;
    uint32_t idx = 0;
    const SceneSlot* scp = d.scenes;
    while (true) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !active);
        const uint32_t n_idle = __popc(idle);
        if (!drained && n_idle >= refill) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(work, n_idle);
            base = __shfl_sync(0xffffffffu, base, 0);
            drained = base + n_idle >= count;
            if (!active) {
                idx = base + __popc(idle & ((1u << lane) - 1u));
                if (idx < count) {
                    const float4 o = d.ray_o[q][idx], dir = d.ray_d[q][idx];
                    TraceRay ray{from4(o), from4(dir), o.w, dir.w};
                    scp = d.scenes + (d.ray_path[q][idx] >> kPathBits);
                    if (tr.init(scp->scene, ray, TraceOptions{kInv, kInv, false})) active = true;
                    else d.hit[idx] = encode_hit(tr.h);
                }
            }
        }
        if (__ballot_sync(0xffffffffu, active) == 0u) {
            if (drained) break;
            continue;
        }
        if (active && !tr.step(scp->scene)) {
            d.hit[idx] = encode_hit(tr.h);
            active = false;
        }
    }
}

// ---------------------------------------------------------------------------
// Shade (Shade.hlsl:6-479) with the wavefront shadow split
// (PbrWavefrontShading.hlsli:207-330).
// ---------------------------------------------------------------------------
struct Material {
    float4 base_metal, emis_rough, trans_ior, atten, f0, ceta, ck;
    uint4 meta;
};

__device__ __forceinline__ Material load_material(const SceneSlot& sc, uint32_t m) {
    const float4* p = sc.materials + size_t(m) * 8u;
    Material r;
    r.base_metal = __ldg(p + 0);
    r.emis_rough = __ldg(p + 1);
    r.trans_ior = __ldg(p + 2);
    r.atten = __ldg(p + 3);
    r.f0 = __ldg(p + 4);
    r.ceta = __ldg(p + 5);
    r.ck = __ldg(p + 6);
    r.meta = __ldg(reinterpret_cast<const uint4*>(p + 7));
    return r;
}

// PbrMaterialToBsdfParamsL6 (pbr_material_bsdf.hlsli:8-42).
__device__ __forceinline__ BsdfParams material_params(const Material& m) {
    BsdfParams p;
    p.base_color = mk(m.base_metal.x, m.base_metal.y, m.base_metal.z);
    p.metallic = m.base_metal.w;
    p.f0 = mk(m.f0.x, m.f0.y, m.f0.z);
    p.roughness = m.emis_rough.w;
    p.cond_eta = mk(m.ceta.x, m.ceta.y, m.ceta.z);
    p.transmission = m.trans_ior.x;
    p.cond_k = mk(m.ck.x, m.ck.y, m.ck.z);
    p.model = m.meta.x;
    p.lobes = m.meta.y;
    p.complex_fresnel = m.meta.z;
    if (p.model == kModelRoughDielectric && isfinite(p.roughness) && p.roughness >= 0.f &&
        p.roughness * p.roughness < kMinAlpha) {
        p.model = kModelSmoothGlass;
        if ((p.lobes & kLobeGlossy) != 0u) p.lobes = (p.lobes & ~kLobeGlossy) | kLobeSpecular;
    }
    return p;
}

// PbrMaterialAuxiliaryIsValidL6 (pbr_material_bsdf.hlsli:60-76).
__device__ __forceinline__ bool material_aux_valid(const Material& m) {
    const f3 e = mk(m.emis_rough.x, m.emis_rough.y, m.emis_rough.z);
    if (!finite3(e) || any_negative(e) || !isfinite(m.atten.x) || !isfinite(m.atten.y) || !isfinite(m.atten.z) ||
        !isfinite(m.atten.w) || m.atten.w < 0.f)
        return false;
    if (m.atten.w > 0.f && (!(m.atten.x > 0.f && m.atten.y > 0.f && m.atten.z > 0.f) ||
                            !(m.atten.x <= 1.f && m.atten.y <= 1.f && m.atten.z <= 1.f)))
        return false;
    return true;
}

struct Hit {
    float t;
    f3 p, ng, ns;
    uint32_t material, instance, primitive, emitter_light, front;
};

// PbrPopulateSoftwareTraversalHitL6 (pbr_software_traversal.hlsli:150-186).
__device__ __forceinline__ Hit make_hit(const SceneSlot& sc, f3 o, f3 dir, float4 h) {
    Hit r;
    const uint32_t code = __float_as_uint(h.w);
    const uint32_t tri = code & 0x7fffffffu;
    r.front = code >> 31;
    r.t = h.x;
    const float4* tp = sc.scene.tris + size_t(tri) * 4u;
    const f3 e1 = from4(__ldg(tp + 1)), e2 = from4(__ldg(tp + 2));
    const float4* a = sc.attrs + size_t(tri) * 4u;
    const float w0 = 1.0f - h.y - h.z;
    f3 gn = normalize3(cross(e1, e2));
    f3 sn = normalize3(w0 * from4(__ldg(a + 0)) + h.y * from4(__ldg(a + 1)) + h.z * from4(__ldg(a + 2)));
    if (r.front == 0u) {
        gn = -gn;
        sn = -sn;
    }
    const uint4 ids = __ldg(reinterpret_cast<const uint4*>(a + 3));
    r.p = o + dir * h.x;
    r.ng = gn;
    r.ns = sn;
    r.material = ids.w;
    r.instance = ids.x;
    r.primitive = ids.y;
    r.emitter_light = __ldg(sc.emitter + tri);
    return r;
}

struct Accum {
    f3 cam, dd, ds, id, is;
};

// WfPbrAccumulateTerminal (PbrWavefrontShading.hlsli:127-187).
__device__ __forceinline__ bool accumulate_terminal(const WfDevice& d, uint32_t p, uint32_t bounce, f3 beta,
                                                    f3 bd, f3 bs, f3 emitted, float mis) {
    if (!finite_nonneg3(emitted) || !isfinite(mis) || mis < 0.f || !finite_nonneg3(beta) || !finite_nonneg3(bd) ||
        !finite_nonneg3(bs))
        return false;
    const f3 w = emitted * mis;
    if (!finite_nonneg3(w)) return false;
    if (bounce == 0u) {
        const f3 a = from4(d.acc_cam[p]) + beta * w;
        if (!finite_nonneg3(a)) return false;
        d.acc_cam[p] = to4(a, 0.f);
    } else {
        float4* dp = bounce == 1u ? d.acc_dd : d.acc_id;
        float4* sp = bounce == 1u ? d.acc_ds : d.acc_is;
        const f3 df = from4(dp[p]) + bd * w;
        const f3 sf = from4(sp[p]) + bs * w;
        if (!finite_nonneg3(df) || !finite_nonneg3(sf)) return false;
        dp[p] = to4(df, 0.f);
        sp[p] = to4(sf, 0.f);
    }
    return true;
}

// Miss (Shade.hlsl:74-118): the environment's radiance, weighted by MIS
// against the previous vertex's BSDF sample unless that bounce was a delta
// (or ReSTIR owns the primary vertex's direct light).  Returns false on a
// non-finite contribution.
__device__ __forceinline__ bool shade_miss(const WfDevice& d, const SceneSlot& sc, const FrameParams& fp,
                                           uint32_t bounce, uint32_t p, uint32_t idw, f3 dir) {
    if (sc.lights.env_light == 0xffffffffu) return true;  // no environment: zero radiance
    const f3 env = env_radiance(sc.lights, fp.env_xf, dir);
    float mis = 1.f;
    if (bounce != 0u && (idw & kPathPrevDelta) == 0u && fp.estimator != 0u) {
        if (fp.estimator == 3u && bounce == 1u && (idw & kPathPrevRestirOwned) != 0u) {
            mis = 0.f;
        } else {
            const float4 pp = d.prev_pos_pdf[p];
            LightContext lctx{from4(pp), from4(d.prev_ng[p]), from4(d.prev_ns[p]), fp.env_xf};
            const float lpdf = selected_light_pdf(sc.lights, sc.lights.env_light, lctx, dir, 0.f, f3s(0.f));
            if (lpdf > 0.f) mis = power_heuristic(pp.w, lpdf);
        }
    }
    if (!finite3(env) || !isfinite(mis)) return false;
    return accumulate_terminal(d, p, bounce, from4(d.beta[p]), from4(d.beta_d[p]), from4(d.beta_s[p]), env, mis);
}

__device__ __forceinline__ float rnd(const FrameParams& fp, uint32_t path, uint32_t sample, uint32_t dim) {
    return counter_random(path, sample, dim, fp.stream, fp.seed_lo, fp.seed_hi);
}

// The per-bounce random numbers of one path vertex, dimensions 0..9 of the
// bounce's block (light selection and shape, BSDF lobe and direction, Russian
// roulette), drawn in one loop: the same counter-based values as drawing each
// where it is used, with one copy of the Philox rounds in the Shade code
// instead of one per draw (the kernel's instruction footprint is what limits
// its issue rate).
constexpr uint32_t kBounceDraws = 10u;
__device__ __forceinline__ void draw_bounce(const FrameParams& fp, uint32_t pix, uint32_t sample, uint32_t bounce,
                                            float* out) {
#pragma unroll 1
    for (uint32_t k = 0; k < kBounceDraws; ++k) out[k] = rnd(fp, pix, sample, bounce_dim(bounce, k));
}

// Single-pass Shade (variant 0): records are held until the end of the
// invocation and appended with one full-warp ballot per queue; BSDF and
// light sampling are out-of-line calls.
struct ShadeOut {
    bool next;
    bool shadow;
    // next ray
    float4 n_o, n_d;
    // shadow record
    float4 s_o, s_d, s_cd, s_cs;
    uint4 s_id;
};


// One Shade invocation for the path owning queue entry i.
__device__ __forceinline__ ShadeOut shade_one_v0(const WfDevice& d, const SceneSlot& sc, const FrameParams& fp,
                                              uint32_t bounce, float4 ro,
                                              float4 rd, uint32_t p, float4 hraw, uint32_t* nonfinite,
                                              uint32_t* negpdf) {
    ShadeOut out;
    out.next = false;
    out.shadow = false;
    uint4 id = d.ident[p];
    const uint32_t sample = id.y;
    const uint32_t pix = id.x;  // pixel within the view: the RNG counter
    const f3 dir = from4(rd);
    const uint32_t code = __float_as_uint(hraw.w);
    auto finish = [&](uint32_t flags_set, uint32_t flags_clear) {
        id.w = (id.w & ~flags_clear) | flags_set;
        d.ident[p] = id;
    };
    if (code == kInv) {
        if (!shade_miss(d, sc, fp, bounce, p, id.w, dir)) {
            atomicAdd(nonfinite, 1u);
            finish(kPathTerminated | kPathError, kPathActive);
        } else {
            finish(kPathTerminated, kPathActive);
        }
        return out;
    }
    if (code == 0xfffffffeu) {
        atomicAdd(nonfinite, 1u);
        finish(kPathTerminated | kPathError, kPathActive);
        return out;
    }
    const Hit hit = make_hit(sc, from4(ro), dir, hraw);
    // WfPbrHitIsValid (PbrWavefrontShading.hlsli:114-125).
    const float gl2 = dot(hit.ng, hit.ng), sl2 = dot(hit.ns, hit.ns);
    const bool hit_ok = isfinite(hit.t) && hit.t >= ro.w && hit.t <= rd.w && finite3(hit.p) && isfinite(gl2) &&
                        gl2 > 0.f && isfinite(sl2) && sl2 > 0.f;
    if (!hit_ok || hit.material >= sc.material_count) {
        atomicAdd(nonfinite, 1u);
        finish(kPathTerminated | kPathError, kPathActive);
        return out;
    }
    const Material mat = load_material(sc, hit.material);
    if (!material_aux_valid(mat)) {
        atomicAdd(nonfinite, 1u);
        finish(kPathTerminated | kPathError, kPathActive);
        return out;
    }
    const BsdfParams params = material_params(mat);
    const bool restir_owned = bounce == 0u && supports_restir_primary(params);
    if (bounce == 0u) {
        // Primary-surface export for reconstruction and ReSTIR
        // (WfPublishPrimarySurfaceV2).
        const float depth = dot(hit.p - fp.cam_pos, normalize3(fp.cam_fwd));
        d.gb_pos[p] = to4(hit.p, depth);
        d.gb_nrm[p] = to4(hit.ns, __uint_as_float(hit.material));
        d.gb_alb[p] = make_float4(mat.base_metal.x, mat.base_metal.y, mat.base_metal.z, mat.emis_rough.w);
        d.gb_id[p] = make_uint4(hit.instance, hit.primitive, hit.material, hit.front);
        if (fp.rs.enabled != 0u)
            write_primary_surface(d.prim[fp.rs.parity], p, hit.p, depth, hit.ng, hit.ns, hit.material, hit.instance,
                                  hit.primitive, hit.front, from4(mat.base_metal), mat.base_metal.w, mat.emis_rough.w,
                                  mat.trans_ior.x, from4(mat.f0), restir_owned);
    }
    const float4 b4 = d.beta[p];
    f3 beta = from4(b4);
    float eta_scale = b4.w;
    f3 bd = from4(d.beta_d[p]);
    f3 bs = from4(d.beta_s[p]);
    // Beer-Lambert inside dielectrics (pbr_material_bsdf.hlsli:78-129).
    if (hit.front == 0u && mat.trans_ior.x > 0.f) {
        bool ok = true;
        if (mat.atten.w > 0.f) {
            const f3 col = mk(mat.atten.x, mat.atten.y, mat.atten.z);
            if (!(col.x > 0.f && col.y > 0.f && col.z > 0.f) || !(col.x <= 1.f && col.y <= 1.f && col.z <= 1.f) ||
                !isfinite(hit.t) || hit.t < 0.f) {
                ok = false;
            } else {
                const float e = hit.t / mat.atten.w;
                const f3 att = mk(powf(col.x, e), powf(col.y, e), powf(col.z, e));
                ok = finite3(att);
                beta *= att;
                bd *= att;
                bs *= att;
                ok = ok && finite3(beta) && finite3(bd) && finite3(bs);
            }
        }
        if (!ok) {
            atomicAdd(nonfinite, 1u);
            d.beta[p] = make_float4(0.f, 0.f, 0.f, eta_scale);
            d.beta_d[p] = make_float4(0.f, 0.f, 0.f, 0.f);
            d.beta_s[p] = make_float4(0.f, 0.f, 0.f, 0.f);
            finish(kPathTerminated | kPathError, kPathActive);
            return out;
        }
    }
    d.beta[p] = to4(beta, eta_scale);
    d.beta_d[p] = to4(bd, 0.f);
    d.beta_s[p] = to4(bs, 0.f);

    // Emission with MIS against the previous vertex's BSDF sample.
    const f3 emission = mk(mat.emis_rough.x, mat.emis_rough.y, mat.emis_rough.z);
    bool emitter_visible = hit.front != 0u;
    if (!emitter_visible && hit.emitter_light < sc.lights.light_count) {
        const LightRecord l = load_light(sc.lights, hit.emitter_light);
        emitter_visible = (l.identity.y & kLightTwoSided) != 0u;
    }
    if (emitter_visible && maxc(emission) > 0.f) {
        float mis = 1.f;
        if (bounce != 0u && (id.w & kPathPrevDelta) == 0u && fp.estimator != 0u) {
            if (fp.estimator == 3u && bounce == 1u && (id.w & kPathPrevRestirOwned) != 0u) {
                mis = 0.f;
            } else {
                const float4 pp = d.prev_pos_pdf[p];
                LightContext ctx{from4(pp), from4(d.prev_ng[p]), from4(d.prev_ns[p]), fp.env_xf};
                const float lpdf = selected_light_pdf(sc.lights, hit.emitter_light, ctx, dir, hit.t, hit.ng);
                if (lpdf > 0.f) mis = power_heuristic(pp.w, lpdf);
            }
        }
        if (!accumulate_terminal(d, p, bounce, beta, bd, bs, emission, mis)) {
            atomicAdd(nonfinite, 1u);
            finish(kPathTerminated | kPathError, kPathActive);
            return out;
        }
    }
    if ((mat.meta.w & 1u) != 0u || !finite3(beta) || any_negative(beta)) {
        finish(kPathTerminated, kPathActive);
        return out;
    }

    // PbrBuildBsdfContextL6 (pbr_material_bsdf.hlsli:44-58).
    BsdfContext ctx;
    ctx.ng = hit.ng;
    ctx.ns = hit.ns;
    f3 tb;
    build_basis(hit.ns, ctx.tangent, tb);
    const float ior = mat.trans_ior.y;
    ctx.eta_i = hit.front != 0u ? 1.f : ior;
    ctx.eta_t = hit.front != 0u ? ior : 1.f;
    ctx.transport = 0u;
    if (!validate_params(ctx, params)) {
        atomicAdd(nonfinite, 1u);
        finish(kPathTerminated | kPathError, kPathActive);
        return out;
    }
    const f3 wo = -dir;
    float rn[kBounceDraws];
    draw_bounce(fp, pix, sample, bounce, rn);

    // Next-event estimation (WfPbrBuildDirectShadow).
    if (fp.estimator != 0u && sc.lights.alias_count != 0u && !(fp.estimator == 3u && bounce == 0u && restir_owned)) {
        LightContext lc{hit.p, hit.ng, hit.ns, fp.env_xf};
        LightRandom lr;
        lr.selection = rn[kDimLightSelection];
        lr.s0 = rn[kDimLightShape0];
        lr.s1 = rn[kDimLightShape1];
        lr.s2 = rn[kDimLightShape2];
        lr.s3 = rn[kDimLightShape3];
        const LightSample ls = sample_one_light<false>(sc.lights, lc, lr);
        if ((ls.flags & kSampleValid) != 0u) {
            const BsdfEval ev = bsdf_evaluate<false>(ctx, params, wo, ls.wi);
            bool go = ev.valid;
            if (go && (!isfinite(ev.pdf) || !finite3(ev.value))) {
                atomicAdd(nonfinite, 1u);
                go = false;
            }
            if (go && ev.pdf < 0.f) {
                atomicAdd(negpdf, 1u);
                go = false;
            }
            const bool delta = (ls.flags & kSampleDelta) != 0u;
            const float est = delta ? ls.selection_pmf : ls.combined_pdf;
            if (go && !isfinite(est)) {
                atomicAdd(nonfinite, 1u);
                go = false;
            }
            if (go && !(est > 0.f)) {
                if (est < 0.f) atomicAdd(negpdf, 1u);
                go = false;
            }
            const float cosine = fabsf(dot(hit.ng, ls.wi));
            if (go && !(cosine > 0.f)) go = false;
            if (go) {
                const float mis = delta ? 1.f : power_heuristic(ls.combined_pdf, ev.pdf);
                const f3 scale = ls.li * (cosine * mis / est);
                const f3 cd = bounce == 0u ? beta * ev.diffuse * scale : bd * ev.value * scale;
                const f3 cs = bounce == 0u ? beta * ev.specular * scale : bs * ev.value * scale;
                if (!finite3(cd) || !finite3(cs) || any_negative(cd) || any_negative(cs)) {
                    atomicAdd(nonfinite, 1u);
                    go = false;
                }
                const float smax = (ls.flags & kSampleInfinite) != 0u ? 1.0e30f : ls.distance - fp.eps;
                if (go && smax > fp.eps) {
                    out.shadow = true;
                    out.s_o = to4(offset_origin(hit.p, hit.ng, ls.wi, fp.eps), fp.eps);
                    out.s_d = to4(ls.wi, smax);
                    out.s_cd = to4(cd, est);
                    out.s_cs = to4(cs, ls.combined_pdf);
                    out.s_id = make_uint4(pack_path(p, fp.scene_slot), bounce, ls.light, ls.primitive);
                }
            }
        }
    }

    // BSDF sampling, Russian roulette, next-bounce candidate.
    if (bounce + 1u < fp.max_depth) {
        const f3 u = mk(rn[kDimBsdfLobe], rn[kDimBsdfU], rn[kDimBsdfV]);
        const BsdfSample bsmp = bsdf_sample<false>(ctx, params, wo, u);
        bool valid = bsmp.valid && isfinite(bsmp.pdf) && bsmp.pdf > 0.f && finite3(bsmp.value) &&
                     finite3(bsmp.dir) && !any_negative(bsmp.value);
        if (bsmp.pdf < 0.f) atomicAdd(negpdf, 1u);
        f3 nb = f3s(0.f), nd = f3s(0.f), ns = f3s(0.f);
        float es = eta_scale;
        if (valid) {
            const float cosine = fabsf(dot(hit.ng, bsmp.dir));
            const f3 factor = bsmp.value * (cosine / bsmp.pdf);
            if (bounce == 0u) {
                nd = beta * bsmp.diffuse * (cosine / bsmp.pdf);
                ns = beta * bsmp.specular * (cosine / bsmp.pdf);
            } else {
                nd = bd * factor;
                ns = bs * factor;
            }
            nb = nd + ns;
            valid = finite3(nb) && finite3(nd) && finite3(ns) && !any_negative(nb);
            if ((bsmp.lobe & kLobeTransmission) != 0u) {
                es *= bsmp.eta * bsmp.eta;
                valid = valid && isfinite(es) && es > 0.f;
            }
        }
        const uint32_t next_bounce = bounce + 1u;
        if (valid && float(next_bounce) >= fp.rr_start) {
            const float mag = maxc(nb * es);
            if (!(mag > 0.f) || !isfinite(mag)) {
                valid = false;
            } else {
                const float cont = fminf(fmaxf(mag, fp.rr_min), fp.rr_max);
                const float rr = rn[kDimRussianRoulette];
                if (rr >= cont) {
                    valid = false;
                } else {
                    nb /= cont;
                    nd /= cont;
                    ns /= cont;
                }
            }
        }
        if (valid) {
            uint32_t ev = 0u;
            if (bsmp.delta) ev |= kPathPrevDelta;
            if ((bsmp.lobe & kLobeDiffuse) == 0u) ev |= kPathPrevSpecular;
            if (restir_owned) ev |= kPathPrevRestirOwned;
            out.next = true;
            out.n_o = to4(offset_origin(hit.p, hit.ng, bsmp.dir, fp.eps), fp.eps);
            out.n_d = to4(normalize3(bsmp.dir), 1.0e30f);
            // NextBounce state update (NextBounce.hlsl:97-112), applied here.
            d.beta[p] = to4(nb, es);
            d.beta_d[p] = to4(nd, 0.f);
            d.beta_s[p] = to4(ns, 0.f);
            d.prev_pos_pdf[p] = to4(hit.p, bsmp.pdf);
            d.prev_ng[p] = to4(hit.ng, 0.f);
            d.prev_ns[p] = to4(hit.ns, 0.f);
            id.z = next_bounce;
            id.w = (id.w & kPathError) | kPathActive | ev;
            d.ident[p] = id;
            return out;
        }
        if (!finite3(nb)) {
            atomicAdd(nonfinite, 1u);
            id.w |= kPathError;
        }
    }
    finish(kPathTerminated, kPathActive);
    return out;
}

template <bool FUSED, int STACK>
__global__ void __launch_bounds__(128) k_shade_v0(WfDevice d, uint32_t bounce) {
    const uint32_t q = bounce & 1u;
    const uint32_t nq = (bounce + 1u) & 1u;
    const uint32_t count = *slot(d, bounce, kSlotRays);
    uint32_t* work = slot(d, bounce, FUSED ? kSlotWorkIntersect : kSlotWorkShade);
    uint32_t base;
    while (fetch(work, count, base)) {
        const uint32_t i = base + (threadIdx.x & 31);
        const bool active = i < count;
        ShadeOut o;
        o.next = false;
        o.shadow = false;
        uint32_t pw = 0;
        if (active) {
            const float4 ro = d.ray_o[q][i];
            const float4 rd = d.ray_d[q][i];
            pw = d.ray_path[q][i];
            const uint32_t p = pw & kPathMask;
            const SceneSlot& sc = d.scenes[pw >> kPathBits];
            const float4 h = FUSED ? intersect_one<STACK>(sc, ro, rd) : d.hit[i];
            if (p >= d.capacity) {
                set_fatal(d, kFatalShadePathIndex);
            } else {
                o = shade_one_v0(d, sc, d.views[d.path_view[p]], bounce, ro, rd, p, h,
                                 slot(d, bounce, kSlotNonFinite), slot(d, bounce, kSlotNegativePdf));
            }
        }
        const bool nx = active && o.next;
        const bool sh = active && o.shadow;
        const uint32_t ns = warp_append(slot(d, bounce + 1u, kSlotRays), nx);
        const uint32_t ss = warp_append(slot(d, bounce, kSlotShadows), sh);
        if (nx) {
            if (ns < d.capacity) {
                d.ray_o[nq][ns] = o.n_o;
                d.ray_d[nq][ns] = o.n_d;
                d.ray_path[nq][ns] = pw;
            } else {
                set_fatal(d, kFatalNextOverflow);
            }
        }
        if (sh) {
            if (ss < d.capacity) {
                d.sh_o[ss] = o.s_o;
                d.sh_d[ss] = o.s_d;
                d.sh_cd[ss] = o.s_cd;
                d.sh_cs[ss] = o.s_cs;
                d.sh_id[ss] = o.s_id;
            } else {
                set_fatal(d, kFatalShadowOverflow);
            }
        }
    }
}


// Live state of one Shade invocation between its phases.
struct ShadeState {
    Hit hit;
    BsdfContext ctx;
    BsdfParams params;
    f3 beta, bd, bs, wo;
    float eta_scale;
    uint4 id;
    uint32_t p;   // path index
    uint32_t pw;  // path word (path | scene slot << kPathBits)
    bool restir_owned;
};

__device__ __forceinline__ void terminate_path(const WfDevice& d, ShadeState& st, uint32_t set) {
    st.id.w = (st.id.w & ~kPathActive) | kPathTerminated | set;
    d.ident[st.p] = st.id;
}

// Phase 1 (Shade.hlsl:84-340): miss / invalid-hit handling, primary-surface
// export, Beer-Lambert, emission with MIS, BSDF context.  Returns true when
// the path continues to NEE and BSDF sampling.
__device__ __forceinline__ bool shade_prepare(const WfDevice& d, const SceneSlot& sc, const FrameParams& fp,
                                              uint32_t bounce,
                                              float4 ro, float4 rd, float4 hraw, ShadeState& st,
                                              uint32_t* nonfinite) {
    const uint32_t p = st.p;
    st.id = d.ident[p];
    const f3 dir = from4(rd);
    const uint32_t code = __float_as_uint(hraw.w);
    if (code == kInv) {
        if (!shade_miss(d, sc, fp, bounce, p, st.id.w, dir)) {
            atomicAdd(nonfinite, 1u);
            terminate_path(d, st, kPathError);
        } else {
            terminate_path(d, st, 0u);
        }
        return false;
    }
    if (code == 0xfffffffeu) {
        atomicAdd(nonfinite, 1u);
        terminate_path(d, st, kPathError);
        return false;
    }
    st.hit = make_hit(sc, from4(ro), dir, hraw);
    const Hit& hit = st.hit;
    // WfPbrHitIsValid (PbrWavefrontShading.hlsli:114-125).
    const float gl2 = dot(hit.ng, hit.ng), sl2 = dot(hit.ns, hit.ns);
    const bool hit_ok = isfinite(hit.t) && hit.t >= ro.w && hit.t <= rd.w && finite3(hit.p) && isfinite(gl2) &&
                        gl2 > 0.f && isfinite(sl2) && sl2 > 0.f;
    if (!hit_ok || hit.material >= sc.material_count) {
        atomicAdd(nonfinite, 1u);
        terminate_path(d, st, kPathError);
        return false;
    }
    const Material mat = load_material(sc, hit.material);
    if (!material_aux_valid(mat)) {
        atomicAdd(nonfinite, 1u);
        terminate_path(d, st, kPathError);
        return false;
    }
    st.params = material_params(mat);
    st.restir_owned = bounce == 0u && supports_restir_primary(st.params);
    if (bounce == 0u) {
        // Primary-surface export for reconstruction and ReSTIR (WfPublishPrimarySurfaceV2).
        const float depth = dot(hit.p - fp.cam_pos, normalize3(fp.cam_fwd));
        d.gb_pos[p] = to4(hit.p, depth);
        d.gb_nrm[p] = to4(hit.ns, __uint_as_float(hit.material));
        d.gb_alb[p] = make_float4(mat.base_metal.x, mat.base_metal.y, mat.base_metal.z, mat.emis_rough.w);
        d.gb_id[p] = make_uint4(hit.instance, hit.primitive, hit.material, hit.front);
        if (fp.rs.enabled != 0u)
            write_primary_surface(d.prim[fp.rs.parity], p, hit.p, depth, hit.ng, hit.ns, hit.material, hit.instance,
                                  hit.primitive, hit.front, from4(mat.base_metal), mat.base_metal.w, mat.emis_rough.w,
                                  mat.trans_ior.x, from4(mat.f0), st.restir_owned);
    }
    const float4 b4 = d.beta[p];
    st.beta = from4(b4);
    st.eta_scale = b4.w;
    st.bd = from4(d.beta_d[p]);
    st.bs = from4(d.beta_s[p]);
    // Beer-Lambert inside dielectrics (pbr_material_bsdf.hlsli:78-129).
    if (hit.front == 0u && mat.trans_ior.x > 0.f && mat.atten.w > 0.f) {
        const f3 col = mk(mat.atten.x, mat.atten.y, mat.atten.z);
        bool ok = col.x > 0.f && col.y > 0.f && col.z > 0.f && col.x <= 1.f && col.y <= 1.f && col.z <= 1.f &&
                  isfinite(hit.t) && hit.t >= 0.f;
        if (ok) {
            const float e = hit.t / mat.atten.w;
            const f3 att = mk(powf(col.x, e), powf(col.y, e), powf(col.z, e));
            st.beta *= att;
            st.bd *= att;
            st.bs *= att;
            ok = finite3(att) && finite3(st.beta) && finite3(st.bd) && finite3(st.bs);
        }
        if (!ok) {
            atomicAdd(nonfinite, 1u);
            d.beta[p] = make_float4(0.f, 0.f, 0.f, st.eta_scale);
            d.beta_d[p] = make_float4(0.f, 0.f, 0.f, 0.f);
            d.beta_s[p] = make_float4(0.f, 0.f, 0.f, 0.f);
            terminate_path(d, st, kPathError);
            return false;
        }
        d.beta[p] = to4(st.beta, st.eta_scale);
        d.beta_d[p] = to4(st.bd, 0.f);
        d.beta_s[p] = to4(st.bs, 0.f);
    }
    // Emission with MIS against the previous vertex's BSDF sample.
    const f3 emission = mk(mat.emis_rough.x, mat.emis_rough.y, mat.emis_rough.z);
    if (maxc(emission) > 0.f) {
        bool visible = hit.front != 0u;
        if (!visible && hit.emitter_light < sc.lights.light_count) {
            const LightRecord l = load_light(sc.lights, hit.emitter_light);
            visible = (l.identity.y & kLightTwoSided) != 0u;
        }
        if (visible) {
            float mis = 1.f;
            if (bounce != 0u && (st.id.w & kPathPrevDelta) == 0u && fp.estimator != 0u) {
                if (fp.estimator == 3u && bounce == 1u && (st.id.w & kPathPrevRestirOwned) != 0u) {
                    mis = 0.f;
                } else {
                    const float4 pp = d.prev_pos_pdf[p];
                    LightContext lctx{from4(pp), from4(d.prev_ng[p]), from4(d.prev_ns[p]), fp.env_xf};
                    const float lpdf = selected_light_pdf(sc.lights, hit.emitter_light, lctx, dir, hit.t, hit.ng);
                    if (lpdf > 0.f) mis = power_heuristic(pp.w, lpdf);
                }
            }
            if (!accumulate_terminal(d, p, bounce, st.beta, st.bd, st.bs, emission, mis)) {
                atomicAdd(nonfinite, 1u);
                terminate_path(d, st, kPathError);
                return false;
            }
        }
    }
    if ((mat.meta.w & 1u) != 0u || !finite3(st.beta) || any_negative(st.beta)) {
        terminate_path(d, st, 0u);
        return false;
    }
    // PbrBuildBsdfContextL6 (pbr_material_bsdf.hlsli:44-58).
    st.ctx.ng = hit.ng;
    st.ctx.ns = hit.ns;
    f3 tb;
    build_basis(hit.ns, st.ctx.tangent, tb);
    const float ior = mat.trans_ior.y;
    st.ctx.eta_i = hit.front != 0u ? 1.f : ior;
    st.ctx.eta_t = hit.front != 0u ? ior : 1.f;
    st.ctx.transport = 0u;
    if (!validate_params(st.ctx, st.params)) {
        atomicAdd(nonfinite, 1u);
        terminate_path(d, st, kPathError);
        return false;
    }
    st.wo = -dir;
    return true;
}

struct ShadowRecord {
    float4 o, d, cd, cs;
    uint4 id;
};

// Phase 2: next-event estimation (WfPbrBuildDirectShadow,
// PbrWavefrontShading.hlsli:207-330).  Returns true when a shadow ray is due.
template <bool INL>
__device__ __forceinline__ bool shade_nee(const WfDevice& d, const SceneSlot& sc, const FrameParams& fp, uint32_t bounce,
                                          const ShadeState& st, ShadowRecord& rec, uint32_t* nonfinite,
                                          uint32_t* negpdf) {
    if (fp.estimator == 0u || sc.lights.alias_count == 0u || (fp.estimator == 3u && bounce == 0u && st.restir_owned))
        return false;
    const uint32_t p = st.p, sample = st.id.y, pix = st.id.x;
    const Hit& hit = st.hit;
    LightContext lc{hit.p, hit.ng, hit.ns, fp.env_xf};
    LightRandom lr;
    lr.selection = rnd(fp, pix, sample, bounce_dim(bounce, kDimLightSelection));
    lr.s0 = rnd(fp, pix, sample, bounce_dim(bounce, kDimLightShape0));
    lr.s1 = rnd(fp, pix, sample, bounce_dim(bounce, kDimLightShape1));
    lr.s2 = rnd(fp, pix, sample, bounce_dim(bounce, kDimLightShape2));
    lr.s3 = rnd(fp, pix, sample, bounce_dim(bounce, kDimLightShape3));
    const LightSample ls = sample_one_light<INL>(sc.lights, lc, lr);
    if ((ls.flags & kSampleValid) == 0u) return false;
    const BsdfEval ev = bsdf_evaluate<INL>(st.ctx, st.params, st.wo, ls.wi);
    if (!ev.valid) return false;
    if (!isfinite(ev.pdf) || !finite3(ev.value)) {
        atomicAdd(nonfinite, 1u);
        return false;
    }
    if (ev.pdf < 0.f) {
        atomicAdd(negpdf, 1u);
        return false;
    }
    const bool delta = (ls.flags & kSampleDelta) != 0u;
    const float est = delta ? ls.selection_pmf : ls.combined_pdf;
    if (!isfinite(est)) {
        atomicAdd(nonfinite, 1u);
        return false;
    }
    if (!(est > 0.f)) {
        if (est < 0.f) atomicAdd(negpdf, 1u);
        return false;
    }
    const float cosine = fabsf(dot(hit.ng, ls.wi));
    if (!(cosine > 0.f)) return false;
    const float mis = delta ? 1.f : power_heuristic(ls.combined_pdf, ev.pdf);
    const f3 scale = ls.li * (cosine * mis / est);
    const f3 cd = bounce == 0u ? st.beta * ev.diffuse * scale : st.bd * ev.value * scale;
    const f3 cs = bounce == 0u ? st.beta * ev.specular * scale : st.bs * ev.value * scale;
    if (!finite3(cd) || !finite3(cs) || any_negative(cd) || any_negative(cs)) {
        atomicAdd(nonfinite, 1u);
        return false;
    }
    const float smax = (ls.flags & kSampleInfinite) != 0u ? 1.0e30f : ls.distance - fp.eps;
    if (!(smax > fp.eps)) return false;
    rec.o = to4(offset_origin(hit.p, hit.ng, ls.wi, fp.eps), fp.eps);
    rec.d = to4(ls.wi, smax);
    rec.cd = to4(cd, est);
    rec.cs = to4(cs, ls.combined_pdf);
    rec.id = make_uint4(pack_path(p, fp.scene_slot), bounce, ls.light, ls.primitive);
    return true;
}

// Phase 3: BSDF sampling, Russian roulette and the NextBounce state update
// (Shade.hlsl:342-455, NextBounce.hlsl:97-112).  Returns true with the next
// ray when the path continues; otherwise terminates the path.
template <bool INL>
__device__ __forceinline__ bool shade_next(const WfDevice& d, const FrameParams& fp, uint32_t bounce, ShadeState& st,
                                           float4& n_o, float4& n_d, uint32_t* nonfinite, uint32_t* negpdf) {
    const uint32_t p = st.p, sample = st.id.y, pix = st.id.x;
    if (bounce + 1u < fp.max_depth) {
        const f3 u = mk(rnd(fp, pix, sample, bounce_dim(bounce, kDimBsdfLobe)),
                        rnd(fp, pix, sample, bounce_dim(bounce, kDimBsdfU)),
                        rnd(fp, pix, sample, bounce_dim(bounce, kDimBsdfV)));
        const BsdfSample bsmp = bsdf_sample<INL>(st.ctx, st.params, st.wo, u);
        bool valid = bsmp.valid && isfinite(bsmp.pdf) && bsmp.pdf > 0.f && finite3(bsmp.value) &&
                     finite3(bsmp.dir) && !any_negative(bsmp.value);
        if (bsmp.pdf < 0.f) atomicAdd(negpdf, 1u);
        f3 nb = f3s(0.f), nd = f3s(0.f), ns = f3s(0.f);
        float es = st.eta_scale;
        const Hit& hit = st.hit;
        if (valid) {
            const float cosine = fabsf(dot(hit.ng, bsmp.dir));
            const f3 factor = bsmp.value * (cosine / bsmp.pdf);
            if (bounce == 0u) {
                nd = st.beta * bsmp.diffuse * (cosine / bsmp.pdf);
                ns = st.beta * bsmp.specular * (cosine / bsmp.pdf);
            } else {
                nd = st.bd * factor;
                ns = st.bs * factor;
            }
            nb = nd + ns;
            valid = finite3(nb) && finite3(nd) && finite3(ns) && !any_negative(nb);
            if ((bsmp.lobe & kLobeTransmission) != 0u) {
                es *= bsmp.eta * bsmp.eta;
                valid = valid && isfinite(es) && es > 0.f;
            }
        }
        const uint32_t next_bounce = bounce + 1u;
        if (valid && float(next_bounce) >= fp.rr_start) {
            const float mag = maxc(nb * es);
            if (!(mag > 0.f) || !isfinite(mag)) {
                valid = false;
            } else {
                const float cont = fminf(fmaxf(mag, fp.rr_min), fp.rr_max);
                const float rr = rnd(fp, pix, sample, bounce_dim(bounce, kDimRussianRoulette));
                if (rr >= cont) {
                    valid = false;
                } else {
                    nb /= cont;
                    nd /= cont;
                    ns /= cont;
                }
            }
        }
        if (valid) {
            uint32_t ev = 0u;
            if (bsmp.delta) ev |= kPathPrevDelta;
            if ((bsmp.lobe & kLobeDiffuse) == 0u) ev |= kPathPrevSpecular;
            if (st.restir_owned) ev |= kPathPrevRestirOwned;
            n_o = to4(offset_origin(hit.p, hit.ng, bsmp.dir, fp.eps), fp.eps);
            n_d = to4(normalize3(bsmp.dir), 1.0e30f);
            d.beta[p] = to4(nb, es);
            d.beta_d[p] = to4(nd, 0.f);
            d.beta_s[p] = to4(ns, 0.f);
            d.prev_pos_pdf[p] = to4(hit.p, bsmp.pdf);
            d.prev_ng[p] = to4(hit.ng, 0.f);
            d.prev_ns[p] = to4(hit.ns, 0.f);
            st.id.z = next_bounce;
            st.id.w = (st.id.w & kPathError) | kPathActive | ev;
            d.ident[p] = st.id;
            return true;
        }
        if (!finite3(nb)) {
            atomicAdd(nonfinite, 1u);
            st.id.w |= kPathError;
        }
    }
    terminate_path(d, st, 0u);
    return false;
}

// Shade kernel: three phases with a full-warp ballot append after each
// emitting phase, so all 32 lanes take part in the compaction and queue
// records leave registers as soon as they are complete.
// VARIANT (three-phase Shade): 0 = out-of-line BSDF/light calls, no register cap; 1 = inlined,
// <= 128 registers (4 CTAs/SM); 2 = inlined, <= 168 registers (3 CTAs/SM).
constexpr int shade_min_blocks(int v) { return v == 0 ? 1 : (v == 1 ? 4 : 3); }

template <bool FUSED, int STACK, int VARIANT>
__global__ void __launch_bounds__(128, shade_min_blocks(VARIANT)) k_shade(WfDevice d, uint32_t bounce) {
    constexpr bool INL = VARIANT != 0;
    const uint32_t q = bounce & 1u;
    const uint32_t nq = (bounce + 1u) & 1u;
    const uint32_t count = *slot(d, bounce, kSlotRays);
    uint32_t* work = slot(d, bounce, FUSED ? kSlotWorkIntersect : kSlotWorkShade);
    uint32_t* nonfinite = slot(d, bounce, kSlotNonFinite);
    uint32_t* negpdf = slot(d, bounce, kSlotNegativePdf);
    uint32_t base;
    while (fetch(work, count, base)) {
        const uint32_t i = base + (threadIdx.x & 31);
        bool alive = i < count;
        ShadeState st;
        const SceneSlot* scp = d.scenes;
        const FrameParams* fpp = d.views;
        if (alive) {
            const float4 ro = d.ray_o[q][i];
            const float4 rd = d.ray_d[q][i];
            st.pw = d.ray_path[q][i];
            st.p = st.pw & kPathMask;
            scp = d.scenes + (st.pw >> kPathBits);
            const float4 h = FUSED ? intersect_one<STACK>(*scp, ro, rd) : d.hit[i];
            if (st.p >= d.capacity) {
                set_fatal(d, kFatalShadePathIndex);
                alive = false;
            } else {
                fpp = d.views + d.path_view[st.p];
                alive = shade_prepare(d, *scp, *fpp, bounce, ro, rd, h, st, nonfinite);
            }
        }
        ShadowRecord rec;
        const bool sh = alive && shade_nee<INL>(d, *scp, *fpp, bounce, st, rec, nonfinite, negpdf);
        const uint32_t ss = warp_append(slot(d, bounce, kSlotShadows), sh);
        if (sh) {
            if (ss < d.capacity) {
                d.sh_o[ss] = rec.o;
                d.sh_d[ss] = rec.d;
                d.sh_cd[ss] = rec.cd;
                d.sh_cs[ss] = rec.cs;
                d.sh_id[ss] = rec.id;
            } else {
                set_fatal(d, kFatalShadowOverflow);
            }
        }
        float4 n_o, n_d;
        const bool nx = alive && shade_next<INL>(d, *fpp, bounce, st, n_o, n_d, nonfinite, negpdf);
        const uint32_t ns = warp_append(slot(d, bounce + 1u, kSlotRays), nx);
        if (nx) {
            if (ns < d.capacity) {
                d.ray_o[nq][ns] = n_o;
                d.ray_d[nq][ns] = n_d;
                d.ray_path[nq][ns] = st.pw;
            } else {
                set_fatal(d, kFatalNextOverflow);
            }
        }
    }
}

// Split Shade (variants 3 / 4): the three phases above in two kernels, so
// each kernel's code is half of the stage's and the BSDF-sampling kernel
// runs only on surviving vertices (terminated lanes drop out between the
// two).  Kernel A: hit, material, emission, NEE and the shadow record; a
// vertex that continues leaves a 48-byte record.  Kernel B rebuilds the
// Shade state from the record and the path state with the same functions
// (material parameters, shading frame, view direction) and samples the
// BSDF, so the next ray is the one the one-kernel Shade emits.
template <bool FUSED, int STACK, bool INL>
__global__ void __launch_bounds__(128) k_shade_a(WfDevice d, uint32_t bounce) {
    const uint32_t q = bounce & 1u;
    const uint32_t count = *slot(d, bounce, kSlotRays);
    uint32_t* work = slot(d, bounce, FUSED ? kSlotWorkIntersect : kSlotWorkShade);
    uint32_t* nonfinite = slot(d, bounce, kSlotNonFinite);
    uint32_t* negpdf = slot(d, bounce, kSlotNegativePdf);
    uint32_t base;
    while (fetch(work, count, base)) {
        const uint32_t i = base + (threadIdx.x & 31);
        bool alive = i < count;
        ShadeState st;
        const SceneSlot* scp = d.scenes;
        const FrameParams* fpp = d.views;
        if (alive) {
            const float4 ro = d.ray_o[q][i];
            const float4 rd = d.ray_d[q][i];
            st.pw = d.ray_path[q][i];
            st.p = st.pw & kPathMask;
            scp = d.scenes + (st.pw >> kPathBits);
            const float4 h = FUSED ? intersect_one<STACK>(*scp, ro, rd) : d.hit[i];
            if (st.p >= d.capacity) {
                set_fatal(d, kFatalShadePathIndex);
                alive = false;
            } else {
                fpp = d.views + d.path_view[st.p];
                alive = shade_prepare(d, *scp, *fpp, bounce, ro, rd, h, st, nonfinite);
            }
        }
        ShadowRecord rec;
        const bool sh = alive && shade_nee<INL>(d, *scp, *fpp, bounce, st, rec, nonfinite, negpdf);
        const uint32_t ss = warp_append(slot(d, bounce, kSlotShadows), sh);
        if (sh) {
            if (ss < d.capacity) {
                d.sh_o[ss] = rec.o;
                d.sh_d[ss] = rec.d;
                d.sh_cd[ss] = rec.cd;
                d.sh_cs[ss] = rec.cs;
                d.sh_id[ss] = rec.id;
            } else {
                set_fatal(d, kFatalShadowOverflow);
            }
        }
        const bool cont = alive && bounce + 1u < fpp->max_depth;
        const uint32_t k = warp_append(slot(d, bounce, kSlotContinue), cont);
        if (cont) {
            if (k < d.capacity) {
                d.vx_pos[k] = to4(st.hit.p, __uint_as_float(st.hit.material));
                d.vx_ng[k] = to4(st.hit.ng, __uint_as_float(st.hit.front));
                d.vx_ns[k] = to4(st.hit.ns, __uint_as_float(i));
            } else {
                set_fatal(d, kFatalNextOverflow);
            }
        } else if (alive) {
            terminate_path(d, st, 0u);  // the last bounce: shade_next's depth rule
        }
    }
}

// Shade state of vertex record k (written by the first split-Shade kernel):
// the record's hit, the path state, and the material parameters, shading
// frame and view direction recomputed with the one-kernel Shade's functions.
__device__ __forceinline__ const FrameParams& resume_state(const WfDevice& d, uint32_t bounce, uint32_t k,
                                                           ShadeState& st, const SceneSlot*& scp) {
    const uint32_t q = bounce & 1u;
    const float4 vp = d.vx_pos[k], vg = d.vx_ng[k], vn = d.vx_ns[k];
    const uint32_t i = __float_as_uint(vn.w);
    st.pw = d.ray_path[q][i];
    st.p = st.pw & kPathMask;
    scp = d.scenes + (st.pw >> kPathBits);
    const FrameParams& fp = d.views[d.path_view[st.p]];
    st.id = d.ident[st.p];
    st.hit.p = from4(vp);
    st.hit.ng = from4(vg);
    st.hit.ns = from4(vn);
    st.hit.material = __float_as_uint(vp.w);
    st.hit.front = __float_as_uint(vg.w);
    const Material mat = load_material(*scp, st.hit.material);
    st.params = material_params(mat);
    st.restir_owned = bounce == 0u && supports_restir_primary(st.params);
    const float4 b4 = d.beta[st.p];
    st.beta = from4(b4);
    st.eta_scale = b4.w;
    st.bd = from4(d.beta_d[st.p]);
    st.bs = from4(d.beta_s[st.p]);
    st.ctx.ng = st.hit.ng;
    st.ctx.ns = st.hit.ns;
    f3 tb;
    build_basis(st.hit.ns, st.ctx.tangent, tb);
    const float ior = mat.trans_ior.y;
    st.ctx.eta_i = st.hit.front != 0u ? 1.f : ior;
    st.ctx.eta_t = st.hit.front != 0u ? ior : 1.f;
    st.ctx.transport = 0u;
    st.wo = -from4(d.ray_d[q][i]);
    return fp;
}

// Three-kernel Shade (variant 5): hit, material and emission | NEE on the
// surviving vertices | BSDF sampling (k_shade_b).  The first kernel records
// every vertex that survives emission.
template <bool FUSED, int STACK>
__device__ __forceinline__ void shade_prep_body(const WfDevice& d, uint32_t bounce) {
    const uint32_t q = bounce & 1u;
    const uint32_t count = *slot(d, bounce, kSlotRays);
    uint32_t* work = slot(d, bounce, FUSED ? kSlotWorkIntersect : kSlotWorkShade);
    uint32_t* nonfinite = slot(d, bounce, kSlotNonFinite);
    uint32_t base;
    while (fetch(work, count, base)) {
        const uint32_t i = base + (threadIdx.x & 31);
        bool alive = i < count;
        ShadeState st;
        if (alive) {
            const float4 ro = d.ray_o[q][i];
            const float4 rd = d.ray_d[q][i];
            st.pw = d.ray_path[q][i];
            st.p = st.pw & kPathMask;
            const SceneSlot& sc = d.scenes[st.pw >> kPathBits];
            const float4 h = FUSED ? intersect_one<STACK>(sc, ro, rd) : d.hit[i];
            if (st.p >= d.capacity) {
                set_fatal(d, kFatalShadePathIndex);
                alive = false;
            } else {
                alive = shade_prepare(d, sc, d.views[d.path_view[st.p]], bounce, ro, rd, h, st, nonfinite);
            }
        }
        const uint32_t k = warp_append(slot(d, bounce, kSlotContinue), alive);
        if (alive) {
            if (k < d.capacity) {
                d.vx_pos[k] = to4(st.hit.p, __uint_as_float(st.hit.material));
                d.vx_ng[k] = to4(st.hit.ng, __uint_as_float(st.hit.front));
                d.vx_ns[k] = to4(st.hit.ns, __uint_as_float(i));
            } else {
                set_fatal(d, kFatalNextOverflow);
            }
        }
    }
}

__device__ __forceinline__ void shade_nee_body(const WfDevice& d, uint32_t bounce) {
    const uint32_t count = min(*slot(d, bounce, kSlotContinue), d.capacity);
    uint32_t* work = slot(d, bounce, kSlotWorkNee);
    uint32_t* nonfinite = slot(d, bounce, kSlotNonFinite);
    uint32_t* negpdf = slot(d, bounce, kSlotNegativePdf);
    uint32_t base;
    while (fetch(work, count, base)) {
        const uint32_t k = base + (threadIdx.x & 31);
        bool sh = false;
        ShadowRecord rec;
        if (k < count) {
            ShadeState st;
            const SceneSlot* scp;
            const FrameParams& fp = resume_state(d, bounce, k, st, scp);
            sh = shade_nee<true>(d, *scp, fp, bounce, st, rec, nonfinite, negpdf);
        }
        const uint32_t ss = warp_append(slot(d, bounce, kSlotShadows), sh);
        if (sh) {
            if (ss < d.capacity) {
                d.sh_o[ss] = rec.o;
                d.sh_d[ss] = rec.d;
                d.sh_cd[ss] = rec.cd;
                d.sh_cs[ss] = rec.cs;
                d.sh_id[ss] = rec.id;
            } else {
                set_fatal(d, kFatalShadowOverflow);
            }
        }
    }
}

template <bool INL>
__device__ __forceinline__ void shade_b_body(const WfDevice& d, uint32_t bounce) {
    const uint32_t nq = (bounce + 1u) & 1u;
    const uint32_t count = min(*slot(d, bounce, kSlotContinue), d.capacity);
    uint32_t* work = slot(d, bounce, kSlotWorkContinue);
    uint32_t* nonfinite = slot(d, bounce, kSlotNonFinite);
    uint32_t* negpdf = slot(d, bounce, kSlotNegativePdf);
    uint32_t base;
    while (fetch(work, count, base)) {
        const uint32_t k = base + (threadIdx.x & 31);
        bool nx = false;
        ShadeState st;
        float4 n_o, n_d;
        if (k < count) {
            const SceneSlot* scp;
            const FrameParams& fp = resume_state(d, bounce, k, st, scp);
            // shade_next ends a path at its last bounce (the three-kernel
            // form records those vertices too, for their NEE).
            nx = shade_next<INL>(d, fp, bounce, st, n_o, n_d, nonfinite, negpdf);
        }
        const uint32_t ns = warp_append(slot(d, bounce + 1u, kSlotRays), nx);
        if (nx) {
            if (ns < d.capacity) {
                d.ray_o[nq][ns] = n_o;
                d.ray_d[nq][ns] = n_d;
                d.ray_path[nq][ns] = st.pw;
            } else {
                set_fatal(d, kFatalNextOverflow);
            }
        }
    }
}

// The Shade kernels of variant 5 and, with the registers capped so that MINB
// CTAs of 128 fit on an SM, of variants 6 (MINB 6) and 7 (MINB 5): more warps
// to hide the stage's latencies, at the cost of spills.
template <bool FUSED, int STACK>
__global__ void __launch_bounds__(128) k_shade_prep(WfDevice d, uint32_t bounce) {
    shade_prep_body<FUSED, STACK>(d, bounce);
}
__global__ void __launch_bounds__(128) k_shade_nee(WfDevice d, uint32_t bounce) { shade_nee_body(d, bounce); }
template <bool INL>
__global__ void __launch_bounds__(128) k_shade_b(WfDevice d, uint32_t bounce) { shade_b_body<INL>(d, bounce); }
template <bool FUSED, int STACK, int MINB>
__global__ void __launch_bounds__(128, MINB) k_shade_prep_capped(WfDevice d, uint32_t bounce) {
    shade_prep_body<FUSED, STACK>(d, bounce);
}
template <int MINB>
__global__ void __launch_bounds__(128, MINB) k_shade_nee_capped(WfDevice d, uint32_t bounce) {
    shade_nee_body(d, bounce);
}
template <int MINB>
__global__ void __launch_bounds__(128, MINB) k_shade_b_capped(WfDevice d, uint32_t bounce) {
    shade_b_body<true>(d, bounce);
}

// ---------------------------------------------------------------------------
// TraceShadow (TraceShadow.hlsl:5-92), Physical shadow method.
// ---------------------------------------------------------------------------
// One shadow query; returns the traversal tests through `c` when counting.
template <int STACK, bool COUNT, int MODE = 0>
__device__ __forceinline__ void shadow_one(const WfDevice& d, uint32_t bounce, uint32_t i, TraceCounters* c) {
    const float4 o = d.sh_o[i];
    const float4 dir = d.sh_d[i];
    const uint4 sid = d.sh_id[i];
    const uint32_t p = sid.x & kPathMask;
    const SceneSlot& sc = d.scenes[sid.x >> kPathBits];
    if (p >= d.capacity) {
        set_fatal(d, kFatalShadePathIndex);
        return;
    }
    TraceRay ray{from4(o), from4(dir), o.w, dir.w};
    // Exclude the sampled light's own (instance, primitive), as the
    // megakernel's PbrEvaluateShadowVisibilityL6 does
    // (pbr_megakernel.hlsl:178-186): with a normal-offset origin and
    // tMax = distance - epsilon the ray otherwise meets the light itself.
    uint32_t ign_inst = kInv;
    if (sid.z < sc.lights.light_count)
        ign_inst = __ldg(reinterpret_cast<const uint4*>(sc.lights.lights + size_t(sid.z) * 6u + 5)).w;
    TraceOptions opt{ign_inst, sid.w, true};
    const TraceHit h = trace_mode<true, COUNT, STACK, MODE>(sc.scene, ray, opt, c);
    if (h.status != 0u) {
        atomicAdd(slot(d, bounce, kSlotNonFinite), 1u);
        uint4 id = d.ident[p];
        id.w = (id.w & ~kPathActive) | kPathTerminated | kPathError;
        d.ident[p] = id;
        return;
    }
    if (h.tri != kInv) return;  // occluded
    const f3 cd = from4(d.sh_cd[i]);
    const f3 cs = from4(d.sh_cs[i]);
    float4* dp = sid.y == 0u ? d.acc_dd : d.acc_id;
    float4* sp = sid.y == 0u ? d.acc_ds : d.acc_is;
    const f3 df = from4(dp[p]) + cd;
    const f3 sf = from4(sp[p]) + cs;
    if (!finite_nonneg3(df) || !finite_nonneg3(sf)) {
        atomicAdd(slot(d, bounce, kSlotNonFinite), 1u);
        uint4 id = d.ident[p];
        id.w = (id.w & ~kPathActive) | kPathTerminated | kPathError;
        d.ident[p] = id;
        return;
    }
    dp[p] = to4(df, 0.f);
    sp[p] = to4(sf, 0.f);
}

template <int STACK, bool COUNT, int MODE = 0, int BLOCK = 128>
__global__ void __launch_bounds__(BLOCK, COUNT ? 1 : 1024 / BLOCK) k_shadow(WfDevice d, uint32_t bounce,
                                                                            unsigned long long* cnt) {
    const uint32_t count = min(*slot(d, bounce, kSlotShadows), d.capacity);
    uint32_t base;
    while (fetch(slot(d, bounce, kSlotWorkShadow), count, base)) {
        const uint32_t i = base + (threadIdx.x & 31);
        TraceCounters c{};
        if (i < count) shadow_one<STACK, COUNT, MODE>(d, bounce, i, &c);
        if (COUNT) add_tests(cnt + 3u * kMaxDepth + bounce * 3u, c);
    }
}

// Accumulates a finished shadow query into its path (TraceShadow.hlsl:33-92).
__device__ __forceinline__ void shadow_finish(const WfDevice& d, uint32_t bounce, uint32_t i, const TraceHit& h) {
    const uint4 sid = d.sh_id[i];
    const uint32_t p = sid.x & kPathMask;
    if (h.status != 0u) {
        atomicAdd(slot(d, bounce, kSlotNonFinite), 1u);
        uint4 id = d.ident[p];
        id.w = (id.w & ~kPathActive) | kPathTerminated | kPathError;
        d.ident[p] = id;
        return;
    }
    if (h.tri != kInv) return;  // occluded
    const f3 cd = from4(d.sh_cd[i]);
    const f3 cs = from4(d.sh_cs[i]);
    float4* dp = sid.y == 0u ? d.acc_dd : d.acc_id;
    float4* sp = sid.y == 0u ? d.acc_ds : d.acc_is;
    const f3 df = from4(dp[p]) + cd;
    const f3 sf = from4(sp[p]) + cs;
    if (!finite_nonneg3(df) || !finite_nonneg3(sf)) {
        atomicAdd(slot(d, bounce, kSlotNonFinite), 1u);
        uint4 id = d.ident[p];
        id.w = (id.w & ~kPathActive) | kPathTerminated | kPathError;
        d.ident[p] = id;
        return;
    }
    dp[p] = to4(df, 0.f);
    sp[p] = to4(sf, 0.f);
}

// TraceShadow with per-lane refill (see k_intersect_refill).
template <int STACK, bool WIDE>
__global__ void __launch_bounds__(128, 8) k_shadow_refill(WfDevice d, uint32_t bounce, uint32_t refill) {
    const uint32_t count = min(*slot(d, bounce, kSlotShadows), d.capacity);
    uint32_t* work = slot(d, bounce, kSlotWorkShadow);
    const uint32_t lane = threadIdx.x & 31;
    std::conditional_t<WIDE, WideTraverser<true, STACK>, Traverser<true, STACK>> tr;
    bool active = false, drained = false;
    uint32_t idx = 0;
    const SceneSlot* scp = d.scenes;
    while (true) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !active);
        const uint32_t n_idle = __popc(idle);
        if (!drained && n_idle >= refill) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(work, n_idle);
            base = __shfl_sync(0xffffffffu, base, 0);
            drained = base + n_idle >= count;
            if (!active) {
                idx = base + __popc(idle & ((1u << lane) - 1u));
                if (idx < count) {
                    const float4 o = d.sh_o[idx], dir = d.sh_d[idx];
                    const uint4 sid = d.sh_id[idx];
                    if ((sid.x & kPathMask) >= d.capacity) {
                        set_fatal(d, kFatalShadePathIndex);
                    } else {
                        scp = d.scenes + (sid.x >> kPathBits);
                        uint32_t ign_inst = kInv;
                        if (sid.z < scp->lights.light_count)
                            ign_inst = __ldg(reinterpret_cast<const uint4*>(scp->lights.lights + size_t(sid.z) * 6u + 5)).w;
                        TraceRay ray{from4(o), from4(dir), o.w, dir.w};
                        if (tr.init(scp->scene, ray, TraceOptions{ign_inst, sid.w, true})) active = true;
                        else shadow_finish(d, bounce, idx, tr.h);
                    }
                }
            }
        }
        if (__ballot_sync(0xffffffffu, active) == 0u) {
            if (drained) break;
            continue;
        }
        if (active && !tr.step(scp->scene)) {
            shadow_finish(d, bounce, idx, tr.h);
            active = false;
        }
    }
}

// ---------------------------------------------------------------------------
// Resolve (Resolve.hlsl) + progressive film accumulation.
// ---------------------------------------------------------------------------
__global__ void k_resolve(WfDevice d) {
    const BatchParams bp = *d.batch;
    if (bp.pad1 != 0u) return;  // profiling passes leave the film and totals untouched
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // Running totals since the film was last reset: frames, path rays,
        // shadow rays (slots 1..4 of film_frames as two 64-bit words).
        atomicAdd(d.film_frames, 1u);
        unsigned long long rays = 0, shadows = 0;
        for (uint32_t b = 0; b < bp.pad0; ++b) {
            rays += min(d.counters[b * kSlotsPerBounce + kSlotRays], d.capacity);
            shadows += min(d.counters[b * kSlotsPerBounce + kSlotShadows], d.capacity);
        }
        unsigned long long* tot = reinterpret_cast<unsigned long long*>(d.film_frames + 2);
        tot[0] += rays;
        tot[1] += shadows;
    }
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < bp.pixel_total; c += gridDim.x * blockDim.x) {
        const uint32_t v = launch_view(d.views, bp.view_count, c);
        const uint32_t i = d.views[v].path_offset + (c - d.views[v].pixel_base);
        const f3 cam = from4(d.acc_cam[i]), dd = from4(d.acc_dd[i]), ds = from4(d.acc_ds[i]),
                 id = from4(d.acc_id[i]), is = from4(d.acc_is[i]);
        f3 s = cam + dd + ds + id + is;
        if (!finite_nonneg3(cam) || !finite_nonneg3(dd) || !finite_nonneg3(ds) || !finite_nonneg3(id) ||
            !finite_nonneg3(is)) {
            atomicAdd(d.counters + kSlotsPerBounce * 0 + kSlotNonFinite, 1u);
            s = mk(1.f, 1.f, 0.f);  // the reference marks the pixel yellow
        }
        d.sample_out[i] = to4(s, 1.f);
        const float4 prev = d.views[v].accumulate ? d.film_sum[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        d.film_sum[i] = make_float4(prev.x + s.x, prev.y + s.y, prev.z + s.z, prev.w + 1.f);
    }
}

}  // namespace

}  // namespace re

// ===========================================================================
// Host renderer
// ===========================================================================
using namespace re;

namespace {

constexpr uint32_t kMaxViews = RE_MAX_BATCH_VIEWS;
constexpr uint32_t kFrameRing = 4;
// One frame record: the batch header followed by up to kMaxViews views.
constexpr size_t kFrameRecordBytes = sizeof(BatchParams) + size_t(kMaxViews) * sizeof(FrameParams);

// Tables of one bound scene slot.
struct SlotState {
    re_scene* scene = nullptr;
    DeviceBuffer materials, lights, alias, pmf, fixtures, emitter;
    uint32_t material_count = 0, light_count = 0, alias_count = 0, fixture_count = 0;
    // Environment map of the slot (re_renderer_set_environment) and its
    // importance tables; env_light is the bound enabled environment light.
    DeviceBuffer env_texels, env_rows, env_cols;
    uint32_t env_width = 0, env_height = 0, env_uniform = 0;
    double env_integrated = 0.0;
    uint32_t env_light = 0xffffffffu;
    uint32_t light_selection = 0;
    uint32_t generation = 0;  // scene / light-set generation (ReSTIR history identity)
    bool wide_view = false;   // the device slot table carries the scene's wide nodes
    bool eight_view = false;  // ... and its eight-wide nodes
};

// ReSTIR history bookkeeping of one view (keyed by the caller's view key).
struct RestirView {
    uint32_t parity = 0, resolution_gen = 1, last_w = 0, last_h = 0, prev_light_count = 0;
    bool has_prev = false;
    FrameParams prev{};
};

}  // namespace

struct re_renderer {
    int device = 0;
    uint32_t max_w = 0, max_h = 0, max_depth = 0, capacity = 0;
    re_renderer_tuning tuning{128, 0, 0, 1, 4, 0, 3};  // split inlined Shade, traversal chosen per launch
    re_scene* scene = nullptr;  // scene of slot 0 (the single-view API)
    SlotState slots[kMaxSceneSlots];
    uint32_t generation_counter = 0;
    // Path state + queues + film.
    DeviceBuffer arena;
    WfDevice dev{};
    DeviceBuffer counters, frame, film_frames, scenes_table, path_view;
    DeviceBuffer export_stage;  // host-bound reconstruction records
    // Pinned ring of frame records: the host writes record k only after the
    // copy that read it kFrameRing launches ago has executed.
    char* host_frame = nullptr;  // pinned, kFrameRing records
    cudaEvent_t ring_done[kFrameRing] = {};
    bool ring_used[kFrameRing] = {};
    uint32_t ring_next = 0;
    uint32_t* host_counters = nullptr;  // pinned
    // Instantiated frame graphs by (depth, traversal stack, ReSTIR) key, most
    // recently used last; a batch whose views change the key between launches
    // replays a cached graph instead of capturing again.
    std::vector<std::pair<uint64_t, cudaGraphExec_t>> graphs;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint32_t last_pixels = 0;    // path_end of the last launch
    uint32_t batch_depth = 0;    // deepest view of the staged launch
    bool frame_pending = false;
    re_frame_telemetry telemetry{};
    // ReSTIR DI.
    re_restir_config restir{};
    DeviceBuffer restir_arena;
    bool restir_active = false;  // the staged launch runs the ReSTIR passes
    bool batch_deep = false;     // the staged launch's traversal kernels need the 128-entry stack
    bool batch_deep_binary = false;  // a child-pair hierarchy of the launch is deeper than 64
    bool batch_wide = false;     // the staged launch traverses four-wide nodes
    uint32_t batch_eight = 0;    // ... or eight-wide nodes: 5 plain, 6 compressed
    uint32_t batch_loop = 1;     // its traversal loop (traversal_mode values 0, 1, 2, 4, 7, 8)
    uint32_t camera_epoch = 1;   // bumped by re_renderer_restir_reset / set_restir
    std::unordered_map<uint64_t, RestirView> rs_views;
    // Asynchronous film reads (re_renderer_read_view_async): two device
    // staging buffers used in turn, the stream that copies them to the
    // host, and per buffer the events after its snapshot and its host copy.
    DeviceBuffer read_stage[2];
    cudaStream_t read_stream = nullptr;
    cudaEvent_t read_snap[2] = {}, read_done[2] = {};
    bool read_used[2] = {};
    uint32_t read_next = 0;

    ~re_renderer() {
        if (read_stream) {
            cudaStreamSynchronize(read_stream);
            cudaStreamDestroy(read_stream);
        }
        for (int k = 0; k < 2; ++k) {
            if (read_snap[k]) cudaEventDestroy(read_snap[k]);
            if (read_done[k]) cudaEventDestroy(read_done[k]);
        }
        for (auto& g : graphs) cudaGraphExecDestroy(g.second);
        if (host_frame) cudaFreeHost(host_frame);
        if (host_counters) cudaFreeHost(host_counters);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (auto& e : ring_done)
            if (e) cudaEventDestroy(e);
    }
};

namespace re {

// Vose alias table with the construction order of BuildVoseAliasTable
// (MegakernelBridge.cpp:40-144): FP64 probabilities, LIFO small/large stacks,
// leftovers set to q = 1.  Entries: (q, pmf, alias, item).
bool build_alias_table(const std::vector<double>& w, const std::vector<uint32_t>& items, std::vector<float4>& out,
                       std::string& err) {
    out.clear();
    if (w.empty()) return true;
    double sum = 0.0;
    for (double x : w) {
        if (!std::isfinite(x) || x < 0.0) {
            err = "alias weights must be finite and non-negative";
            return false;
        }
        sum += x;
    }
    const size_t n = w.size();
    const bool uniform = sum == 0.0;
    const double norm = sum > 0.0 ? sum : double(n);
    std::vector<double> prob(n), scaled(n);
    std::vector<uint32_t> small, large;
    out.resize(n);
    std::vector<float> q(n, 0.f);
    std::vector<uint32_t> alias(n);
    for (size_t i = 0; i < n; ++i) {
        prob[i] = uniform ? 1.0 / double(n) : w[i] / norm;
        scaled[i] = prob[i] * double(n);
        alias[i] = uint32_t(i);
        if (scaled[i] < 1.0) small.push_back(uint32_t(i));
        else large.push_back(uint32_t(i));
    }
    while (!small.empty() && !large.empty()) {
        const uint32_t s = small.back();
        small.pop_back();
        const uint32_t l = large.back();
        large.pop_back();
        q[s] = float(std::min(std::max(scaled[s], 0.0), 1.0));
        alias[s] = l;
        scaled[l] = scaled[l] + scaled[s] - 1.0;
        if (scaled[l] < 1.0) small.push_back(l);
        else large.push_back(l);
    }
    for (uint32_t i : large) { q[i] = 1.f; alias[i] = i; }
    for (uint32_t i : small) { q[i] = 1.f; alias[i] = i; }
    for (size_t i = 0; i < n; ++i) {
        float a, it;
        const uint32_t item = items.empty() ? uint32_t(i) : items[i];
        std::memcpy(&a, &alias[i], 4);
        std::memcpy(&it, &item, 4);
        out[i] = make_float4(q[i], float(prob[i]), a, it);
    }
    return true;
}

// LightPowerWeight (MegakernelBridge.cpp:275-351); an environment light's
// weight is pi R^2 scale times the map's integrated luminance.
double light_power(const re_light& l, float scene_radius, double env_integrated) {
    const double lum = (0.2126 * double(l.radiance_scale.x) + 0.7152 * double(l.radiance_scale.y) +
                        0.0722 * double(l.radiance_scale.z)) * double(l.radiance_scale.w);
    const double pi = 3.141592653589793238462643383279502884;
    const double two = (l.identity.y & RE_LIGHT_FLAG_TWO_SIDED) != 0u ? 2.0 : 1.0;
    switch (l.identity.x) {
        case RE_LIGHT_POINT: return 4.0 * pi * lum;
        case RE_LIGHT_DIRECTIONAL: return pi * double(scene_radius) * double(scene_radius) * lum;
        case RE_LIGHT_SPOT: {
            const double co = l.direction_cos_outer.w, ci = l.shape_params.y;
            return 2.0 * pi * lum * ((1.0 - ci) + 0.5 * (ci - co));
        }
        case RE_LIGHT_SPHERE_AREA:
            return 4.0 * pi * pi * double(l.shape_params.x) * double(l.shape_params.x) * lum * two;
        case RE_LIGHT_EMISSIVE_TRIANGLE: return pi * double(l.shape_params.z) * lum * two;
        case RE_LIGHT_ENVIRONMENT:
            return pi * double(scene_radius) * double(scene_radius) * double(l.radiance_scale.w) * env_integrated;
        default: return 0.0;
    }
}

// BuildEnvironmentDistribution (MegakernelBridge.cpp:191-273): texel weight
// = luminance x texel solid angle (FP64), a column alias table per row and a
// row alias table over the row sums; a black map falls back to weights equal
// to the solid angles (uniform-sphere sampling).
bool build_environment_distribution(uint32_t w, uint32_t h, const std::vector<float>& lum, std::vector<float4>& rows,
                                    std::vector<float4>& cols, double& integrated, bool& fallback,
                                    std::string& err) {
    const double pi = 3.141592653589793238462643383279502884;
    auto solid_angle = [&](uint32_t row) {
        const double t0 = pi * double(row) / double(h), t1 = pi * double(row + 1u) / double(h);
        return 2.0 * pi / double(w) * (std::cos(t0) - std::cos(t1));
    };
    std::vector<double> tw(size_t(w) * h);
    integrated = 0.0;
    for (uint32_t r = 0; r < h; ++r) {
        const double sa = solid_angle(r);
        for (uint32_t c = 0; c < w; ++c) {
            const double l = double(lum[size_t(r) * w + c]);
            if (!std::isfinite(l) || l < 0.0) {
                err = "environment luminance must be finite and non-negative";
                return false;
            }
            tw[size_t(r) * w + c] = l * sa;
            integrated += l * sa;
        }
    }
    if (!std::isfinite(integrated)) {
        err = "environment luminance integral overflowed";
        return false;
    }
    fallback = integrated == 0.0;
    if (fallback)
        for (uint32_t r = 0; r < h; ++r)
            for (uint32_t c = 0; c < w; ++c) tw[size_t(r) * w + c] = solid_angle(r);
    std::vector<double> rw(h, 0.0);
    cols.clear();
    cols.reserve(size_t(w) * h);
    std::vector<float4> t;
    const std::vector<uint32_t> none;
    for (uint32_t r = 0; r < h; ++r) {
        const std::vector<double> span(tw.begin() + size_t(r) * w, tw.begin() + size_t(r + 1) * w);
        for (double x : span) rw[r] += x;
        if (!build_alias_table(span, none, t, err)) return false;
        cols.insert(cols.end(), t.begin(), t.end());
    }
    return build_alias_table(rw, none, rows, err);
}

}  // namespace re

namespace {

template <typename T>
T* carve(char*& cursor, size_t count) {
    T* p = reinterpret_cast<T*>(cursor);
    cursor += ((count * sizeof(T) + 255) / 256) * 256;
    return p;
}

// 128-entry traversal stacks when a scene of the staged launch needs more
// than 64 (child-pair: deeper than 64 levels; four-wide: a stack bound above
// 64).
bool frame_stack_deep(const re_renderer* r) { return r->batch_deep; }

constexpr size_t kGraphCache = 8;

void drop_graph(re_renderer* r) {
    for (auto& g : r->graphs) cudaGraphExecDestroy(g.second);
    r->graphs.clear();
}

// Profiling hooks of one recorded frame: counting kernels (cnt != null) or
// events between the stage launches (ev != null, 2 + 3 * depth + 2 events).
struct FrameHooks {
    unsigned long long* cnt = nullptr;
    cudaEvent_t* ev = nullptr;
};

// Traversal kernels at a CTA size of 128, 256 or 512 threads.
template <int STACK, int MODE, typename G>
void launch_intersect_tb(int tb, G&& grid_tb, cudaStream_t s, const WfDevice& d, uint32_t b) {
    if (tb == 512) {
        auto k = k_intersect<STACK, MODE, 512>;
        k<<<grid_tb(k, 512), 512, 0, s>>>(d, b);
    } else if (tb == 256) {
        auto k = k_intersect<STACK, MODE, 256>;
        k<<<grid_tb(k, 256), 256, 0, s>>>(d, b);
    } else {
        auto k = k_intersect<STACK, MODE, 128>;
        k<<<grid_tb(k, 128), 128, 0, s>>>(d, b);
    }
}
template <int STACK, int MODE, typename G>
void launch_shadow_tb(int tb, G&& grid_tb, cudaStream_t s, const WfDevice& d, uint32_t b) {
    if (tb == 512) {
        auto k = k_shadow<STACK, false, MODE, 512>;
        k<<<grid_tb(k, 512), 512, 0, s>>>(d, b, nullptr);
    } else if (tb == 256) {
        auto k = k_shadow<STACK, false, MODE, 256>;
        k<<<grid_tb(k, 256), 256, 0, s>>>(d, b, nullptr);
    } else {
        auto k = k_shadow<STACK, false, MODE, 128>;
        k<<<grid_tb(k, 128), 128, 0, s>>>(d, b, nullptr);
    }
}

template <bool FUSED, int STACK, typename G>
void launch_shade(uint32_t variant, G&& grid_for, cudaStream_t s, const WfDevice& d, uint32_t b) {
    if (variant == 3) {
        auto ka = k_shade_a<FUSED, STACK, false>;
        ka<<<grid_for(ka), 128, 0, s>>>(d, b);
        auto kb = k_shade_b<false>;
        kb<<<grid_for(kb), 128, 0, s>>>(d, b);
    } else if (variant == 4) {
        auto ka = k_shade_a<FUSED, STACK, true>;
        ka<<<grid_for(ka), 128, 0, s>>>(d, b);
        auto kb = k_shade_b<true>;
        kb<<<grid_for(kb), 128, 0, s>>>(d, b);
    } else if (variant == 5) {
        auto kp = k_shade_prep<FUSED, STACK>;
        kp<<<grid_for(kp), 128, 0, s>>>(d, b);
        auto kn = k_shade_nee;
        kn<<<grid_for(kn), 128, 0, s>>>(d, b);
        auto kb = k_shade_b<true>;
        kb<<<grid_for(kb), 128, 0, s>>>(d, b);
    } else if (variant == 6) {
        auto kp = k_shade_prep_capped<FUSED, STACK, 6>;
        kp<<<grid_for(kp), 128, 0, s>>>(d, b);
        auto kn = k_shade_nee_capped<6>;
        kn<<<grid_for(kn), 128, 0, s>>>(d, b);
        auto kb = k_shade_b_capped<6>;
        kb<<<grid_for(kb), 128, 0, s>>>(d, b);
    } else if (variant == 7) {
        auto kp = k_shade_prep_capped<FUSED, STACK, 5>;
        kp<<<grid_for(kp), 128, 0, s>>>(d, b);
        auto kn = k_shade_nee_capped<5>;
        kn<<<grid_for(kn), 128, 0, s>>>(d, b);
        auto kb = k_shade_b_capped<5>;
        kb<<<grid_for(kb), 128, 0, s>>>(d, b);
    } else if (variant == 1) {
        auto k = k_shade<FUSED, STACK, 1>;
        k<<<grid_for(k), 128, 0, s>>>(d, b);
    } else if (variant == 2) {
        auto k = k_shade<FUSED, STACK, 2>;
        k<<<grid_for(k), 128, 0, s>>>(d, b);
    } else {
        auto k = k_shade_v0<FUSED, STACK>;
        k<<<grid_for(k), 128, 0, s>>>(d, b);
    }
}

// Records one launch of the staged batch.  Grids do not depend on the batch
// (persistent stage kernels sized by occupancy, grid-stride RayGen / ReSTIR /
// Resolve), so the recorded sequence replays for every batch of the same
// depth: one CUDA graph per (depth, stack depth, ReSTIR on/off, tuning).
template <int STACK>
cudaError_t record_frame_t(re_renderer* r, uint32_t depth, cudaStream_t s, const FrameHooks& hk) {
    const WfDevice& d = r->dev;
    cudaError_t e = cudaMemsetAsync(r->counters.ptr, 0, kCounterWords * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    uint32_t evi = 0;
    auto mark = [&] {
        if (hk.ev != nullptr) cudaEventRecord(hk.ev[evi++], s);
    };
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, r->device);
    const uint32_t stride_blocks = uint32_t(sms) * 8u;
    mark();
    k_raygen<<<stride_blocks, 256, 0, s>>>(d);
    mark();
    auto grid_for = [&](auto kernel) {
        int per = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, 128, 0);
        if (r->tuning.blocks_per_sm != 0) per = std::min<int>(per, int(r->tuning.blocks_per_sm));
        per = std::max(per, 1);
        return sms * per;
    };
    // Traversal kernels at the tuned CTA size: as many CTAs per SM as fit
    // (blocks_per_sm, counted in 128-thread units, caps the warps per SM).
    const int tb = int(r->tuning.block_size);
    auto grid_tb = [&](auto kernel, int threads) {
        int per = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, 0);
        if (r->tuning.blocks_per_sm != 0)
            per = std::min<int>(per, std::max(1, int(r->tuning.blocks_per_sm) * 128 / threads));
        per = std::max(per, 1);
        return sms * per;
    };
    const bool fuse = r->tuning.fuse_intersect_shade != 0 && hk.cnt == nullptr && hk.ev == nullptr;
    for (uint32_t b = 0; b < depth; ++b) {
        if (fuse) {
            launch_shade<true, STACK>(r->tuning.shade_variant, grid_for, s, d, b);
        } else {
            if (hk.cnt != nullptr && r->batch_eight != 0u) {
                auto ki = r->batch_eight == 6u ? k_intersect_counted<STACK, 6> : k_intersect_counted<STACK, 5>;
                ki<<<grid_for(ki), 128, 0, s>>>(d, b, hk.cnt);
            } else if (r->batch_eight == 5u) {
                launch_intersect_tb<STACK, 5>(tb, grid_tb, s, d, b);
            } else if (r->batch_eight == 6u) {
                launch_intersect_tb<STACK, 6>(tb, grid_tb, s, d, b);
            } else if (hk.cnt != nullptr && r->batch_wide && r->batch_loop >= 7u) {
                auto ki = k_intersect_counted<STACK, 7>;
                ki<<<grid_for(ki), 128, 0, s>>>(d, b, hk.cnt);
            } else if (hk.cnt != nullptr && r->batch_wide) {
                auto ki = k_intersect_counted<STACK, 2>;
                ki<<<grid_for(ki), 128, 0, s>>>(d, b, hk.cnt);
            } else if (hk.cnt != nullptr) {
                auto ki = k_intersect_counted<STACK, 0>;
                ki<<<grid_for(ki), 128, 0, s>>>(d, b, hk.cnt);
            } else if (r->batch_wide && r->tuning.traversal_refill != 0) {
                auto ki = k_intersect_refill<STACK, true>;
                ki<<<grid_for(ki), 128, 0, s>>>(d, b, std::min(r->tuning.traversal_refill, 32u));
            } else if (r->batch_wide && r->batch_loop == 4u) {
                launch_intersect_tb<STACK, 4>(tb, grid_tb, s, d, b);
            } else if (r->batch_wide && r->batch_loop == 7u) {
                launch_intersect_tb<STACK, 7>(tb, grid_tb, s, d, b);
            } else if (r->batch_wide && r->batch_loop == 8u) {
                launch_intersect_tb<STACK, 8>(tb, grid_tb, s, d, b);
            } else if (r->batch_wide) {
                launch_intersect_tb<STACK, 2>(tb, grid_tb, s, d, b);
            } else if (r->tuning.traversal_refill != 0) {
                auto ki = k_intersect_refill<STACK, false>;
                ki<<<grid_for(ki), 128, 0, s>>>(d, b, std::min(r->tuning.traversal_refill, 32u));
            } else if (r->batch_loop == 1u) {
                launch_intersect_tb<STACK, 1>(tb, grid_tb, s, d, b);
            } else {
                launch_intersect_tb<STACK, 0>(tb, grid_tb, s, d, b);
            }
            mark();
            launch_shade<false, STACK>(r->tuning.shade_variant, grid_for, s, d, b);
        }
        mark();
        if (hk.cnt != nullptr && r->batch_eight != 0u) {
            auto kh = r->batch_eight == 6u ? k_shadow<STACK, true, 6> : k_shadow<STACK, true, 5>;
            kh<<<grid_for(kh), 128, 0, s>>>(d, b, hk.cnt);
        } else if (r->batch_eight == 5u) {
            launch_shadow_tb<STACK, 5>(tb, grid_tb, s, d, b);
        } else if (r->batch_eight == 6u) {
            launch_shadow_tb<STACK, 6>(tb, grid_tb, s, d, b);
        } else if (hk.cnt != nullptr && r->batch_wide && r->batch_loop >= 7u) {
            auto kh = k_shadow<STACK, true, 7>;
            kh<<<grid_for(kh), 128, 0, s>>>(d, b, hk.cnt);
        } else if (hk.cnt != nullptr && r->batch_wide) {
            auto kh = k_shadow<STACK, true, 2>;
            kh<<<grid_for(kh), 128, 0, s>>>(d, b, hk.cnt);
        } else if (hk.cnt != nullptr) {
            auto kh = k_shadow<STACK, true, 0>;
            kh<<<grid_for(kh), 128, 0, s>>>(d, b, hk.cnt);
        } else if (r->batch_wide && r->tuning.traversal_refill != 0) {
            auto kh = k_shadow_refill<STACK, true>;
            kh<<<grid_for(kh), 128, 0, s>>>(d, b, std::min(r->tuning.traversal_refill, 32u));
        } else if (r->batch_wide && r->batch_loop == 4u) {
            launch_shadow_tb<STACK, 4>(tb, grid_tb, s, d, b);
        } else if (r->batch_wide && r->batch_loop == 7u) {
            launch_shadow_tb<STACK, 7>(tb, grid_tb, s, d, b);
        } else if (r->batch_wide && r->batch_loop == 8u) {
            launch_shadow_tb<STACK, 8>(tb, grid_tb, s, d, b);
        } else if (r->batch_wide) {
            launch_shadow_tb<STACK, 2>(tb, grid_tb, s, d, b);
        } else if (r->tuning.traversal_refill != 0) {
            auto kh = k_shadow_refill<STACK, false>;
            kh<<<grid_for(kh), 128, 0, s>>>(d, b, std::min(r->tuning.traversal_refill, 32u));
        } else if (r->batch_loop == 1u) {
            launch_shadow_tb<STACK, 1>(tb, grid_tb, s, d, b);
        } else {
            launch_shadow_tb<STACK, 0>(tb, grid_tb, s, d, b);
        }
        mark();
    }
    if (r->restir_active) {
        // Winner visibility walks the launch's hierarchy form: four-wide nodes
        // within the launch's stack, or child pairs with the binary depth.
        launch_restir(d, stride_blocks * 2u, r->batch_wide ? r->batch_deep : r->batch_deep_binary, r->batch_wide, s);
        mark();
    }
    k_resolve<<<stride_blocks, 256, 0, s>>>(d);
    mark();
    return cudaGetLastError();
}

cudaError_t record_frame(re_renderer* r, uint32_t depth, cudaStream_t s, const FrameHooks& hk = FrameHooks{}) {
    return frame_stack_deep(r) ? record_frame_t<128>(r, depth, s, hk) : record_frame_t<64>(r, depth, s, hk);
}

// ReSTIR state: two primary-surface planes and two published reservoir
// planes (ping-pong by each view's frame parity), the temporal reservoirs,
// rejection reasons and the ReSTIR direct planes: 996 B per path.
re_status ensure_restir_buffers(re_renderer* r) {
    if (r->restir_arena.ptr != nullptr) return RE_SUCCESS;
    const size_t c = r->capacity;
    const size_t bytes = c * (2 * 96 + 3 * 256 + 4 + 32) + 16 * 256;
    RE_CUDA_TRY(r->restir_arena.reserve(bytes));
    RE_CUDA_TRY(cudaMemset(r->restir_arena.ptr, 0, bytes));
    char* cur = static_cast<char*>(r->restir_arena.ptr);
    WfDevice& d = r->dev;
    d.prim[0] = carve<float4>(cur, c * 6);
    d.prim[1] = carve<float4>(cur, c * 6);
    d.rs_temporal = carve<Reservoir>(cur, c);
    d.rs_published[0] = carve<Reservoir>(cur, c);
    d.rs_published[1] = carve<Reservoir>(cur, c);
    d.rs_reasons = carve<uint32_t>(cur, c);
    d.rs_direct = carve<float4>(cur, 2 * c);
    drop_graph(r);
    return RE_SUCCESS;
}

// PbrFrameSamplingIsValidL6 (pbr_l6_types.hlsli:270-316) and the RayGen
// contract checks (RayGen.hlsl:21-39), evaluated once on the host.
re_status validate_frame(const re_renderer* r, const re_frame_constants* f) {
    const uint32_t w = f->image.x, h = f->image.y, depth = f->image.w;
    const float rs = f->russian_roulette.x, rmin = f->russian_roulette.y, rmax = f->russian_roulette.z,
                eps = f->russian_roulette.w;
    const bool frame_ok = w != 0 && h != 0 && f->image.z != 0xffffffffu && depth != 0 && w <= 16384 &&
                          h <= 16384 && f->sampling.z <= 1u && f->sampling.w <= 3u && std::isfinite(rs) &&
                          rs >= 0.f && std::floor(rs) == rs && std::isfinite(rmin) && std::isfinite(rmax) &&
                          rmin > 0.f && rmin <= rmax && rmax <= 1.f && std::isfinite(eps) && eps > 0.f;
    if (!frame_ok) return set_error(RE_INVALID_ARGUMENT, "frame constants violate the PBR frame contract");
    if (uint64_t(w) * h > r->capacity) return set_error(RE_INVALID_ARGUMENT, "frame exceeds the path capacity");
    if (depth > r->max_depth) return set_error(RE_INVALID_ARGUMENT, "frame depth exceeds the renderer maximum");
    if (f->output.w != RE_SHADOW_PHYSICAL) return set_error(RE_UNSUPPORTED, "only the Physical shadow method is built");
    if (f->output.z != 0u) return set_error(RE_UNSUPPORTED, "only the PBR transport is built");
    return RE_SUCCESS;
}

// Frame parameters of one view.  ReSTIR parameters follow
// BuildReSTIRFrameParameters (GpuRestirParametersV3); a profiling pass runs
// the passes on the parity the next frame will use and commits nothing.
void fill_view(re_renderer* r, const re_view_desc& v, uint32_t profile, FrameParams& fp) {
    const re_frame_constants* f = v.frame;
    const uint32_t w = f->image.x, h = f->image.y;
    fp = FrameParams{};
    fp.cam_pos = mk(f->camera_position_tan_half_fov.x, f->camera_position_tan_half_fov.y,
                    f->camera_position_tan_half_fov.z);
    fp.tan_half_fov = f->camera_position_tan_half_fov.w;
    fp.cam_fwd = mk(f->camera_forward_aspect.x, f->camera_forward_aspect.y, f->camera_forward_aspect.z);
    fp.aspect = f->camera_forward_aspect.w;
    fp.cam_right = mk(f->camera_right_lens_radius.x, f->camera_right_lens_radius.y, f->camera_right_lens_radius.z);
    fp.cam_up = mk(f->camera_up_exposure.x, f->camera_up_exposure.y, f->camera_up_exposure.z);
    fp.width = w;
    fp.height = h;
    fp.sample = f->image.z;
    fp.max_depth = f->image.w;
    fp.seed_lo = f->sampling.x;
    fp.seed_hi = f->sampling.y;
    fp.estimator = f->sampling.w;
    fp.stream = f->output.x;
    fp.rr_start = f->russian_roulette.x;
    fp.rr_min = f->russian_roulette.y;
    fp.rr_max = f->russian_roulette.z;
    fp.eps = f->russian_roulette.w;
    fp.accumulate = v.accumulate;
    fp.pixel_count = w * h;
    fp.profile = profile;
    fp.path_offset = v.path_offset;
    fp.scene_slot = v.scene_slot;
    bool xf_zero = true;
    for (int k = 0; k < 3; ++k) {
        const re_float4 a = f->environment_to_world[k], b = f->world_to_environment[k];
        fp.env_xf[k] = make_float4(a.x, a.y, a.z, a.w);
        fp.env_xf[3 + k] = make_float4(b.x, b.y, b.z, b.w);
        xf_zero = xf_zero && a.x == 0.f && a.y == 0.f && a.z == 0.f && b.x == 0.f && b.y == 0.f && b.z == 0.f;
    }
    if (xf_zero) {
        for (int k = 0; k < 3; ++k) {
            fp.env_xf[k] = make_float4(k == 0 ? 1.f : 0.f, k == 1 ? 1.f : 0.f, k == 2 ? 1.f : 0.f, 0.f);
            fp.env_xf[3 + k] = fp.env_xf[k];
        }
    }
    fp.rs = RestirParams{};
    if (f->sampling.w != RE_ESTIMATOR_RESTIR_PRIMARY) return;
    const SlotState& sl = r->slots[v.scene_slot];
    RestirView& st = r->rs_views[v.view_key];
    const bool resized = w != st.last_w || h != st.last_h;
    const uint32_t res_gen = st.resolution_gen + (resized ? 1u : 0u);
    const uint32_t parity = st.parity ^ 1u;
    const re_restir_config& c = r->restir;
    RestirParams& q = fp.rs;
    q.enabled = 1u;
    q.candidates = c.candidates;
    q.neighbors = c.spatial_neighbors;
    q.max_m = c.max_m;
    q.max_age = c.max_history_age;
    q.history_enabled = c.temporal;
    q.neighbor_mode = c.neighbor_mode;
    q.parity = parity;
    q.scene_gen = sl.generation;
    q.light_gen = sl.generation;
    q.camera_gen = r->camera_epoch;
    q.resolution_gen = res_gen;
    q.history_gen = 1u;
    q.frame_lo = f->image.z;
    q.frame_hi = 0u;
    q.prev_valid = st.has_prev ? 1u : 0u;
    q.candidate_source = sl.light_selection == RE_LIGHT_SELECTION_POWER ? 2u : 1u;
    q.light_count = sl.light_count;
    q.prev_light_count = st.prev_light_count;
    q.normal_cos = c.normal_cos;
    q.rel_depth = c.relative_depth;
    q.position_dist = c.position_distance;
    q.estimator = c.estimator;
    q.disk_radius = c.disk_radius;
    q.prev_pos = st.prev.cam_pos;
    q.prev_tan = st.prev.tan_half_fov;
    q.prev_fwd = st.prev.cam_fwd;
    q.prev_aspect = st.prev.aspect;
    q.prev_right = st.prev.cam_right;
    q.prev_up = st.prev.cam_up;
    if (!profile) {
        st.parity = parity;
        st.resolution_gen = res_gen;
        st.last_w = w;
        st.last_h = h;
        st.has_prev = true;
        st.prev = fp;
        st.prev_light_count = sl.light_count;
    }
}

// Validates and uploads the views of one launch (ordered by scene slot, then
// path offset).
re_status stage_views(re_renderer* r, const re_view_desc* views, uint32_t n, uint32_t profile, cudaStream_t s) {
    if (r == nullptr || views == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (n == 0 || n > kMaxViews) return set_error(RE_INVALID_ARGUMENT, "a launch takes 1 to 256 views");
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; ++i) {
        const re_view_desc& v = views[i];
        if (v.frame == nullptr) return set_error(RE_INVALID_ARGUMENT, "view without frame constants");
        if (v.scene_slot >= kMaxSceneSlots || r->slots[v.scene_slot].scene == nullptr)
            return set_error(RE_MISSING_SCENE, "view references an unbound scene slot");
        const re_status st = validate_frame(r, v.frame);
        if (st != RE_SUCCESS) return st;
        if (v.frame->sampling.w == RE_ESTIMATOR_RESTIR_PRIMARY && r->slots[v.scene_slot].env_light != 0xffffffffu)
            return set_error(RE_UNSUPPORTED, "ReSTIR DI over a scene with an environment light is not built");
        const uint64_t end = uint64_t(v.path_offset) + uint64_t(v.frame->image.x) * v.frame->image.y;
        if (end > r->capacity) return set_error(RE_INVALID_ARGUMENT, "view's paths exceed the path capacity");
        order[i] = i;
    }
    std::sort(order.begin(), order.end(),
              [&](uint32_t a, uint32_t b) { return views[a].path_offset < views[b].path_offset; });
    uint32_t path_end = 0, depth = 0;
    bool restir = false, deep = false;
    for (uint32_t k = 0; k < n; ++k) {
        const re_view_desc& v = views[order[k]];
        deep |= r->slots[v.scene_slot].scene->flat.max_depth > 64;
        if (v.path_offset < path_end) return set_error(RE_INVALID_ARGUMENT, "views' path ranges overlap");
        path_end = v.path_offset + v.frame->image.x * v.frame->image.y;
        depth = std::max(depth, v.frame->image.w);
        restir |= v.frame->sampling.w == RE_ESTIMATOR_RESTIR_PRIMARY;
    }
    static_assert(offsetof(SceneSlot, scene) == 0, "the slot's traversal view leads the record");
    // Traversal loop of the launch (split stages; the fused kernels walk
    // child pairs; with lane refill the four-wide modes take one node or leaf
    // per step).  Mode 3 chooses per launch:
    // four-wide nodes, with postponed leaves unless a scene of the launch is
    // an LBVH (one triangle per leaf: parking such leaves costs more than it
    // saves; several per leaf, as in the SAH trees, it pays).  Four-wide
    // needs every scene's wide nodes (built on first use) within the
    // 128-entry stack, else the launch falls back to the while-while loop.
    uint32_t loop = r->tuning.traversal_mode;
    if (loop == 3u) {
        bool lbvh = false;
        for (uint32_t k = 0; k < n; ++k) lbvh |= r->slots[views[k].scene_slot].scene->build_kind == RE_BUILD_LBVH;
        loop = lbvh ? 4u : 2u;
    }
    // Eight-wide nodes (5 plain, 6 compressed): built on first use; the
    // launch falls back to the four-wide loop when a scene's eight-wide
    // traversal could need more than 128 stack entries.
    uint32_t eight = (loop == 5u || loop == 6u) && r->tuning.fuse_intersect_shade == 0u ? loop : 0u;
    uint32_t eight_need = 0;
    if (eight != 0u) {
        RE_CUDA_TRY(cudaSetDevice(r->device));
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t slot = views[k].scene_slot;
            re_scene* sc = r->slots[slot].scene;
            if (sc->eight_node_count == 0u) {
                const re_status st = ensure_eight_layout(sc);
                if (st != RE_SUCCESS) return st;
            }
            if (!r->slots[slot].eight_view) {
                const TraceSceneView view = scene_view(sc);
                RE_CUDA_TRY(cudaMemcpy(static_cast<SceneSlot*>(r->scenes_table.ptr) + slot, &view, sizeof(view),
                                       cudaMemcpyHostToDevice));
                r->slots[slot].eight_view = true;
                r->slots[slot].wide_view = sc->wide_node_count != 0u;
            }
            eight_need = std::max(eight_need, sc->eight_stack_bound);
        }
        if (eight_need > 128u) {
            eight = 0u;
            loop = 4u;
        }
    }
    bool wide = (loop == 2u || loop == 4u || loop == 7u || loop == 8u) && r->tuning.fuse_intersect_shade == 0u;
    uint32_t wide_need = 0;
    if (wide) {
        RE_CUDA_TRY(cudaSetDevice(r->device));
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t slot = views[k].scene_slot;
            re_scene* sc = r->slots[slot].scene;
            if (sc->wide_node_count == 0u) {
                const re_status st = ensure_wide_layout(sc);
                if (st != RE_SUCCESS) return st;
            }
            if (!r->slots[slot].wide_view) {
                const TraceSceneView view = scene_view(sc);
                RE_CUDA_TRY(cudaMemcpy(static_cast<SceneSlot*>(r->scenes_table.ptr) + slot, &view, sizeof(view),
                                       cudaMemcpyHostToDevice));
                r->slots[slot].wide_view = true;
                r->slots[slot].eight_view = sc->eight_node_count != 0u;
            }
            wide_need = std::max(wide_need, sc->wide_stack_bound);
        }
        if (wide_need > 128u) wide = false;  // the child-pair loop for this launch
    }
    if (!wide && eight == 0u && loop != 0u) loop = 1u;
    // Launch order: scene-major, so the rays of one scene stay contiguous in
    // the queues and a launch that mixes scenes walks one hierarchy at a time.
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return views[a].scene_slot < views[b].scene_slot; });
    RE_CUDA_TRY(cudaSetDevice(r->device));
    if (restir) {
        const re_status st = ensure_restir_buffers(r);
        if (st != RE_SUCCESS) return st;
    }
    const uint32_t ring = r->ring_next;
    r->ring_next = (ring + 1u) % kFrameRing;
    if (r->ring_used[ring]) RE_CUDA_TRY(cudaEventSynchronize(r->ring_done[ring]));
    char* rec = r->host_frame + size_t(ring) * kFrameRecordBytes;
    FrameParams* fps = reinterpret_cast<FrameParams*>(rec + sizeof(BatchParams));
    uint32_t pixel_total = 0;
    for (uint32_t k = 0; k < n; ++k) {
        fill_view(r, views[order[k]], profile, fps[k]);
        fps[k].pixel_base = pixel_total;
        pixel_total += fps[k].pixel_count;
    }
    BatchParams bp{n, path_end, depth, profile, pixel_total, 0u, 0u, 0u};
    std::memcpy(rec, &bp, sizeof(bp));
    RE_CUDA_TRY(cudaMemcpyAsync(r->frame.ptr, rec, sizeof(BatchParams) + size_t(n) * sizeof(FrameParams),
                                cudaMemcpyHostToDevice, s));
    RE_CUDA_TRY(cudaEventRecord(r->ring_done[ring], s));
    r->ring_used[ring] = true;
    r->restir_active = restir;
    r->batch_deep_binary = deep;
    r->batch_wide = wide;
    r->batch_eight = eight;
    r->batch_loop = loop;
    r->batch_deep = eight != 0u ? eight_need > 64u : (wide ? wide_need > 64u : deep);
    r->batch_depth = depth;
    r->last_pixels = path_end;
    return RE_SUCCESS;
}

// One launch of the staged views: CUDA-graph replay (or direct launches).
re_status launch_staged(re_renderer* r, cudaStream_t s) {
    const uint32_t depth = r->batch_depth;
    RE_CUDA_TRY(cudaEventRecord(r->ev0, s));
    const uint64_t key = (uint64_t(depth) << 4) ^ (frame_stack_deep(r) ? 1 : 0) ^ (r->restir_active ? 2 : 0) ^
                         (r->batch_wide ? 4 : 0) ^ (r->batch_deep_binary ? 8 : 0) ^
                         (uint64_t(r->batch_loop) << 32);
    if (r->tuning.use_graph) {
        auto it = std::find_if(r->graphs.begin(), r->graphs.end(),
                               [key](const std::pair<uint64_t, cudaGraphExec_t>& g) { return g.first == key; });
        cudaGraphExec_t exec = nullptr;
        if (it != r->graphs.end()) {
            exec = it->second;
            r->graphs.erase(it);
        } else {
            if (r->graphs.size() >= kGraphCache) {
                cudaGraphExecDestroy(r->graphs.front().second);
                r->graphs.erase(r->graphs.begin());
            }
            cudaStream_t cap;
            RE_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            cudaGraph_t g;
            RE_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = record_frame(r, depth, cap);
            cudaError_t e2 = cudaStreamEndCapture(cap, &g);
            cudaStreamDestroy(cap);
            RE_CUDA_TRY(e);
            RE_CUDA_TRY(e2);
            e = cudaGraphInstantiate(&exec, g, 0);
            cudaGraphDestroy(g);
            RE_CUDA_TRY(e);
        }
        r->graphs.emplace_back(key, exec);
        RE_CUDA_TRY(cudaGraphLaunch(exec, s));
    } else {
        RE_CUDA_TRY(record_frame(r, depth, s));
    }
    RE_CUDA_TRY(cudaEventRecord(r->ev1, s));
    RE_CUDA_TRY(cudaMemcpyAsync(r->host_counters, r->counters.ptr, kCounterWords * sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, s));
    RE_CUDA_TRY(cudaEventRecord(r->ev1, s));
    r->frame_pending = true;
    return RE_SUCCESS;
}

re_status single_view(re_renderer* r, const re_frame_constants* f, uint32_t accumulate, uint32_t profile,
                      cudaStream_t s) {
    if (r == nullptr || f == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (r->scene == nullptr) return set_error(RE_MISSING_SCENE, "no scene bound");
    re_view_desc v{};
    v.frame = f;
    v.scene_slot = 0;
    v.path_offset = 0;
    v.accumulate = accumulate;
    v.view_key = 0;
    const re_status st = stage_views(r, &v, 1u, profile, s);
    if (st != RE_SUCCESS) return st;
    if (!accumulate && !profile) RE_CUDA_TRY(cudaMemsetAsync(r->film_frames.ptr, 0, 32, s));
    return RE_SUCCESS;
}

}  // namespace

extern "C" {

RE_API re_status re_renderer_create(const re_renderer_desc* desc, re_renderer** out) {
    if (desc == nullptr || out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (desc->max_width == 0 || desc->max_height == 0 || desc->max_width > 16384 || desc->max_height > 16384)
        return set_error(RE_INVALID_ARGUMENT, "renderer dimensions must be in [1, 16384]");
    if (desc->max_depth == 0 || desc->max_depth > kMaxDepth)
        return set_error(RE_INVALID_ARGUMENT, "maximum depth must be in [1, 16]");
    const uint64_t cap64 = uint64_t(desc->max_width) * desc->max_height;
    if (cap64 > kPathMask) return set_error(RE_INVALID_ARGUMENT, "path capacity exceeds 2^27");
    RE_CUDA_TRY(cudaSetDevice(int(desc->device)));
    auto r = new re_renderer();
    r->device = int(desc->device);
    r->max_w = desc->max_width;
    r->max_h = desc->max_height;
    r->max_depth = desc->max_depth;
    r->capacity = uint32_t(cap64);
    re_restir_default_config(&r->restir);
    const size_t c = r->capacity;
    // 16 B lanes per path: 3 throughput + 5 accumulators + 3 previous-vertex +
    // ident + 2x2 ray queue + hit + 5 shadow + film sum + sample + 4 G-buffer +
    // 3 split-Shade records (31 of the 34 reserved; the rest, with the fixed
    // term, covers the 256 B alignment of each array).
    const size_t bytes = c * 16u * 34u + c * 4u * 2u + 64u * 256u;
    cudaError_t e = r->arena.reserve(bytes);
    if (e != cudaSuccess) {
        delete r;
        return set_error(e == cudaErrorMemoryAllocation ? RE_OUT_OF_MEMORY : RE_CUDA_ERROR,
                         std::string("path-state allocation failed: ") + cudaGetErrorString(e));
    }
    char* cur = static_cast<char*>(r->arena.ptr);
    WfDevice& d = r->dev;
    d.capacity = r->capacity;
    d.beta = carve<float4>(cur, c);
    d.beta_d = carve<float4>(cur, c);
    d.beta_s = carve<float4>(cur, c);
    d.acc_cam = carve<float4>(cur, c);
    d.acc_dd = carve<float4>(cur, c);
    d.acc_ds = carve<float4>(cur, c);
    d.acc_id = carve<float4>(cur, c);
    d.acc_is = carve<float4>(cur, c);
    d.prev_pos_pdf = carve<float4>(cur, c);
    d.prev_ng = carve<float4>(cur, c);
    d.prev_ns = carve<float4>(cur, c);
    d.ident = carve<uint4>(cur, c);
    for (int k = 0; k < 2; ++k) {
        d.ray_o[k] = carve<float4>(cur, c);
        d.ray_d[k] = carve<float4>(cur, c);
        d.ray_path[k] = carve<uint32_t>(cur, c);
    }
    d.hit = carve<float4>(cur, c);
    d.sh_o = carve<float4>(cur, c);
    d.sh_d = carve<float4>(cur, c);
    d.sh_cd = carve<float4>(cur, c);
    d.sh_cs = carve<float4>(cur, c);
    d.sh_id = carve<uint4>(cur, c);
    d.film_sum = carve<float4>(cur, c);
    d.sample_out = carve<float4>(cur, c);
    d.gb_pos = carve<float4>(cur, c);
    d.gb_nrm = carve<float4>(cur, c);
    d.gb_alb = carve<float4>(cur, c);
    d.gb_id = carve<uint4>(cur, c);
    d.vx_pos = carve<float4>(cur, c);
    d.vx_ng = carve<float4>(cur, c);
    d.vx_ns = carve<float4>(cur, c);
    if (r->counters.reserve(kCounterWords * sizeof(uint32_t)) != cudaSuccess ||
        r->frame.reserve(kFrameRecordBytes) != cudaSuccess || r->film_frames.reserve(32) != cudaSuccess ||
        r->scenes_table.reserve(kMaxSceneSlots * sizeof(SceneSlot)) != cudaSuccess ||
        r->path_view.reserve(size_t(r->capacity) * sizeof(uint32_t)) != cudaSuccess ||
        cudaMallocHost(&r->host_frame, kFrameRecordBytes * kFrameRing) != cudaSuccess ||
        cudaMallocHost(&r->host_counters, kCounterWords * sizeof(uint32_t)) != cudaSuccess ||
        cudaEventCreate(&r->ev0) != cudaSuccess || cudaEventCreate(&r->ev1) != cudaSuccess) {
        delete r;
        return set_error(RE_OUT_OF_MEMORY, "renderer bookkeeping allocation failed");
    }
    d.counters = static_cast<uint32_t*>(r->counters.ptr);
    d.batch = static_cast<const BatchParams*>(r->frame.ptr);
    d.views = reinterpret_cast<const FrameParams*>(static_cast<char*>(r->frame.ptr) + sizeof(BatchParams));
    d.scenes = static_cast<const SceneSlot*>(r->scenes_table.ptr);
    d.path_view = static_cast<uint32_t*>(r->path_view.ptr);
    d.film_frames = static_cast<uint32_t*>(r->film_frames.ptr);
    cudaMemset(r->film_frames.ptr, 0, 32);
    cudaMemset(r->scenes_table.ptr, 0, kMaxSceneSlots * sizeof(SceneSlot));
    for (uint32_t k = 0; k < kFrameRing; ++k) {
        if (cudaEventCreateWithFlags(&r->ring_done[k], cudaEventDisableTiming) != cudaSuccess) {
            delete r;
            return set_error(RE_CUDA_ERROR, "event creation failed");
        }
    }
    cudaMemset(d.film_sum, 0, c * sizeof(float4));
    *out = r;
    return clear_error();
}

RE_API re_status re_renderer_destroy(re_renderer* r) {
    if (r != nullptr) {
        cudaSetDevice(r->device);
        cudaDeviceSynchronize();
    }
    delete r;
    return clear_error();
}

RE_API re_status re_renderer_set_tuning(re_renderer* r, const re_renderer_tuning* t) {
    if (r == nullptr || t == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (t->block_size != 128 && t->block_size != 256 && t->block_size != 512)
        return set_error(RE_UNSUPPORTED, "traversal block size must be 128, 256 or 512");
    if (t->shade_variant > 7) return set_error(RE_INVALID_ARGUMENT, "shade variant must be 0 to 7");
    if (t->traversal_mode > 8) return set_error(RE_INVALID_ARGUMENT, "traversal mode must be 0 to 8");
    r->tuning = *t;
    drop_graph(r);
    return clear_error();
}

RE_API re_status re_renderer_bind_scene(re_renderer* r, uint32_t slot, re_scene* scene, const re_material* materials,
                                        uint32_t material_count, const re_light* lights, uint32_t light_count,
                                        const re_float4* fixtures, uint32_t fixture_count, uint32_t light_selection,
                                        float scene_radius) {
    if (r == nullptr || scene == nullptr) return set_error(RE_MISSING_SCENE, "renderer or scene is null");
    if (slot >= kMaxSceneSlots) return set_error(RE_INVALID_ARGUMENT, "scene slot out of range");
    if (scene->device != r->device) return set_error(RE_INVALID_ARGUMENT, "scene lives on another device");
    if (material_count == 0 || materials == nullptr) return set_error(RE_INVALID_ARGUMENT, "no materials");
    if (light_selection > RE_LIGHT_SELECTION_POWER) return set_error(RE_INVALID_ARGUMENT, "unknown light selection");
    RE_CUDA_TRY(cudaSetDevice(r->device));
    // Top-level light distribution (BuildTopLevelLightDistribution,
    // MegakernelBridge.cpp:403-455): enabled lights only.
    // One enabled environment light at most, and only with a map set for
    // the slot (Wave2Runtime.cpp:560-612).
    SlotState& pre = r->slots[slot];
    uint32_t env_light = 0xffffffffu;
    for (uint32_t i = 0; i < light_count; ++i) {
        if (lights[i].identity.x != RE_LIGHT_ENVIRONMENT || (lights[i].identity.y & RE_LIGHT_FLAG_ENABLED) == 0u)
            continue;
        if (env_light != 0xffffffffu)
            return set_error(RE_INVALID_ARGUMENT, "one active environment light per scene is supported");
        env_light = i;
    }
    if (env_light != 0xffffffffu && pre.env_width == 0u)
        return set_error(RE_INVALID_ARGUMENT,
                         "an enabled environment light requires an environment map (re_renderer_set_environment)");
    std::vector<double> weights;
    std::vector<uint32_t> items;
    for (uint32_t i = 0; i < light_count; ++i) {
        if ((lights[i].identity.y & RE_LIGHT_FLAG_ENABLED) == 0u) continue;
        weights.push_back(light_selection == RE_LIGHT_SELECTION_UNIFORM
                              ? 1.0
                              : light_power(lights[i], scene_radius, pre.env_integrated));
        items.push_back(i);
    }
    std::vector<float4> alias;
    std::string err;
    if (!build_alias_table(weights, items, alias, err)) return set_error(RE_INVALID_ARGUMENT, err);
    std::vector<float> pmf(std::max(1u, light_count), 0.f);
    for (const float4& a : alias) {
        uint32_t item;
        std::memcpy(&item, &a.w, 4);
        pmf[item] = a.y;
    }
    // Emitter map per leaf-ordered triangle: (instance, primitive) -> light
    // (BuildEmitterMap, MegakernelBridge.cpp:353-401).
    std::unordered_map<uint64_t, uint32_t> emap;
    for (uint32_t i = 0; i < light_count; ++i) {
        if (lights[i].identity.x != RE_LIGHT_EMISSIVE_TRIANGLE) continue;
        const uint64_t key = (uint64_t(lights[i].payload.w) << 32) | lights[i].identity.w;
        if (!emap.emplace(key, i).second)
            return set_error(RE_INVALID_ARGUMENT, "multiple emissive lights reference the same instance/primitive pair");
    }
    const uint32_t n = scene->triangle_count;
    std::vector<uint32_t> em(n, 0xffffffffu);
    if (!emap.empty()) {
        std::vector<DeviceTriangle> tris(n);
        RE_CUDA_TRY(cudaMemcpy(tris.data(), scene->tris.ptr, n * sizeof(DeviceTriangle), cudaMemcpyDeviceToHost));
        for (uint32_t t = 0; t < n; ++t) {
            const uint64_t key = (uint64_t(tris[t].key[0]) << 32) | tris[t].key[1];
            auto it = emap.find(key);
            if (it != emap.end()) em[t] = it->second;
        }
    }
    // Launches in flight may still read the slot's tables.
    RE_CUDA_TRY(cudaDeviceSynchronize());
    SlotState& sl = r->slots[slot];
    RE_CUDA_TRY(sl.materials.reserve(size_t(material_count) * sizeof(re_material)));
    RE_CUDA_TRY(cudaMemcpy(sl.materials.ptr, materials, size_t(material_count) * sizeof(re_material),
                           cudaMemcpyHostToDevice));
    RE_CUDA_TRY(sl.lights.reserve(std::max<size_t>(1, light_count) * sizeof(re_light)));
    if (light_count)
        RE_CUDA_TRY(cudaMemcpy(sl.lights.ptr, lights, size_t(light_count) * sizeof(re_light), cudaMemcpyHostToDevice));
    RE_CUDA_TRY(sl.alias.reserve(std::max<size_t>(1, alias.size()) * sizeof(float4)));
    if (!alias.empty())
        RE_CUDA_TRY(cudaMemcpy(sl.alias.ptr, alias.data(), alias.size() * sizeof(float4), cudaMemcpyHostToDevice));
    RE_CUDA_TRY(sl.pmf.reserve(pmf.size() * sizeof(float)));
    RE_CUDA_TRY(cudaMemcpy(sl.pmf.ptr, pmf.data(), pmf.size() * sizeof(float), cudaMemcpyHostToDevice));
    RE_CUDA_TRY(sl.fixtures.reserve(std::max<size_t>(1, fixture_count) * 4 * sizeof(float4)));
    if (fixture_count)
        RE_CUDA_TRY(cudaMemcpy(sl.fixtures.ptr, fixtures, size_t(fixture_count) * 4 * sizeof(float4),
                               cudaMemcpyHostToDevice));
    RE_CUDA_TRY(sl.emitter.reserve(size_t(n) * sizeof(uint32_t)));
    RE_CUDA_TRY(cudaMemcpy(sl.emitter.ptr, em.data(), size_t(n) * sizeof(uint32_t), cudaMemcpyHostToDevice));
    sl.scene = scene;
    sl.wide_view = scene->wide_node_count != 0u;
    sl.eight_view = scene->eight_node_count != 0u;
    sl.generation = ++r->generation_counter;  // ReSTIR history of another scene / light set is rejected
    sl.light_selection = light_selection;
    sl.material_count = material_count;
    sl.light_count = light_count;
    sl.alias_count = uint32_t(alias.size());
    sl.fixture_count = fixture_count;
    sl.env_light = env_light;
    if (slot == 0) r->scene = scene;
    SceneSlot dv{};
    dv.scene = scene_view(scene);
    dv.attrs = static_cast<const float4*>(scene->attrs.ptr);
    dv.emitter = static_cast<const uint32_t*>(sl.emitter.ptr);
    dv.materials = static_cast<const float4*>(sl.materials.ptr);
    dv.material_count = material_count;
    dv.lights.lights = static_cast<const float4*>(sl.lights.ptr);
    dv.lights.alias = static_cast<const float4*>(sl.alias.ptr);
    dv.lights.pmf_by_light = static_cast<const float*>(sl.pmf.ptr);
    dv.lights.fixtures = static_cast<const float4*>(sl.fixtures.ptr);
    dv.lights.light_count = light_count;
    dv.lights.alias_count = sl.alias_count;
    dv.lights.fixture_count = fixture_count;
    dv.lights.env_light = env_light;
    dv.lights.env_texels = static_cast<const float4*>(sl.env_texels.ptr);
    dv.lights.env_rows = static_cast<const float4*>(sl.env_rows.ptr);
    dv.lights.env_cols = static_cast<const float4*>(sl.env_cols.ptr);
    dv.lights.env_width = env_light != 0xffffffffu ? sl.env_width : 0u;
    dv.lights.env_height = env_light != 0xffffffffu ? sl.env_height : 0u;
    dv.lights.env_uniform = sl.env_uniform;
    RE_CUDA_TRY(cudaMemcpy(static_cast<SceneSlot*>(r->scenes_table.ptr) + slot, &dv, sizeof(SceneSlot),
                           cudaMemcpyHostToDevice));
    return clear_error();
}

RE_API re_status re_renderer_set_scene(re_renderer* r, re_scene* scene, const re_material* materials,
                                       uint32_t material_count, const re_light* lights, uint32_t light_count,
                                       const re_float4* fixtures, uint32_t fixture_count, uint32_t light_selection,
                                       float scene_radius) {
    return re_renderer_bind_scene(r, 0u, scene, materials, material_count, lights, light_count, fixtures,
                                  fixture_count, light_selection, scene_radius);
}

RE_API re_status re_renderer_set_environment(re_renderer* r, uint32_t slot, const re_float4* texels, uint32_t width,
                                             uint32_t height) {
    if (r == nullptr || slot >= kMaxSceneSlots) return set_error(RE_INVALID_ARGUMENT, "bad renderer or slot");
    SlotState& sl = r->slots[slot];
    if (sl.scene != nullptr)
        return set_error(RE_INVALID_ARGUMENT, "set the environment of a slot before binding its scene");
    if (texels == nullptr) {
        sl.env_texels.release();
        sl.env_rows.release();
        sl.env_cols.release();
        sl.env_width = sl.env_height = sl.env_uniform = 0u;
        sl.env_integrated = 0.0;
        return clear_error();
    }
    if (width == 0u || height == 0u || uint64_t(width) * height > 0xffffffffull)
        return set_error(RE_INVALID_ARGUMENT, "environment dimensions must be non-zero and index in 32 bits");
    const size_t n = size_t(width) * height;
    // Linear luminance per texel (Wave2Runtime.cpp:589-600), validated as there.
    std::vector<float> lum(n);
    for (size_t i = 0; i < n; ++i) {
        const re_float4 t = texels[i];
        if (!std::isfinite(t.x) || !std::isfinite(t.y) || !std::isfinite(t.z) || !std::isfinite(t.w) || t.x < 0.f ||
            t.y < 0.f || t.z < 0.f)
            return set_error(RE_INVALID_ARGUMENT, "environment contains invalid linear radiance");
        lum[i] = 0.2126f * t.x + 0.7152f * t.y + 0.0722f * t.z;
    }
    std::vector<float4> rows, cols;
    double integrated = 0.0;
    bool fallback = false;
    std::string err;
    if (!build_environment_distribution(width, height, lum, rows, cols, integrated, fallback, err))
        return set_error(RE_INVALID_ARGUMENT, err);
    RE_CUDA_TRY(cudaSetDevice(r->device));
    RE_CUDA_TRY(sl.env_texels.reserve(n * sizeof(float4)));
    RE_CUDA_TRY(cudaMemcpy(sl.env_texels.ptr, texels, n * sizeof(float4), cudaMemcpyHostToDevice));
    RE_CUDA_TRY(sl.env_rows.reserve(rows.size() * sizeof(float4)));
    RE_CUDA_TRY(cudaMemcpy(sl.env_rows.ptr, rows.data(), rows.size() * sizeof(float4), cudaMemcpyHostToDevice));
    RE_CUDA_TRY(sl.env_cols.reserve(cols.size() * sizeof(float4)));
    RE_CUDA_TRY(cudaMemcpy(sl.env_cols.ptr, cols.data(), cols.size() * sizeof(float4), cudaMemcpyHostToDevice));
    sl.env_width = width;
    sl.env_height = height;
    sl.env_uniform = fallback ? 1u : 0u;
    sl.env_integrated = integrated;
    return clear_error();
}

RE_API re_status re_renderer_environment_tables(re_renderer* r, uint32_t slot, re_float4* rows_out,
                                                re_float4* columns_out, double* integrated_luminance) {
    if (r == nullptr || slot >= kMaxSceneSlots) return set_error(RE_INVALID_ARGUMENT, "bad renderer or slot");
    const SlotState& sl = r->slots[slot];
    if (sl.env_width == 0u) return set_error(RE_INVALID_ARGUMENT, "the slot has no environment map");
    RE_CUDA_TRY(cudaSetDevice(r->device));
    if (rows_out)
        RE_CUDA_TRY(cudaMemcpy(rows_out, sl.env_rows.ptr, size_t(sl.env_height) * sizeof(float4),
                               cudaMemcpyDeviceToHost));
    if (columns_out)
        RE_CUDA_TRY(cudaMemcpy(columns_out, sl.env_cols.ptr, size_t(sl.env_height) * sl.env_width * sizeof(float4),
                               cudaMemcpyDeviceToHost));
    if (integrated_luminance) *integrated_luminance = sl.env_integrated;
    return clear_error();
}

RE_API re_status re_renderer_unbind_scene(re_renderer* r, uint32_t slot) {
    if (r == nullptr || slot >= kMaxSceneSlots) return set_error(RE_INVALID_ARGUMENT, "bad renderer or slot");
    RE_CUDA_TRY(cudaSetDevice(r->device));
    RE_CUDA_TRY(cudaDeviceSynchronize());
    SlotState& sl = r->slots[slot];
    sl = SlotState{};
    if (slot == 0) r->scene = nullptr;
    RE_CUDA_TRY(cudaMemset(static_cast<SceneSlot*>(r->scenes_table.ptr) + slot, 0, sizeof(SceneSlot)));
    return clear_error();
}

RE_API re_status re_renderer_render(re_renderer* r, const re_frame_constants* f, uint32_t accumulate, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    re_status st = single_view(r, f, accumulate, 0u, s);
    if (st != RE_SUCCESS) return st;
    st = launch_staged(r, s);
    return st == RE_SUCCESS ? clear_error() : st;
}

RE_API re_status re_renderer_render_views(re_renderer* r, const re_view_desc* views, uint32_t view_count,
                                          void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    re_status st = stage_views(r, views, view_count, 0u, s);
    if (st != RE_SUCCESS) return st;
    st = launch_staged(r, s);
    return st == RE_SUCCESS ? clear_error() : st;
}

RE_API re_status re_renderer_release_view(re_renderer* r, uint64_t view_key) {
    if (r == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    r->rs_views.erase(view_key);
    return clear_error();
}

RE_API re_status re_renderer_path_capacity(const re_renderer* r, uint32_t* out) {
    if (r == nullptr || out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    *out = r->capacity;
    return clear_error();
}

RE_API re_status re_renderer_collect(re_renderer* r, re_frame_telemetry* out) {
    if (r == nullptr || out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    RE_CUDA_TRY(cudaSetDevice(r->device));
    if (r->frame_pending) RE_CUDA_TRY(cudaEventSynchronize(r->ev1));
    re_frame_telemetry t{};
    const uint32_t* c = r->host_counters;
    for (uint32_t b = 0; b < kMaxDepth; ++b) {
        const uint32_t rays = std::min(c[b * kSlotsPerBounce + kSlotRays], r->capacity);
        const uint32_t sh = std::min(c[b * kSlotsPerBounce + kSlotShadows], r->capacity);
        t.path_rays += (b < r->max_depth) ? rays : 0;
        t.shadow_rays += (b < r->max_depth) ? sh : 0;
        t.active_per_bounce[b] = rays;
        t.shadow_per_bounce[b] = sh;
        t.non_finite += c[b * kSlotsPerBounce + kSlotNonFinite];
        t.negative_pdf += c[b * kSlotsPerBounce + kSlotNegativePdf];
    }
    t.fatal_mask = c[kSlotFatal];
    uint32_t words[8] = {};
    RE_CUDA_TRY(cudaMemcpy(words, r->film_frames.ptr, 32, cudaMemcpyDeviceToHost));
    t.frames_accumulated = words[0];
    std::memcpy(&t.total_path_rays, words + 2, 8);
    std::memcpy(&t.total_shadow_rays, words + 4, 8);
    float ms = 0.f;
    if (r->frame_pending && cudaEventElapsedTime(&ms, r->ev0, r->ev1) == cudaSuccess) t.gpu_ms = ms;
    r->telemetry = t;
    *out = t;
    if (t.fatal_mask != 0u) return set_error(RE_FATAL_QUEUE, "wavefront frame reported fatal flags");
    return clear_error();
}

RE_API re_status re_renderer_film_pointer(re_renderer* r, uint32_t plane, void** out) {
    if (r == nullptr || out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    const WfDevice& d = r->dev;
    float4* p = nullptr;
    switch (plane) {
        case RE_FILM_MEAN: p = d.film_sum; break;
        case RE_FILM_SAMPLE: p = d.sample_out; break;
        case RE_FILM_CAMERA_EMISSION: p = d.acc_cam; break;
        case RE_FILM_DIRECT_DIFFUSE: p = d.acc_dd; break;
        case RE_FILM_DIRECT_SPECULAR: p = d.acc_ds; break;
        case RE_FILM_INDIRECT_DIFFUSE: p = d.acc_id; break;
        case RE_FILM_INDIRECT_SPECULAR: p = d.acc_is; break;
        case RE_FILM_PRIMARY_POSITION: p = d.gb_pos; break;
        case RE_FILM_PRIMARY_NORMAL: p = d.gb_nrm; break;
        case RE_FILM_PRIMARY_ALBEDO: p = d.gb_alb; break;
        case RE_FILM_PRIMARY_IDENTITY: p = reinterpret_cast<float4*>(d.gb_id); break;
        default: return set_error(RE_INVALID_ARGUMENT, "unknown film plane");
    }
    *out = p;
    return clear_error();
}

__global__ void k_film_mean(const float4* sum, float4* out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 s = sum[i];
    const float inv = s.w > 0.f ? 1.f / s.w : 0.f;
    out[i] = make_float4(s.x * inv, s.y * inv, s.z * inv, s.w);
}

RE_API re_status re_renderer_read_view(re_renderer* r, uint32_t plane, uint32_t path_offset, uint32_t pixel_count,
                                       re_float4* out, uint32_t memory, void* stream) {
    if (r == nullptr || out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (uint64_t(path_offset) + pixel_count > r->capacity)
        return set_error(RE_INVALID_ARGUMENT, "read exceeds the path capacity");
    void* base = nullptr;
    re_status st = re_renderer_film_pointer(r, plane, &base);
    if (st != RE_SUCCESS) return st;
    RE_CUDA_TRY(cudaSetDevice(r->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t bytes = size_t(pixel_count) * sizeof(float4);
    const float4* src = static_cast<const float4*>(base) + path_offset;
    if (plane == RE_FILM_MEAN) {
        // The progressive mean is formed in the hit buffer (free between launches).
        float4* tmp = r->dev.hit + path_offset;
        k_film_mean<<<(pixel_count + 255) / 256, 256, 0, s>>>(src, tmp, pixel_count);
        RE_CUDA_TRY(cudaGetLastError());
        src = tmp;
    }
    RE_CUDA_TRY(cudaMemcpyAsync(out, src, bytes,
                                memory == RE_MEMORY_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s));
    if (memory == RE_MEMORY_HOST) RE_CUDA_TRY(cudaStreamSynchronize(s));
    return clear_error();
}

RE_API re_status re_renderer_read_film(re_renderer* r, uint32_t plane, re_float4* out, uint32_t pixel_count,
                                       uint32_t memory, void* stream) {
    return re_renderer_read_view(r, plane, 0u, pixel_count, out, memory, stream);
}

// Two frames in flight, as the reference keeps two frame slots
// (Wave2Runtime.hpp:24, CollectCompletedFrame after the slot fence): the
// plane is snapshotted on `stream` into one of two staging buffers (taken in
// turn; a snapshot first waits, on the device, for the host copy that last
// read its buffer), and the renderer's own stream copies the snapshot to
// `host_out` while the next frame queued on `stream` runs.
RE_API re_status re_renderer_read_view_async(re_renderer* r, uint32_t plane, uint32_t path_offset,
                                             uint32_t pixel_count, re_float4* host_out, void* stream) {
    if (r == nullptr || host_out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (pixel_count == 0) return set_error(RE_INVALID_ARGUMENT, "a read of zero pixels");
    if (uint64_t(path_offset) + pixel_count > r->capacity)
        return set_error(RE_INVALID_ARGUMENT, "read exceeds the path capacity");
    void* base = nullptr;
    re_status st = re_renderer_film_pointer(r, plane, &base);
    if (st != RE_SUCCESS) return st;
    RE_CUDA_TRY(cudaSetDevice(r->device));
    if (r->read_stream == nullptr) {
        RE_CUDA_TRY(cudaStreamCreateWithFlags(&r->read_stream, cudaStreamNonBlocking));
        for (int k = 0; k < 2; ++k) {
            RE_CUDA_TRY(cudaEventCreateWithFlags(&r->read_snap[k], cudaEventDisableTiming));
            RE_CUDA_TRY(cudaEventCreateWithFlags(&r->read_done[k], cudaEventDisableTiming));
        }
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint32_t k = r->read_next;
    const size_t bytes = size_t(pixel_count) * sizeof(float4);
    if (r->read_stage[k].bytes < bytes) {
        // Growing frees the old buffer: its last host copy must have landed.
        if (r->read_used[k]) RE_CUDA_TRY(cudaEventSynchronize(r->read_done[k]));
        RE_CUDA_TRY(r->read_stage[k].reserve(bytes));
    }
    const float4* src = static_cast<const float4*>(base) + path_offset;
    if (plane == RE_FILM_MEAN) {
        float4* tmp = r->dev.hit + path_offset;
        k_film_mean<<<(pixel_count + 255) / 256, 256, 0, s>>>(src, tmp, pixel_count);
        RE_CUDA_TRY(cudaGetLastError());
        src = tmp;
    }
    if (r->read_used[k]) RE_CUDA_TRY(cudaStreamWaitEvent(s, r->read_done[k], 0));
    RE_CUDA_TRY(cudaMemcpyAsync(r->read_stage[k].ptr, src, bytes, cudaMemcpyDeviceToDevice, s));
    RE_CUDA_TRY(cudaEventRecord(r->read_snap[k], s));
    RE_CUDA_TRY(cudaStreamWaitEvent(r->read_stream, r->read_snap[k], 0));
    RE_CUDA_TRY(cudaMemcpyAsync(host_out, r->read_stage[k].ptr, bytes, cudaMemcpyDeviceToHost, r->read_stream));
    RE_CUDA_TRY(cudaEventRecord(r->read_done[k], r->read_stream));
    r->read_used[k] = true;
    r->read_next = k ^ 1u;
    return clear_error();
}

RE_API re_status re_renderer_wait_reads(re_renderer* r) {
    if (r == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (r->read_stream != nullptr) {
        RE_CUDA_TRY(cudaSetDevice(r->device));
        RE_CUDA_TRY(cudaStreamSynchronize(r->read_stream));
    }
    return clear_error();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Reconstruction inputs: G-buffer and signal records of one view for SVGF.
// ---------------------------------------------------------------------------
namespace re {
namespace {

// Camera matrices of a pinhole frame in the reconstruction module's
// conventions (reconstruction/include/reconstruction/Math.hpp:110-129,
// MotionVectors.hpp:7-18): row-major, column vectors, right-handed view
// space looking down -Z.  The view-projection's clip w is the view depth and
// its NDC is the renderer's image plane (x right, y up: uv = ndc * 0.5 + 0.5
// with v flipped, the pixel a camera ray of RayGen starts from); its z row
// is unused by the reprojection and left zero.
void camera_matrices(const re_frame_constants& f, float vp[16], float w2v[16]) {
    const float px = f.camera_position_tan_half_fov.x, py = f.camera_position_tan_half_fov.y,
                pz = f.camera_position_tan_half_fov.z, tan_half = f.camera_position_tan_half_fov.w;
    const float fx = f.camera_forward_aspect.x, fy = f.camera_forward_aspect.y, fz = f.camera_forward_aspect.z,
                aspect = f.camera_forward_aspect.w;
    const float rx = f.camera_right_lens_radius.x, ry = f.camera_right_lens_radius.y, rz = f.camera_right_lens_radius.z;
    const float ux = f.camera_up_exposure.x, uy = f.camera_up_exposure.y, uz = f.camera_up_exposure.z;
    const float rt = -(rx * px + ry * py + rz * pz);
    const float ut = -(ux * px + uy * py + uz * pz);
    const float ft = fx * px + fy * py + fz * pz;
    const float w[16] = {rx, ry, rz, rt, ux, uy, uz, ut, -fx, -fy, -fz, ft, 0.f, 0.f, 0.f, 1.f};
    std::memcpy(w2v, w, sizeof(w));
    const float sx = 1.0f / (tan_half * aspect), sy = 1.0f / tan_half;
    const float m[16] = {rx * sx, ry * sx, rz * sx, rt * sx, ux * sy, uy * sy, uz * sy, ut * sy,
                         0.f,     0.f,     0.f,     0.f,     fx,      fy,      fz,      -ft};
    std::memcpy(vp, m, sizeof(m));
}

struct ExportArgs {
    uint32_t offset, width, height, slot;
    uint32_t has_prev, pad0, pad1, pad2;
    float cur_vp[16], prev_vp[16], prev_w2v[16];
};

// Transform (Math.hpp:122-129) in its operation order.
__device__ __forceinline__ float4 xform(const float* m, float4 v) {
    return make_float4(m[0] * v.x + m[1] * v.y + m[2] * v.z + m[3] * v.w,
                       m[4] * v.x + m[5] * v.y + m[6] * v.z + m[7] * v.w,
                       m[8] * v.x + m[9] * v.y + m[10] * v.z + m[11] * v.w,
                       m[12] * v.x + m[13] * v.y + m[14] * v.z + m[15] * v.w);
}

__device__ __forceinline__ bool finite4(float4 v) {
    return isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && isfinite(v.w);
}

// ProjectToUv (MotionVectors.cpp:14-33) with identity object transforms and
// zero jitter.
__device__ __forceinline__ bool project_uv(const float* vp, float4 world, float& u, float& v) {
    const float4 clip = xform(vp, world);
    if (!finite4(world) || !finite4(clip) || clip.w <= 1.0e-8f) return false;
    const float rw = 1.0f / clip.w;
    const float nx = clip.x * rw, ny = clip.y * rw;
    u = nx * 0.5f + 0.5f + 0.0f;
    v = 0.5f - ny * 0.5f + 0.0f;
    return isfinite(u) && isfinite(v);
}

// Per pixel of the view: the primary hit as a GBufferPixel (linear depth,
// shading normal, albedos from the hit material, IDs, motion to the previous
// camera as ComputeMotionVector, MotionVectors.cpp:37-74, computes it) and
// that frame's radiance as a SignalPixel.  Albedos: Lambert -> diffuse base
// color; metallic-roughness -> diffuse base * (1 - metallic) * (1 -
// transmission), specular f0 * (1 - metallic) + base * metallic; conductor
// -> specular base color; dielectric reflection -> specular f0; glass ->
// specular one.  Signal: diffuse = camera-visible emission + direct +
// indirect diffuse, specular = direct + indirect specular.
__global__ void k_export_reconstruction(WfDevice d, ExportArgs a, re_gbuffer_pixel* gb, re_signal_pixel* sig) {
    const uint32_t n = a.width * a.height;
    const SceneSlot& sc = d.scenes[a.slot];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t p = a.offset + i;
        const uint4 id = d.gb_id[p];
        const float4 pos = d.gb_pos[p];
        const float4 nrm = d.gb_nrm[p];
        re_gbuffer_pixel g;
        g.linear_depth = 0.f;
        g.world_normal[0] = g.world_normal[1] = g.world_normal[2] = 0.f;
        g.diffuse_albedo[0] = g.diffuse_albedo[1] = g.diffuse_albedo[2] = 0.f;
        g.specular_albedo[0] = g.specular_albedo[1] = g.specular_albedo[2] = 0.f;
        g.expected_previous_linear_depth = 0.f;
        g.motion[0] = g.motion[1] = 0.f;
        g.material_id = kInv;
        g.object_id = kInv;
        g.flags = 0u;
        const f3 ns = from4(nrm);
        const bool hit = id.x != kInv && id.z < sc.material_count;
        if (hit && isfinite(pos.w) && pos.w >= 0.f && finite3(ns) && dot(ns, ns) > 0.f) {
            const Material m = load_material(sc, id.z);
            const f3 base = from4(m.base_metal), f0 = from4(m.f0);
            const float metal = m.base_metal.w, trans = m.trans_ior.x;
            f3 dif = f3s(0.f), spec = f3s(0.f);
            switch (m.meta.x) {
                case kModelLambert: dif = base; break;
                case kModelMetallicRoughness:
                    dif = base * ((1.f - metal) * (1.f - trans));
                    spec = f0 * (1.f - metal) + base * metal;
                    break;
                case kModelGgxConductor: spec = base; break;
                case kModelGgxDielectricReflection: spec = f0; break;
                default: spec = f3s(1.f); break;
            }
            g.linear_depth = pos.w;
            g.world_normal[0] = ns.x; g.world_normal[1] = ns.y; g.world_normal[2] = ns.z;
            g.diffuse_albedo[0] = dif.x; g.diffuse_albedo[1] = dif.y; g.diffuse_albedo[2] = dif.z;
            g.specular_albedo[0] = spec.x; g.specular_albedo[1] = spec.y; g.specular_albedo[2] = spec.z;
            g.material_id = id.z;
            g.object_id = id.x;
            g.flags = RE_GBUFFER_VALID;
            if (a.has_prev != 0u) {
                const float4 world = make_float4(pos.x, pos.y, pos.z, 1.f);
                float cu = 0.f, cv = 0.f, pu = 0.f, pv = 0.f;
                const bool cur_ok = project_uv(a.cur_vp, world, cu, cv);
                const bool prev_ok = project_uv(a.prev_vp, world, pu, pv);
                const float4 view = xform(a.prev_w2v, world);
                const float prev_depth = -view.z;
                const bool depth_ok = finite4(world) && finite4(view) && isfinite(prev_depth) && prev_depth >= 0.f;
                if (cur_ok && prev_ok && depth_ok) {
                    g.motion[0] = pu - cu;
                    g.motion[1] = pv - cv;
                    g.expected_previous_linear_depth = prev_depth;
                    g.flags |= RE_GBUFFER_MOTION_VALID;
                }
            }
        }
        const f3 dfs = from4(d.acc_cam[p]) + from4(d.acc_dd[p]) + from4(d.acc_id[p]);
        const f3 sps = from4(d.acc_ds[p]) + from4(d.acc_is[p]);
        re_signal_pixel s;
        s.diffuse[0] = dfs.x; s.diffuse[1] = dfs.y; s.diffuse[2] = dfs.z;
        s.specular[0] = sps.x; s.specular[1] = sps.y; s.specular[2] = sps.z;
        gb[i] = g;
        sig[i] = s;
    }
}

}  // namespace
}  // namespace re

extern "C" {

RE_API re_status re_camera_matrices(const re_frame_constants* frame, float view_projection[16],
                                    float world_to_view[16]) {
    if (frame == nullptr || view_projection == nullptr || world_to_view == nullptr)
        return set_error(RE_INVALID_ARGUMENT, "null argument");
    camera_matrices(*frame, view_projection, world_to_view);
    return clear_error();
}

RE_API re_status re_renderer_export_reconstruction(re_renderer* r, uint32_t scene_slot, uint32_t path_offset,
                                                   const re_frame_constants* current,
                                                   const re_frame_constants* previous, re_gbuffer_pixel* gbuffer,
                                                   re_signal_pixel* signal, uint32_t memory, void* stream) {
    if (r == nullptr || current == nullptr || gbuffer == nullptr || signal == nullptr)
        return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (scene_slot >= kMaxSceneSlots || r->slots[scene_slot].scene == nullptr)
        return set_error(RE_MISSING_SCENE, "scene slot is not bound");
    if (memory != RE_MEMORY_HOST && memory != RE_MEMORY_DEVICE)
        return set_error(RE_INVALID_ARGUMENT, "unknown memory kind");
    const uint64_t n = uint64_t(current->image.x) * current->image.y;
    if (n == 0 || uint64_t(path_offset) + n > r->capacity)
        return set_error(RE_INVALID_ARGUMENT, "view exceeds the path capacity");
    ExportArgs a{};
    a.offset = path_offset;
    a.width = current->image.x;
    a.height = current->image.y;
    a.slot = scene_slot;
    float unused[16];
    camera_matrices(*current, a.cur_vp, unused);
    if (previous != nullptr) {
        a.has_prev = 1u;
        camera_matrices(*previous, a.prev_vp, a.prev_w2v);
    }
    RE_CUDA_TRY(cudaSetDevice(r->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    re_gbuffer_pixel* dg = gbuffer;
    re_signal_pixel* ds = signal;
    const size_t gb_bytes = size_t(n) * sizeof(re_gbuffer_pixel), sig_bytes = size_t(n) * sizeof(re_signal_pixel);
    if (memory == RE_MEMORY_HOST) {
        RE_CUDA_TRY(r->export_stage.reserve(gb_bytes + sig_bytes + 256));
        dg = static_cast<re_gbuffer_pixel*>(r->export_stage.ptr);
        ds = reinterpret_cast<re_signal_pixel*>(static_cast<char*>(r->export_stage.ptr) + ((gb_bytes + 255) / 256) * 256);
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, r->device);
    const uint32_t blocks = uint32_t(std::min<uint64_t>((n + 255) / 256, uint64_t(sms) * 8u));
    k_export_reconstruction<<<blocks, 256, 0, s>>>(r->dev, a, dg, ds);
    RE_CUDA_TRY(cudaGetLastError());
    if (memory == RE_MEMORY_HOST) {
        RE_CUDA_TRY(cudaMemcpyAsync(gbuffer, dg, gb_bytes, cudaMemcpyDeviceToHost, s));
        RE_CUDA_TRY(cudaMemcpyAsync(signal, ds, sig_bytes, cudaMemcpyDeviceToHost, s));
        RE_CUDA_TRY(cudaStreamSynchronize(s));
    }
    return clear_error();
}

}  // extern "C"

namespace re {

re_status renderer_copy_mean_async(re_renderer* r, uint32_t offset, uint32_t n, void* host_dst, cudaStream_t s) {
    if (r == nullptr || host_dst == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (uint64_t(offset) + n > r->capacity) return set_error(RE_INVALID_ARGUMENT, "read exceeds the path capacity");
    float4* tmp = r->dev.hit + offset;  // free between launches; later launches are stream-ordered after the copy
    k_film_mean<<<(n + 255) / 256, 256, 0, s>>>(r->dev.film_sum + offset, tmp, n);
    RE_CUDA_TRY(cudaGetLastError());
    RE_CUDA_TRY(cudaMemcpyAsync(host_dst, tmp, size_t(n) * sizeof(float4), cudaMemcpyDeviceToHost, s));
    return RE_SUCCESS;
}

re_status renderer_reserve_restir(re_renderer* r) { return ensure_restir_buffers(r); }

uint64_t renderer_device_bytes(const re_renderer* r) {
    uint64_t b = r->arena.bytes + r->restir_arena.bytes + r->path_view.bytes + r->counters.bytes + r->frame.bytes +
                 r->scenes_table.bytes;
    for (const SlotState& s : r->slots)
        b += s.materials.bytes + s.lights.bytes + s.alias.bytes + s.pmf.bytes + s.fixtures.bytes + s.emitter.bytes;
    return b;
}

re_status renderer_ray_totals(re_renderer* r, uint64_t* path_rays, uint64_t* shadow_rays) {
    uint32_t words[8] = {};
    RE_CUDA_TRY(cudaSetDevice(r->device));
    RE_CUDA_TRY(cudaMemcpy(words, r->film_frames.ptr, 32, cudaMemcpyDeviceToHost));
    std::memcpy(path_rays, words + 2, 8);
    std::memcpy(shadow_rays, words + 4, 8);
    return RE_SUCCESS;
}

}  // namespace re

extern "C" {

RE_API re_status re_restir_default_config(re_restir_config* out) {
    if (out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    // RuntimeConfig RestirSettings (RuntimeConfig.hpp:181-192) and the
    // ReSTIRFrameParameterSources validation defaults (ReSTIRFrameParameters.hpp:19-20).
    *out = re_restir_config{8u, 5u, 32u, 20u, 1u, 0u, 30.f, 0.8f, 0.05f, 0.02f, 0u};
    return clear_error();
}

RE_API re_status re_renderer_set_restir(re_renderer* r, const re_restir_config* c) {
    if (r == nullptr || c == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (c->candidates > 1024u || c->spatial_neighbors > 30u || c->max_m == 0u || c->neighbor_mode > 1u ||
        c->temporal > 1u || !std::isfinite(c->disk_radius) || c->disk_radius < 1.f || c->disk_radius > 256.f ||
        !std::isfinite(c->normal_cos) || c->normal_cos < -1.f || c->normal_cos > 1.f ||
        !std::isfinite(c->relative_depth) || c->relative_depth < 0.f || !std::isfinite(c->position_distance) ||
        c->position_distance < 0.f || c->estimator > 1u)
        return set_error(RE_INVALID_ARGUMENT, "ReSTIR configuration is out of range");
    r->restir = *c;
    ++r->camera_epoch;  // a new configuration starts a new history epoch
    return clear_error();
}

RE_API re_status re_renderer_restir_reset(re_renderer* r) {
    if (r == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    ++r->camera_epoch;
    return clear_error();
}

RE_API re_status re_renderer_restir_statistics(re_renderer* r, re_restir_statistics* out) {
    if (r == nullptr || out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    RE_CUDA_TRY(cudaSetDevice(r->device));
    if (r->frame_pending) RE_CUDA_TRY(cudaEventSynchronize(r->ev1));
    uint32_t v[12];
    std::memcpy(v, r->host_counters + kSlotRestirBase, sizeof(v));
    *out = re_restir_statistics{v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8], v[9], v[10], v[11]};
    return clear_error();
}

RE_API re_status re_renderer_restir_pointer(re_renderer* r, uint32_t plane, void** out) {
    if (r == nullptr || out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (r->restir_arena.ptr == nullptr) return set_error(RE_NOT_READY, "no RestirPrimary frame has been rendered");
    const WfDevice& d = r->dev;
    const auto it = r->rs_views.find(0u);
    const uint32_t parity = it != r->rs_views.end() ? it->second.parity : 0u;
    switch (plane) {
        case RE_RESTIR_PUBLISHED: *out = d.rs_published[parity]; break;
        case RE_RESTIR_TEMPORAL: *out = d.rs_temporal; break;
        case RE_RESTIR_SURFACES: *out = d.prim[parity]; break;
        case RE_RESTIR_DIRECT: *out = d.rs_direct; break;
        case RE_RESTIR_REASONS: *out = d.rs_reasons; break;
        default: return set_error(RE_INVALID_ARGUMENT, "unknown ReSTIR plane");
    }
    return clear_error();
}

RE_API re_status re_renderer_restir_debug(re_renderer* r, uint32_t mode, uint32_t pixel_count, void* records_out,
                                          re_float4* image_out, uint32_t memory, void* stream) {
    void* pub = nullptr;
    const re_status st = re_renderer_restir_pointer(r, RE_RESTIR_PUBLISHED, &pub);
    if (st != RE_SUCCESS) return st;
    if (pixel_count == 0u || pixel_count > r->capacity)
        return set_error(RE_INVALID_ARGUMENT, "debug pixel count must be 1 to the path capacity");
    if (records_out == nullptr && image_out == nullptr) return set_error(RE_INVALID_ARGUMENT, "no debug output");
    if (memory != RE_MEMORY_HOST && memory != RE_MEMORY_DEVICE)
        return set_error(RE_INVALID_ARGUMENT, "memory kind is invalid");
    RE_CUDA_TRY(cudaSetDevice(r->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t rec_bytes = size_t(pixel_count) * 64u, img_bytes = size_t(pixel_count) * sizeof(float4);
    void* rec = records_out;
    void* img = image_out;
    if (memory == RE_MEMORY_HOST) {
        RE_CUDA_TRY(r->export_stage.reserve(rec_bytes + img_bytes));
        rec = records_out != nullptr ? r->export_stage.ptr : nullptr;
        img = image_out != nullptr ? static_cast<char*>(r->export_stage.ptr) + rec_bytes : nullptr;
    }
    launch_restir_debug(pub, pixel_count, mode, r->restir.max_m, r->restir.max_history_age, rec, img, s);
    RE_CUDA_TRY(cudaGetLastError());
    if (memory == RE_MEMORY_HOST) {
        if (records_out != nullptr) RE_CUDA_TRY(cudaMemcpyAsync(records_out, rec, rec_bytes, cudaMemcpyDeviceToHost, s));
        if (image_out != nullptr) RE_CUDA_TRY(cudaMemcpyAsync(image_out, img, img_bytes, cudaMemcpyDeviceToHost, s));
        RE_CUDA_TRY(cudaStreamSynchronize(s));
    }
    return clear_error();
}

RE_API re_status re_renderer_restir_read(re_renderer* r, uint32_t plane, void* dst, uint64_t bytes, uint32_t memory,
                                         void* stream) {
    void* src = nullptr;
    const re_status st = re_renderer_restir_pointer(r, plane, &src);
    if (st != RE_SUCCESS) return st;
    if (dst == nullptr) return set_error(RE_INVALID_ARGUMENT, "null destination");
    const size_t per = plane == RE_RESTIR_SURFACES ? 96u : plane == RE_RESTIR_DIRECT ? 32u
                     : plane == RE_RESTIR_REASONS ? 4u : 256u;
    if (bytes > size_t(r->capacity) * per) return set_error(RE_INVALID_ARGUMENT, "read exceeds the plane");
    RE_CUDA_TRY(cudaSetDevice(r->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const cudaMemcpyKind kind = memory == RE_MEMORY_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (plane == RE_RESTIR_DIRECT) {
        // Diffuse records of the frame's paths, then the specular ones (the
        // specular plane starts `capacity` records after the diffuse one).
        const size_t half = bytes / 2;
        RE_CUDA_TRY(cudaMemcpyAsync(dst, src, half, kind, s));
        RE_CUDA_TRY(cudaMemcpyAsync(static_cast<char*>(dst) + half,
                                    static_cast<const char*>(src) + size_t(r->capacity) * 16u, half, kind, s));
    } else {
        RE_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, kind, s));
    }
    if (memory == RE_MEMORY_HOST) RE_CUDA_TRY(cudaStreamSynchronize(s));
    return clear_error();
}

RE_API re_status re_renderer_profile(re_renderer* r, const re_frame_constants* f, re_stage_profile* out) {
    if (r == nullptr || f == nullptr || out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    std::memset(out, 0, sizeof(*out));
    RE_CUDA_TRY(cudaSetDevice(r->device));
    RE_CUDA_TRY(cudaDeviceSynchronize());  // frames in flight share the path state
    cudaStream_t s = nullptr;
    RE_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    const uint32_t depth = f->image.w;
    DeviceBuffer cnt;
    std::vector<cudaEvent_t> ev(3 * kMaxDepth + 4, nullptr);
    re_status st = RE_SUCCESS;
    auto fail = [&](cudaError_t e, const char* what) {
        st = set_error(RE_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
    };
    do {
        // Pass 1: counting traversal kernels.
        st = single_view(r, f, 1u, 1u, s);
        if (st != RE_SUCCESS) break;
        // Three counters (node tests, triangle tests, node bytes) per bounce,
        // Intersect then TraceShadow.
        constexpr size_t kCnt = 6 * kMaxDepth;
        cudaError_t e = cnt.reserve(kCnt * sizeof(unsigned long long));
        if (e != cudaSuccess) { fail(e, "counter allocation"); break; }
        cudaMemsetAsync(cnt.ptr, 0, kCnt * sizeof(unsigned long long), s);
        FrameHooks hk;
        hk.cnt = static_cast<unsigned long long*>(cnt.ptr);
        e = record_frame(r, depth, s, hk);
        if (e != cudaSuccess) { fail(e, "counted frame"); break; }
        unsigned long long c[kCnt];
        uint32_t q[kCounterWords];
        cudaMemcpyAsync(c, cnt.ptr, sizeof(c), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(q, r->counters.ptr, sizeof(q), cudaMemcpyDeviceToHost, s);
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { fail(e, "counted frame"); break; }
        for (uint32_t b = 0; b < depth; ++b) {
            out->intersect_node_tests[b] = c[b * 3];
            out->intersect_triangle_tests[b] = c[b * 3 + 1];
            out->intersect_node_bytes[b] = c[b * 3 + 2];
            out->shadow_node_tests[b] = c[3 * kMaxDepth + b * 3];
            out->shadow_triangle_tests[b] = c[3 * kMaxDepth + b * 3 + 1];
            out->shadow_node_bytes[b] = c[3 * kMaxDepth + b * 3 + 2];
            out->rays[b] = std::min(q[b * kSlotsPerBounce + kSlotRays], r->capacity);
            out->shadows[b] = std::min(q[b * kSlotsPerBounce + kSlotShadows], r->capacity);
        }
        // Pass 2: events between the split stage launches.
        st = single_view(r, f, 1u, 1u, s);
        if (st != RE_SUCCESS) break;
        for (auto& x : ev) cudaEventCreate(&x);
        FrameHooks th;
        th.ev = ev.data();
        e = record_frame(r, depth, s, th);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { fail(e, "timed frame"); break; }
        cudaEventElapsedTime(&out->raygen_ms, ev[0], ev[1]);
        for (uint32_t b = 0; b < depth; ++b) {
            cudaEventElapsedTime(&out->intersect_ms[b], ev[1 + 3 * b], ev[2 + 3 * b]);
            cudaEventElapsedTime(&out->shade_ms[b], ev[2 + 3 * b], ev[3 + 3 * b]);
            cudaEventElapsedTime(&out->shadow_ms[b], ev[3 + 3 * b], ev[4 + 3 * b]);
        }
        if (r->restir_active) {
            cudaEventElapsedTime(&out->restir_ms, ev[1 + 3 * depth], ev[2 + 3 * depth]);
            cudaEventElapsedTime(&out->resolve_ms, ev[2 + 3 * depth], ev[3 + 3 * depth]);
        } else {
            cudaEventElapsedTime(&out->resolve_ms, ev[1 + 3 * depth], ev[2 + 3 * depth]);
        }
    } while (false);
    for (auto& x : ev)
        if (x) cudaEventDestroy(x);
    cudaStreamDestroy(s);
    return st == RE_SUCCESS ? clear_error() : st;
}

}  // extern "C"
