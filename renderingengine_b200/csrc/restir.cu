// ReSTIR DI passes of the wavefront frame (estimator RestirPrimary), after
// the bounce loop and before Resolve.  The reference runs seven compute
// passes with a materialised candidate buffer (pixels x candidates x 160 B)
// and reservoir round trips between them
// (resources/shaders/integrators/pbr_restir_candidate_export_v3.hlsl,
//  resources/shaders/restir/Restir{InitialV3,TemporalV3,SpatialV3,
//  WinnerVisibilityPrepareV3,WinnerResolveV3,PublishDirectV3,
//  PublishHistoryV3}.comp.hlsl).  Here they are four kernels:
//   k_restir_initial   candidate generation streamed into the initial RIS
//                      reservoir (no candidate buffer)
//   k_restir_reuse     temporal reuse of the previous frame's published
//                      reservoir (split from the candidate loop only so that
//                      loop's kernel runs at 80 registers, 6 CTAs per SM: the
//                      reuse pass holds two reservoirs and two surfaces)
//   k_restir_spatial   spatial reuse over the neighbours' temporal
//                      reservoirs (+ the reference-correction re-weighting)
//   k_restir_visibility the winner's shadow ray (any-hit traversal) + resolve
//                      + direct-light publish into the path's film
//                      accumulators + history publish; apart from the merge
//                      so the traversal runs at 64 registers
// Every random stream is the shader's (RestirHashV3 seeds, Philox light
// dimensions), so the result is the reference pipeline's, pass for pass.
#include "wavefront.cuh"

namespace re {
namespace {

constexpr uint32_t kStreamTagRestir = 0x52335354u;  // pbr_restir_candidate_export_v3.hlsl:17

__device__ __forceinline__ void rs_count(const WfDevice& d, uint32_t k, bool flag) {
    const uint32_t mask = __ballot_sync(0xffffffffu, flag);
    if ((threadIdx.x & 31) == 0 && mask != 0u) atomicAdd(d.counters + kSlotRestirBase + k, uint32_t(__popc(mask)));
}

__device__ __forceinline__ void store_reservoir(Reservoir* base, uint32_t p, const Reservoir& r) {
    float4* q = reinterpret_cast<float4*>(base + p);
    const float4* s = reinterpret_cast<const float4*>(&r);
#pragma unroll
    for (int k = 0; k < 16; ++k) q[k] = s[k];
}
__device__ __forceinline__ Reservoir load_reservoir(const Reservoir* base, uint32_t p) {
    Reservoir r;
    const float4* q = reinterpret_cast<const float4*>(base + p);
    float4* s = reinterpret_cast<float4*>(&r);
#pragma unroll
    for (int k = 0; k < 16; ++k) s[k] = q[k];
    return r;
}

__device__ __forceinline__ uint32_t measure_to_abi(uint32_t m) {  // PbrPrivateLightMeasureToAbiV1L6
    return m == kMeasureLightDiscrete ? 1u : (m == kMeasureLightArea ? 3u : (m == kMeasureLightSolidAngle ? 2u : 0u));
}

// PbrToPersistentLightSampleV3 (pbr_restir_candidate_export_v3.hlsl:37-82).
__device__ __forceinline__ LightSampleV3 to_persistent(const LightView& lights, const RestirParams& rp,
                                                       const LightSample& ls, uint32_t flattened) {
    LightSampleV3 s;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const uint4 u = make_uint4(0u, 0u, 0u, 0u);
    s.pos_dist = z; s.dir_pdf = z; s.rad_pmf = z; s.cond = z;
    s.identity = u; s.generation = u; s.metadata = u; s.source = u;
    if ((ls.flags & kSampleValid) == 0u || ls.light >= lights.light_count) return s;
    const uint4 lid = __ldg(reinterpret_cast<const uint4*>(lights.lights + size_t(ls.light) * 6u + 4));
    s.pos_dist = to4(ls.position, ls.distance);
    s.dir_pdf = to4(ls.wi, ls.combined_pdf);
    s.rad_pmf = to4(ls.li, ls.selection_pmf);
    if (ls.measure == kMeasureLightArea) s.cond.x = ls.conditional_pdf;
    else if (ls.measure == kMeasureLightSolidAngle) s.cond.y = ls.conditional_pdf;
    s.identity = make_uint4(lid.z, ls.primitive, flattened, rp.frame_lo);
    s.generation = make_uint4(rp.light_gen, rp.scene_gen, rp.frame_lo, 0u);
    uint32_t flags = kRsSampleValid;
    if ((ls.flags & kSampleDelta) != 0u) flags |= kRsSampleDelta;
    if (ls.measure == kMeasureLightArea) flags |= kRsSampleArea;
    if (ls.measure == kMeasureLightSolidAngle) flags |= kRsSampleSolidAngle;
    s.metadata = make_uint4(measure_to_abi(ls.measure), flags, lid.y, ls.light);
    return s;
}

// Previous-frame UV and linear depth of a world point through the previous
// pinhole camera: the inverse of RayGen's pixel -> direction map, i.e. the
// motion vector of a static surface (MotionVectors.cpp:37-67).
__device__ __forceinline__ bool previous_uv(const RestirParams& rp, f3 p, float& u, float& v, float& depth) {
    if (rp.prev_valid == 0u) return false;
    const f3 dlt = p - rp.prev_pos;
    const float z = dot(dlt, rp.prev_fwd);
    if (!(z > 1.0e-8f) || !isfinite(z)) return false;
    const float sx = dot(dlt, rp.prev_right) / (z * rp.prev_aspect * rp.prev_tan);
    const float sy = dot(dlt, rp.prev_up) / (z * rp.prev_tan);
    u = sx * 0.5f + 0.5f;
    v = 0.5f - sy * 0.5f;
    depth = dot(dlt, normalize3(rp.prev_fwd));
    return isfinite(u) && isfinite(v) && isfinite(depth) && depth >= 0.f;
}

// Spatial neighbour k of pixel p.  Mode 0 is the reference's host-built table
// (Wave3DebugRuntime.cpp:1888-1922): 8-direction rings, clamped to the image.
// Mode 1 draws integer offsets uniformly from a disk of `disk_radius` pixels
// (hash-seeded by pixel, frame and k; integer arithmetic only).
__device__ __forceinline__ uint32_t neighbor_index(const RestirParams& rp, uint32_t w, uint32_t h, uint32_t p,
                                                   uint32_t k) {
    const int x = int(p % w), y = int(p / w);
    int dx = 0, dy = 0;
    const int ring = int(k / 8u) + 1;
    const int dirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, 1}, {1, -1}, {-1, -1}};
    dx = dirs[k % 8u][0] * ring;
    dy = dirs[k % 8u][1] * ring;
    if (rp.neighbor_mode == 1u) {
        const int r = max(1, int(rp.disk_radius));
        const uint32_t span = uint32_t(2 * r + 1);
        uint32_t st = restir_hash(p ^ restir_hash(rp.frame_lo + 0x68e31da4u * (k + 1u)));
        for (int attempt = 0; attempt < 8; ++attempt) {
            st = restir_hash(st + 0x9e3779b9u);
            const int ox = int(st % span) - r;
            const int oy = int((st >> 16) % span) - r;
            if ((ox != 0 || oy != 0) && ox * ox + oy * oy <= r * r) {
                dx = ox;
                dy = oy;
                break;
            }
        }
    }
    const int sx = min(max(x + dx, 0), int(w) - 1);
    const int sy = min(max(y + dy, 0), int(h) - 1);
    return uint32_t(sy) * w + uint32_t(sx);
}

}  // namespace

// Initial RIS over `candidates` streamed light samples
// (RestirInitialV3.comp.hlsl:9-58), the statistics it counts and the
// history stamps of this frame; the reservoir before temporal reuse.
__device__ __forceinline__ Reservoir initial_ris(const WfDevice& d, bool live, const FrameParams& fp,
                                                 const SceneSlot& sc, uint32_t pix, const PrimarySurface& s) {
    const RestirParams& rp = fp.rs;
    const uint32_t C = rp.candidates;
    Reservoir r = empty_reservoir();
    const bool sv = surface_valid(s);
    uint32_t n_valid = 0u;
    if (live && sv && C != 0u) {
        // An invalid surface makes every candidate invalid (correction 0),
        // leaving the reservoir empty: the loop only runs on valid surfaces.
        uint32_t rs = restir_hash(pix ^ rp.frame_lo ^ 0xa511e9b3u);
        const LightContext lc{xyz(s.pos_depth), xyz(s.gn_rough), xyz(s.sn_metal), fp.env_xf};
        const uint32_t stream = fp.stream ^ kStreamTagRestir;
        // Candidate c of this pixel's initial RIS stream (the same light
        // sample and evaluation whenever it is asked for).
        auto candidate = [&](uint32_t c) {
            const uint32_t sample = fp.sample * C + c;
            LightRandom lr;
            lr.selection = counter_random(pix, sample, kDimLightSelection, stream, fp.seed_lo, fp.seed_hi);
            lr.s0 = counter_random(pix, sample, kDimLightShape0, stream, fp.seed_lo, fp.seed_hi);
            lr.s1 = counter_random(pix, sample, kDimLightShape1, stream, fp.seed_lo, fp.seed_hi);
            lr.s2 = counter_random(pix, sample, kDimLightShape2, stream, fp.seed_lo, fp.seed_hi);
            lr.s3 = counter_random(pix, sample, kDimLightShape3, stream, fp.seed_lo, fp.seed_hi);
            const LightSample ls = sample_one_light<false>(sc.lights, lc, lr);
            LightSampleV3 ps = to_persistent(sc.lights, rp, ls, pix * C + c);
            ps.source = make_uint4(pix, s.identity.x, s.identity.y, s.identity.z);
            return evaluate_candidate(ps, s, fp.cam_pos, rp.scene_gen, rp.candidate_source, kReuseNone, pix);
        };
        // update_reservoir's fold over the stream, keeping the index of the
        // selected candidate instead of a copy of its 160 bytes: weight sum
        // and M evolve exactly as there (same additions in the same order,
        // same random number per candidate), and the selected candidate is
        // evaluated once more after the loop.  The loop then carries a few
        // scalars instead of the reservoir.
        float wsum = 0.f;
        uint32_t m = 0u, win = kRsInvalidIndex;
        for (uint32_t c = 0; c < C; ++c) {
            const Candidate cand = candidate(c);
            const bool valid = candidate_valid(cand, rp.scene_gen);
            if (valid) ++n_valid;
            if (fold_update(wsum, m, valid, candidate_weight(cand, rp.scene_gen), 1u, restir_random(rs))) win = c;
        }
        r.weight.x = wsum;
        r.state.x = m;
        if (win != kRsInvalidIndex) {
            const Candidate cand = candidate(win);
            select_candidate(r, cand, candidate_weight(cand, rp.scene_gen));
        }
    }
    clamp_m(r, rp.max_m);
    finalize_reservoir(r);
    rs_count(d, kRsStatMClamped, live && (r.state.z & kRsMClamped) != 0u);
    if (live) {
        atomicAdd(d.counters + kSlotRestirBase + kRsStatGenerated, C);
        if (n_valid) atomicAdd(d.counters + kSlotRestirBase + kRsStatValid, n_valid);
        if (C - n_valid) atomicAdd(d.counters + kSlotRestirBase + kRsStatRejected, C - n_valid);
    }
    r.state.y = 0u;
    r.h_surface = make_uint4(s.identity.x, s.identity.y, s.identity.z, 0u);
    r.h_scene = make_uint4(rp.scene_gen, rp.light_gen, rp.camera_gen, rp.resolution_gen);
    r.h_frame = make_uint4(rp.frame_lo, rp.frame_hi, rp.history_gen, kRsHistoryValid);
    r.h_reproj = make_uint4(pix, fp.width, fp.height, kRejNone);
    return r;
}

// PART 1: the initial RIS of one pixel, left in rs_temporal.  PART 2: the
// temporal reuse (RestirTemporalV3.comp.hlsl:20-215) of that reservoir,
// written back in place.
template <int PART>
__device__ __forceinline__ void restir_temporal_one(const WfDevice& d, uint32_t v, uint32_t p) {
    const bool live = v != kNoView && d.views[v].rs.enabled != 0u;
    const FrameParams& fp = d.views[live ? v : 0u];
    const RestirParams& rp = fp.rs;
    const SceneSlot& sc = d.scenes[fp.scene_slot];
    const uint32_t pp = live ? p : 0u;
    const uint32_t pix = pp - fp.path_offset;  // pixel within the view: RNG and reprojection coordinates
    const float4* surf_cur = d.prim[rp.parity];
    const float4* surf_prev = d.prim[rp.parity ^ 1u];
    const PrimarySurface s = load_surface(surf_cur, pp);
    if constexpr (PART == 1) {
        const Reservoir r = initial_ris(d, live, fp, sc, pix, s);
        if (live) store_reservoir(d.rs_temporal, p, r);
        return;
    }
    Reservoir r = live ? load_reservoir(d.rs_temporal, p) : empty_reservoir();

    // Temporal reuse.
    uint32_t rejection = kRejNone;
    bool accepted = false;
    if (rp.history_enabled != 0u && live) {
        float pu = 0.f, pv = 0.f, pdepth = 0.f;
        const bool hit_surface = s.pos_depth.w > 0.f;
        const bool motion_ok = hit_surface && previous_uv(rp, xyz(s.pos_depth), pu, pv, pdepth);
        uint32_t prior = kRsInvalidIndex;
        if (!motion_ok) {
            rejection = kRejMotionInvalid;
        } else if (pu < 0.f || pv < 0.f || pu >= 1.f || pv >= 1.f) {
            rejection = kRejReprojectionOutside;
        } else {
            const uint32_t px = min(uint32_t(pu * float(fp.width)), fp.width - 1u);
            const uint32_t py = min(uint32_t(pv * float(fp.height)), fp.height - 1u);
            prior = py * fp.width + px;
        }
        Reservoir hist = empty_reservoir();
        if (prior < fp.pixel_count) hist = load_reservoir(d.rs_published[rp.parity ^ 1u], fp.path_offset + prior);
        if (rejection == kRejNone &&
            ((hist.state.z & kRsValid) == 0u || hist.state.x == 0u || (hist.h_frame.w & kRsHistoryValid) == 0u))
            rejection = kRejInvalidCandidate;
        uint32_t exp_lo = rp.frame_lo, exp_hi = rp.frame_hi;
        if (exp_lo == 0u) {
            exp_lo = 0xffffffffu;
            exp_hi -= 1u;
        } else {
            exp_lo -= 1u;
        }
        if (rejection == kRejNone &&
            (hist.h_frame.x != exp_lo || hist.h_frame.y != exp_hi || hist.h_frame.z != rp.history_gen))
            rejection = kRejInvalidCandidate;
        else if (rejection == kRejNone && hist.h_scene.x != rp.scene_gen)
            rejection = kRejSceneGeneration;
        else if (rejection == kRejNone && hist.h_scene.y != rp.light_gen)
            rejection = kRejLightGeneration;
        else if (rejection == kRejNone && hist.h_scene.z != rp.camera_gen)
            rejection = kRejCameraCut;
        else if (rejection == kRejNone && hist.h_scene.w != rp.resolution_gen)
            rejection = kRejResize;
        else if (rejection == kRejNone && hist.state.y >= rp.max_age)
            rejection = kRejAge;
        else if (rejection == kRejNone && prior >= fp.pixel_count)
            rejection = kRejReprojectionOutside;
        else if (rejection == kRejNone)
            rejection = validate_surface_pair(s, load_surface(surf_prev, fp.path_offset + prior), rp);
        if (rejection == kRejNone) {
            const float hd = load_surface(surf_prev, fp.path_offset + prior).pos_depth.w;
            const float scale = fmaxf(1.f, fmaxf(fabsf(pdepth), fabsf(hd)));
            if (fabsf(pdepth - hd) / scale > rp.rel_depth) rejection = kRejDepth;
        }
        const uint32_t prev_light = hist.sel.metadata.w;
        if (rejection == kRejNone) {
            // The light table is the same across frames of one light-set
            // generation: the previous -> current map is the identity.
            if (prev_light >= rp.prev_light_count || prev_light >= rp.light_count ||
                rp.light_gen != hist.sel.generation.x)
                rejection = kRejLightGeneration;
        }
        if (rejection == kRejNone) {
            LightSampleV3 rm = hist.sel;
            if (rm.pos_dist.w < 1.0e29f) {
                const f3 delta = xyz(rm.pos_dist) - xyz(s.pos_depth);
                const float dist = length3(delta);
                if (isfinite(dist) && dist > 1.0e-6f) {
                    rm.pos_dist.w = dist;
                    const f3 dir = delta / dist;
                    rm.dir_pdf.x = dir.x;
                    rm.dir_pdf.y = dir.y;
                    rm.dir_pdf.z = dir.z;
                } else {
                    rm.metadata.y &= ~kRsSampleValid;
                }
            }
            rm.metadata.w = prev_light;
            Candidate cand =
                evaluate_candidate(rm, s, fp.cam_pos, rp.scene_gen, hist.prov.x, kReuseTemporal, prior);
            cand.t.w = hist.weight.y;
            const float mw = cand.t.x * cand.t.z * hist.weight.y * float(hist.state.x);
            uint32_t rs2 = restir_hash(pix ^ rp.frame_lo ^ 0x63d83595u);
            if (candidate_valid(cand, rp.scene_gen) && isfinite(mw) && mw >= 0.f) {
                update_reservoir(r, cand, mw, hist.state.x, restir_random(rs2), rp.scene_gen);
                r.state.z |= kRsTemporalAccepted;
                r.state.y = min(hist.state.y + 1u, rp.max_age);
                accepted = true;
            } else {
                rejection = kRejInvalidCandidate;
            }
        }
    }
    rs_count(d, kRsStatTemporalAttempts, live && rp.history_enabled != 0u);
    rs_count(d, kRsStatTemporalAccepted, accepted);
    clamp_m(r, rp.max_m);
    finalize_reservoir(r);
    r.state.w = rejection;
    r.h_reproj.w = rejection;
    if (live) {
        d.rs_reasons[p] = rejection;
        store_reservoir(d.rs_temporal, p, r);
    }
}

// Spatial reuse, winner visibility, resolve, direct publish and history
// publish (RestirSpatialV3 / WinnerVisibilityPrepareV3 / WinnerResolveV3 /
// PublishDirectV3 / PublishHistoryV3).
// WIDE: the winner's visibility ray walks the scene's four-wide nodes (as
// the launch's traversal stages do); visibility is the same either way.
// Binary (Physical) visibility of a reservoir's selected sample from a
// primary surface: the ray of RestirMakeVisibilityRayV3 (RestirProductionV3.
// hlsli:140-205) traced with the any-hit traversal; false for an invalid
// surface (the prepare pass emits no ray) or a blocked / invalid trace.
template <int STACK, bool WIDE>
__device__ __forceinline__ bool sample_visible(const SceneSlot& sc, const LightSampleV3& sel, const PrimarySurface& s,
                                               bool& traced) {
    traced = false;
    if (!surface_valid(s)) return false;
    const f3 normal = normalize3(xyz(s.gn_rough));
    f3 dir = normalize3(xyz(sel.dir_pdf));
    float max_dist = 1.0e30f;
    if (isfinite(sel.pos_dist.w) && sel.pos_dist.w > 0.f) {
        const f3 disp = xyz(sel.pos_dist) - xyz(s.pos_depth);
        const float dist = length3(disp);
        if (dist > 2.0e-4f) {
            dir = disp / dist;
            max_dist = fmaxf(dist - 1.0e-4f, 1.0e-4f);
        }
    }
    TraceRay ray{xyz(s.pos_depth) + normal * 1.0e-4f, dir, 1.0e-4f, max_dist};
    TraceOptions opt{0xffffffffu, 0xffffffffu, true};
    const TraceHit h = WIDE ? trace_wide<true, false, STACK>(sc.scene, ray, opt, nullptr)
                            : trace<true, false, STACK>(sc.scene, ray, opt, nullptr);
    traced = true;
    return h.status == 0u && h.tri == 0xffffffffu;
}

template <int STACK, bool WIDE>
__device__ __forceinline__ void restir_spatial_merge(const WfDevice& d, uint32_t v, uint32_t p) {
    const bool live = v != kNoView && d.views[v].rs.enabled != 0u;
    const FrameParams& fp = d.views[live ? v : 0u];
    const RestirParams& rp = fp.rs;
    const SceneSlot& sc = d.scenes[fp.scene_slot];
    const uint32_t pp = live ? p : 0u;
    const uint32_t pix = pp - fp.path_offset;
    const float4* surf_cur = d.prim[rp.parity];
    const PrimarySurface s = load_surface(surf_cur, pp);
    const Reservoir center = load_reservoir(d.rs_temporal, pp);
    Reservoir r;
    uint32_t n_attempt = 0u, n_accept = 0u;
    if (rp.neighbors == 0u) {
        r = center;
    } else {
        r = empty_reservoir();
        uint32_t rs = restir_hash(pix ^ rp.frame_lo ^ 0x9e3779b9u);
        uint32_t agg = live ? d.rs_reasons[p] : 0u;
        // The centre's and neighbour k's candidate against this pixel's
        // surface, with its multiple-importance weight: evaluated in the
        // merge and once more for the selected one after it (the merge keeps
        // the selected source's index, as initial_ris does).
        auto centre_candidate = [&](float& w) {
            Candidate cc =
                evaluate_candidate(center.sel, s, fp.cam_pos, rp.scene_gen, center.prov.x, center.prov.y, pix);
            cc.t.w = center.weight.y;
            w = cc.t.x * cc.t.z * center.weight.y * float(center.state.x);
            return cc;
        };
        auto neighbour_candidate = [&](const Reservoir& nb, uint32_t ni, float& w) {
            Candidate cand = evaluate_candidate(nb.sel, s, fp.cam_pos, rp.scene_gen, nb.prov.x, kReuseSpatial, ni);
            cand.t.w = nb.weight.y;
            w = cand.t.x * cand.t.z * nb.weight.y * float(nb.state.x);
            return cand;
        };
        float wsum = 0.f;
        uint32_t m = 0u, win = kRsInvalidIndex;  // 0: the centre, k + 1: neighbour k
        {
            float w;
            const Candidate cc = centre_candidate(w);
            if (fold_update(wsum, m, candidate_valid(cc, rp.scene_gen), w, center.state.x, restir_random(rs)))
                win = 0u;
        }
        uint32_t flags = center.state.z & (kRsMClamped | kRsTemporalAccepted);
        if (live) {
            for (uint32_t k = 0; k < rp.neighbors; ++k) {
                ++n_attempt;
                const uint32_t ni = neighbor_index(rp, fp.width, fp.height, pix, k);
                if (ni >= fp.pixel_count) {
                    agg = kRejReprojectionOutside;
                    continue;
                }
                const PrimarySurface ns = load_surface(surf_cur, fp.path_offset + ni);
                const uint32_t rej = validate_surface_pair(s, ns, rp);
                const Reservoir nb = load_reservoir(d.rs_temporal, fp.path_offset + ni);
                if (rej != kRejNone || (nb.state.z & kRsValid) == 0u) {
                    agg = rej != kRejNone ? rej : kRejInvalidCandidate;
                    continue;
                }
                float mw;
                const Candidate cand = neighbour_candidate(nb, ni, mw);
                if (candidate_valid(cand, rp.scene_gen) && isfinite(mw) && mw >= 0.f) {
                    if (fold_update(wsum, m, true, mw, nb.state.x, restir_random(rs))) win = k + 1u;
                    flags |= kRsSpatialAccepted;
                    ++n_accept;
                } else {
                    agg = kRejInvalidCandidate;
                }
            }
        }
        r.weight.x = wsum;
        r.state.x = m;
        r.state.z |= flags;
        if (win == 0u) {
            float w;
            select_candidate(r, centre_candidate(w), w);
        } else if (win != kRsInvalidIndex) {
            const uint32_t ni = neighbor_index(rp, fp.width, fp.height, pix, win - 1u);
            float w;
            const Candidate cand = neighbour_candidate(load_reservoir(d.rs_temporal, fp.path_offset + ni), ni, w);
            select_candidate(r, cand, w);
        }
        clamp_m(r, rp.max_m);
        finalize_reservoir(r);
        r.state.y = center.state.y;
        r.h_surface = center.h_surface;
        r.h_scene = center.h_scene;
        r.h_frame = center.h_frame;
        r.h_reproj = center.h_reproj;
        r.h_reproj.x = pix;
        r.h_reproj.w = agg;
        r.state.w = agg;
        if (live) d.rs_reasons[p] = agg;
    }
    if (n_attempt) atomicAdd(d.counters + kSlotRestirBase + kRsStatSpatialAttempts, n_attempt);
    if (n_accept) atomicAdd(d.counters + kSlotRestirBase + kRsStatSpatialAccepted, n_accept);

    // Reference correction (RestirReferenceVisibilityPrepareV3 +
    // RestirReferenceResolveV3): the selected sample re-evaluated with
    // visibility at the centre and at every neighbour it could have come
    // from; W = wsum * p(selected source) / (p(centre) * sum_i M_i p_i).
    if (live && rp.estimator == 1u && (r.state.z & kRsValid) != 0u) {
        float denom = 0.f, sel_target = 0.f, cur_target = 0.f;
        uint32_t n_submit = 0u, n_eval = 0u, n_vis = 0u;
        for (uint32_t k = 0; k <= rp.neighbors; ++k) {
            const uint32_t src = k == 0u ? pix : neighbor_index(rp, fp.width, fp.height, pix, k - 1u);
            if (src >= fp.pixel_count) continue;
            const PrimarySurface ss = load_surface(surf_cur, fp.path_offset + src);
            bool traced;
            const float vis = sample_visible<STACK, WIDE>(sc, r.sel, ss, traced) ? 1.f : 0.f;
            f3 dif, spec;
            const float target = evaluate_unshadowed(r.sel, ss, fp.cam_pos, rp.scene_gen, dif, spec);
            const uint32_t m_src = max(load_reservoir(d.rs_temporal, fp.path_offset + src).state.x, 1u);
            denom += float(m_src) * target * vis;
            if (src == pix) cur_target = target;
            if (src == r.prov.z) sel_target = target * vis;
            n_submit += traced ? 1u : 0u;
            ++n_eval;
            n_vis += vis > 0.f ? 1u : 0u;
        }
        const float nd = cur_target * denom;
        r.weight.y = nd > 0.f ? r.weight.x * sel_target / nd : 0.f;
        r.terms.w = r.weight.y;
        r.state.z |= kRsReferenceMode;
        if (!(r.weight.y > 0.f) || !isfinite(r.weight.y)) r.state.z &= ~kRsValid;
        atomicAdd(d.counters + kSlotRestirBase + kRsStatVisSubmitted, n_submit);
        atomicAdd(d.counters + kSlotRestirBase + kRsStatVisEvaluated, n_eval);
        if (n_vis) atomicAdd(d.counters + kSlotRestirBase + kRsStatVisVisible, n_vis);
    }

    if (live) store_reservoir(d.rs_published[rp.parity], p, r);
}

// Winner visibility, direct publish and history publish of the merged
// reservoir left in rs_published (written back in place).  Only the
// flags and the selected sample's position and direction are read before
// the shadow ray, the rest of the reservoir after it, so the traversal runs
// without the reservoir in registers.
template <int STACK, bool WIDE>
__device__ __forceinline__ void restir_visibility_one(const WfDevice& d, uint32_t v, uint32_t p) {
    const bool live = v != kNoView && d.views[v].rs.enabled != 0u;
    const FrameParams& fp = d.views[live ? v : 0u];
    const RestirParams& rp = fp.rs;
    const SceneSlot& sc = d.scenes[fp.scene_slot];
    const uint32_t pp = live ? p : 0u;
    const uint32_t pix = pp - fp.path_offset;
    const PrimarySurface s = load_surface(d.prim[rp.parity], pp);
    Reservoir* pub = d.rs_published[rp.parity];
    uint32_t flags = 0u;
    LightSampleV3 sel_ray;
    sel_ray.pos_dist = make_float4(0.f, 0.f, 0.f, 0.f);
    sel_ray.dir_pdf = make_float4(0.f, 0.f, 0.f, 0.f);
    if (live) {
        flags = pub[p].state.z;
        sel_ray.pos_dist = pub[p].sel.pos_dist;
        sel_ray.dir_pdf = pub[p].sel.dir_pdf;
    }

    // Winner visibility: one shadow ray per valid reservoir (Physical
    // shadows, RestirMakeVisibilityRayV3), traced here with the any-hit
    // traversal.
    const bool valid = live && (flags & kRsValid) != 0u;
    const bool duplicate = live && (flags & kRsFinalVisibility) != 0u;
    bool submitted = false, visible = false, evaluated = false;
    if (valid && !duplicate && surface_valid(s)) visible = sample_visible<STACK, WIDE>(sc, sel_ray, s, submitted);
    Reservoir r = live ? load_reservoir(pub, p) : empty_reservoir();
    if (valid && !duplicate) {
        // RestirResolveWinnerVisibilityV3 for the Physical mode: binary.
        const float vis = visible ? 1.f : 0.f;
        const float fw = r.weight.y * vis;
        const bool finite_result = isfinite(vis) && vis >= 0.f && vis <= 1.f && isfinite(fw) && fw >= 0.f;
        const bool vis_ok = finite_result && vis > 0.f;
        r.state.z |= kRsFinalVisibility;
        r.terms.w = finite_result ? fw : 0.f;
        if (!finite_result) {
            r.state.z &= ~kRsValid;
            r.state.w = kRejInvalidCandidate;
            r.h_reproj.w = kRejInvalidCandidate;
        }
        if (vis_ok) r.state.z |= kRsVisibilityValid;
        else r.state.z &= ~kRsVisibilityValid;
        evaluated = true;
        visible = vis_ok;
    }
    rs_count(d, kRsStatVisSubmitted, submitted);
    rs_count(d, kRsStatVisEvaluated, evaluated);
    rs_count(d, kRsStatVisVisible, evaluated && visible);
    rs_count(d, kRsStatVisDuplicate, duplicate);
    if (!live) return;

    // RestirPublishDirectV3: the primary direct term joins the path's
    // direct-lighting accumulators (Resolve adds them into the film).
    if ((r.state.z & kRsValid) != 0u && (r.state.z & kRsFinalVisibility) != 0u &&
        (r.state.z & kRsVisibilityValid) != 0u) {
        f3 dif, spec;
        evaluate_unshadowed(r.sel, s, fp.cam_pos, rp.scene_gen, dif, spec);
        dif = dif * r.terms.w;
        spec = spec * r.terms.w;
        d.rs_direct[p] = to4(dif, 0.f);
        d.rs_direct[d.capacity + p] = to4(spec, 0.f);
        const f3 a = from4(d.acc_dd[p]) + dif;
        const f3 b = from4(d.acc_ds[p]) + spec;
        if (finite_nonneg3(a) && finite_nonneg3(b)) {
            d.acc_dd[p] = to4(a, 0.f);
            d.acc_ds[p] = to4(b, 0.f);
        }
    } else {
        d.rs_direct[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        d.rs_direct[d.capacity + p] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    // RestirPublishHistoryV3.
    r.h_surface = make_uint4(s.identity.x, s.identity.y, s.identity.z, 0u);
    r.h_scene.x = rp.scene_gen;
    r.h_scene.y = rp.light_gen;
    const uint32_t hflags =
        (r.state.z & kRsValid) != 0u && (r.state.z & kRsFinalVisibility) != 0u ? kRsHistoryValid : kRsHistoryReset;
    r.h_frame = make_uint4(rp.frame_lo, rp.frame_hi, rp.history_gen, hflags);
    r.h_reproj = make_uint4(pix, fp.width, fp.height, r.h_reproj.w);
    store_reservoir(pub, p, r);
}

// Launch index c -> (view, path); kNoView past the batch's pixels.
__device__ __forceinline__ uint32_t launch_path(const WfDevice& d, uint32_t view_count, uint32_t total, uint32_t c,
                                                uint32_t& p) {
    p = 0u;
    if (c >= total) return kNoView;
    const uint32_t v = launch_view(d.views, view_count, c);
    p = d.views[v].path_offset + (c - d.views[v].pixel_base);
    return v;
}

// Grid-stride launches over the batch's pixels: every warp walks the same
// index blocks, so the warp-wide statistics ballots stay convergent, and the
// grid does not depend on the batch (one CUDA graph serves every batch).
// Four CTAs per SM (at most 128 registers): the candidate loop is ALU work
// whose fixed latencies need more warps than 156 registers leave.
// Six CTAs per SM for the candidate loop (80 registers, a few spills):
// measured against four (117 registers) and eight (64), and against one
// kernel for both passes (128 registers): 7.60 ms per many-light frame
// against 7.63, 7.64 and 7.81.
__global__ void __launch_bounds__(128, 6) k_restir_initial(WfDevice d) {
    const uint32_t total = d.batch->pixel_total, n = d.batch->view_count;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < total; base += stride) {
        uint32_t p;
        const uint32_t v = launch_path(d, n, total, base + threadIdx.x, p);
        restir_temporal_one<1>(d, v, p);
    }
}
__global__ void __launch_bounds__(128, 4) k_restir_reuse(WfDevice d) {
    const uint32_t total = d.batch->pixel_total, n = d.batch->view_count;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < total; base += stride) {
        uint32_t p;
        const uint32_t v = launch_path(d, n, total, base + threadIdx.x, p);
        restir_temporal_one<2>(d, v, p);
    }
}


// Four CTAs per SM (128 registers): six and eight measured slower (7.65 and
// 7.66 against 7.59 ms per many-light frame, same run).
template <int STACK, bool WIDE>
__global__ void __launch_bounds__(128, 4) k_restir_spatial(WfDevice d) {
    const uint32_t total = d.batch->pixel_total, n = d.batch->view_count;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < total; base += stride) {
        uint32_t p;
        const uint32_t v = launch_path(d, n, total, base + threadIdx.x, p);
        restir_spatial_merge<STACK, WIDE>(d, v, p);
    }
}
// Eight CTAs per SM (64 registers, the traversal kernels' budget, with a
// few spills): 7.52 ms per many-light frame against 7.56 at six and 7.71
// at four CTAs per SM, and 7.60 with the shadow ray inside the merge kernel.
template <int STACK, bool WIDE>
__global__ void __launch_bounds__(128, 8) k_restir_visibility(WfDevice d) {
    const uint32_t total = d.batch->pixel_total, n = d.batch->view_count;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < total; base += stride) {
        uint32_t p;
        const uint32_t v = launch_path(d, n, total, base + threadIdx.x, p);
        restir_visibility_one<STACK, WIDE>(d, v, p);
    }
}

// RestirDebugV3 (resources/shaders/restir/RestirDebugV3.comp.hlsl): per
// pixel of the published reservoirs, the raw debug record (identity,
// generation, weight sum / W / target / final weight with non-finite values
// as 0, state) and a float4 view selected by `mode` -- 0: M and age over the
// M cap and the age cap, M-clamped flag; 1: the weights as w / (1 + w);
// 2: light and primitive IDs and the sample generation, 3: provenance and
// source, 4: reuse source and the temporal / spatial accepted flags, 5:
// rejection reason, reprojected pixel and source surface, each as the
// fractional part of a golden-ratio multiple; 6 and above: final visibility,
// visibility evaluated, visibility valid.  The alpha channel flags whether
// every float of the reservoir is finite (mode 1 keeps the final weight).
__device__ __forceinline__ float finite_or_zero(float v) { return isfinite(v) ? v : 0.f; }
__device__ __forceinline__ bool finite4(float4 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && isfinite(v.w); }
__device__ __forceinline__ float frac_golden(float v, float m) {
    const float x = fmaxf(v, 0.f) * m;
    return x - floorf(x);
}

__global__ void k_restir_debug(const Reservoir* pub, uint32_t n, uint32_t mode, uint32_t max_m, uint32_t max_age,
                               uint4* records, float4* image) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Reservoir r = pub[i];
    if (records != nullptr) {
        uint4* o = records + size_t(i) * 4u;
        o[0] = make_uint4(r.sel.identity.x, r.sel.identity.y, r.prov.x, r.prov.y);
        o[1] = r.sel.generation;
        o[2] = make_uint4(__float_as_uint(finite_or_zero(r.weight.x)), __float_as_uint(finite_or_zero(r.weight.y)),
                          __float_as_uint(finite_or_zero(r.weight.z)), __float_as_uint(finite_or_zero(r.terms.w)));
        o[3] = r.state;
    }
    if (image == nullptr) return;
    const bool finite = finite4(r.weight) && finite4(r.terms) && finite4(r.sel.pos_dist) && finite4(r.sel.dir_pdf) &&
                        finite4(r.sel.rad_pmf) && finite4(r.sel.cond);
    const float a = finite ? 1.f : 0.f;
    float4 v;
    if (mode == 0u) {
        v = make_float4(float(r.state.x), float(r.state.y), (r.state.z & kRsMClamped) != 0u ? 1.f : 0.f, a);
        v.x = v.x / float(max(max_m, 1u));
        v.y = v.y / float(max(max_age, 1u));
    } else if (mode == 1u) {
        v = make_float4(finite_or_zero(r.weight.x), finite_or_zero(r.weight.y), finite_or_zero(r.weight.z),
                        finite_or_zero(r.terms.w));
        const float x = fmaxf(v.x, 0.f), y = fmaxf(v.y, 0.f), z = fmaxf(v.z, 0.f);
        v.x = x / (1.f + x);
        v.y = y / (1.f + y);
        v.z = z / (1.f + z);
    } else if (mode <= 5u) {
        float x, y, z;
        if (mode == 2u) {
            x = float(r.sel.identity.x); y = float(r.sel.identity.y); z = float(r.sel.generation.x);
        } else if (mode == 3u) {
            x = float(r.prov.x); y = float(r.prov.z); z = float(r.sel.source.x);
        } else if (mode == 4u) {
            x = float(r.prov.y);
            y = (r.state.z & kRsTemporalAccepted) != 0u ? 1.f : 0.f;
            z = (r.state.z & kRsSpatialAccepted) != 0u ? 1.f : 0.f;
        } else {
            x = float(r.state.w); y = float(r.h_reproj.x); z = float(r.prov.z);
        }
        v = make_float4(frac_golden(x, 0.6180339f), frac_golden(y, 0.381966f), frac_golden(z, 0.7548777f), a);
    } else {
        float vis = 0.f;
        if ((r.state.z & kRsFinalVisibility) != 0u && r.weight.y > 0.f && isfinite(r.weight.y) && isfinite(r.terms.w))
            vis = fminf(fmaxf(r.terms.w / r.weight.y, 0.f), 1.f);
        v = make_float4(vis, (r.state.z & kRsFinalVisibility) != 0u ? 1.f : 0.f,
                        (r.state.z & kRsVisibilityValid) != 0u ? 1.f : 0.f, a);
    }
    image[i] = v;
}

void launch_restir_debug(const void* published, uint32_t n, uint32_t mode, uint32_t max_m, uint32_t max_age,
                         void* records, void* image, cudaStream_t s) {
    k_restir_debug<<<(n + 255) / 256, 256, 0, s>>>(static_cast<const Reservoir*>(published), n, mode, max_m, max_age,
                                                   static_cast<uint4*>(records), static_cast<float4*>(image));
}

void launch_restir(const WfDevice& d, uint32_t blocks, bool deep_stack, bool wide, cudaStream_t s) {
    k_restir_initial<<<blocks, 128, 0, s>>>(d);
    k_restir_reuse<<<blocks, 128, 0, s>>>(d);
    if (wide) {
        if (deep_stack) {
            k_restir_spatial<128, true><<<blocks, 128, 0, s>>>(d);
            k_restir_visibility<128, true><<<blocks, 128, 0, s>>>(d);
        } else {
            k_restir_spatial<64, true><<<blocks, 128, 0, s>>>(d);
            k_restir_visibility<64, true><<<blocks, 128, 0, s>>>(d);
        }
    } else {
        if (deep_stack) {
            k_restir_spatial<128, false><<<blocks, 128, 0, s>>>(d);
            k_restir_visibility<128, false><<<blocks, 128, 0, s>>>(d);
        } else {
            k_restir_spatial<64, false><<<blocks, 128, 0, s>>>(d);
            k_restir_visibility<64, false><<<blocks, 128, 0, s>>>(d);
        }
    }
}

}  // namespace re
