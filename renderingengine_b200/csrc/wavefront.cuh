// Device-side state of the wavefront path tracer.
//
// Path state lives in HBM as structure-of-arrays: every field is its own
// 16-byte-per-path array, so each stage loads and stores exactly the lanes it
// uses with coalesced 128-bit accesses (the reference keeps one 192-byte
// WfPathState record per path, WavefrontTypes.hpp:182-196).  Ray and shadow
// queues are SoA too.  Queue counts, per-warp work counters and error counters
// sit in one small counter block that is zeroed once per frame.
#pragma once

#include "lights.cuh"
#include "restir.cuh"
#include "traverse.cuh"

namespace re {

constexpr uint32_t kMaxDepth = 16u;
constexpr uint32_t kSlotsPerBounce = 10u;
// Per-bounce counter slots.  Continue: vertices the first split-Shade kernel
// records; the NEE and BSDF-sampling kernels' work counters.
constexpr uint32_t kSlotRays = 0, kSlotShadows = 1, kSlotWorkIntersect = 2, kSlotWorkShade = 3,
                   kSlotWorkShadow = 4, kSlotWorkNee = 5, kSlotNonFinite = 6, kSlotNegativePdf = 7,
                   kSlotContinue = 8, kSlotWorkContinue = 9;
// Global counter slots after the per-bounce block.
constexpr uint32_t kGlobalBase = kMaxDepth * kSlotsPerBounce;
constexpr uint32_t kSlotFatal = kGlobalBase + 0;
// ReSTIR statistics (GpuRestirStatisticsV3 counts, RestirAbiV3.hpp:172-178).
constexpr uint32_t kSlotRestirBase = kGlobalBase + 4;
constexpr uint32_t kRsStatGenerated = 0, kRsStatValid = 1, kRsStatRejected = 2, kRsStatMClamped = 3,
                   kRsStatTemporalAttempts = 4, kRsStatTemporalAccepted = 5, kRsStatSpatialAttempts = 6,
                   kRsStatSpatialAccepted = 7, kRsStatVisSubmitted = 8, kRsStatVisEvaluated = 9,
                   kRsStatVisVisible = 10, kRsStatVisDuplicate = 11;
constexpr uint32_t kCounterWords = kGlobalBase + 16;

// Path flags (WavefrontTypes.hlsli:42-50).
constexpr uint32_t kPathActive = 1u << 0, kPathPrevDelta = 1u << 1, kPathPrevSpecular = 1u << 2,
                   kPathTerminated = 1u << 3, kPathError = 1u << 4, kPathPrevRestirOwned = 1u << 5;

constexpr uint32_t kFatalRayOverflow = 1u << 0, kFatalNextOverflow = 1u << 2, kFatalShadowOverflow = 1u << 3,
                   kFatalShadePathIndex = 1u << 17;

// Frame parameters derived from re_frame_constants (validated on the host).
struct FrameParams {
    f3 cam_pos;
    float tan_half_fov;
    f3 cam_fwd;
    float aspect;
    f3 cam_right;
    float pad0;
    f3 cam_up;
    float pad1;
    uint32_t width, height, sample, max_depth;
    uint32_t seed_lo, seed_hi, estimator, stream;
    float rr_start, rr_min, rr_max, eps;
    uint32_t accumulate, pixel_count, profile, pad3;  // profile: leave the film untouched
    uint32_t path_offset;  // first path of this view in the path pool
    uint32_t scene_slot;   // index into WfDevice::scenes
    uint32_t pixel_base;   // first launch index of this view (pixels of earlier views)
    uint32_t pad5;
    RestirParams rs;  // rs.enabled: ReSTIR owns primary direct lighting this frame
    // environment_to_world rows 0..2, world_to_environment rows 3..5 of the
    // frame record (identity when the record leaves them all zero).
    float4 env_xf[6];
};

// A resident scene as the kernels see it: traversal view, hit attributes,
// emitter map, materials and light tables.
struct SceneSlot {
    TraceSceneView scene;
    const float4* attrs;          // DeviceAttr (normals + identity)
    const uint32_t* emitter;      // light index per leaf-ordered triangle
    const float4* materials;      // 8 x float4 per PbrMaterialGpu
    uint32_t material_count;
    LightView lights;
};

// The views of one launch: views[0 .. view_count) in launch order (by scene
// slot, then path_offset); the paths of view v are [path_offset,
// path_offset + pixel_count).  Views need not be adjacent in the pool: the
// per-pixel kernels walk the launch indices [0, pixel_total), view v owning
// [pixel_base, pixel_base + pixel_count).
struct BatchParams {
    uint32_t view_count;
    uint32_t path_end;     // one past the last path of the last view
    uint32_t pad0, pad1;   // deepest view's maximum depth; profiling pass
    uint32_t pixel_total;  // pixels of all views
    uint32_t pad2, pad3, pad4;
};

// Ray-queue path words carry the path's scene slot in the top bits, so the
// traversal kernels find the scene without another dependent load.
constexpr uint32_t kPathBits = 27u;
constexpr uint32_t kPathMask = (1u << kPathBits) - 1u;
constexpr uint32_t kMaxSceneSlots = RE_MAX_SCENE_SLOTS;
constexpr uint32_t kNoView = 0xffffffffu;
__host__ __device__ __forceinline__ uint32_t pack_path(uint32_t path, uint32_t slot) {
    return path | (slot << kPathBits);
}

// View of launch index c < pixel_total: binary search over pixel_base
// (views[0].pixel_base == 0, so the search ends at a view).
__device__ __forceinline__ uint32_t launch_view(const FrameParams* views, uint32_t view_count, uint32_t c) {
    uint32_t lo = 1, hi = view_count;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (views[mid].pixel_base <= c) lo = mid + 1;
        else hi = mid;
    }
    return lo - 1u;
}

struct WfDevice {
    const SceneSlot* scenes;      // scene table (kMaxSceneSlots entries)
    uint32_t capacity;
    const FrameParams* views;     // per-view frame parameters
    const BatchParams* batch;
    uint32_t* path_view;          // view index of every path (kNoView: unused)
    // Path state.
    float4* beta;                 // throughput.xyz, eta scale
    float4* beta_d;               // diffuse throughput
    float4* beta_s;               // specular throughput
    float4* acc_cam;              // camera emission
    float4* acc_dd;               // direct diffuse
    float4* acc_ds;               // direct specular
    float4* acc_id;               // indirect diffuse
    float4* acc_is;               // indirect specular
    float4* prev_pos_pdf;
    float4* prev_ng;
    float4* prev_ns;
    uint4* ident;                 // pixel, sample, bounce, flags
    // Ray queues (ping-pong by bounce parity) and the hit buffer.
    float4* ray_o[2];
    float4* ray_d[2];
    uint32_t* ray_path[2];
    float4* hit;                  // t, u, v, triangle | front << 31
    // Shadow queue.
    float4* sh_o;
    float4* sh_d;
    float4* sh_cd;                // diffuse contribution, estimator pdf
    float4* sh_cs;                // specular contribution, combined pdf
    uint4* sh_id;                 // path, bounce, light, ignored primitive
    uint32_t* counters;
    // Film and primary-surface planes.
    float4* film_sum;
    float4* sample_out;
    float4* gb_pos;               // position, view depth
    float4* gb_nrm;               // shading normal, material index bits
    float4* gb_alb;               // base color, roughness
    uint4* gb_id;                 // primary hit: instance, primitive, material, front face (instance ~0: miss)
    // Split Shade hand-off, one record per surviving vertex: position +
    // material, geometric normal + front face, shading normal + queue index.
    float4* vx_pos;
    float4* vx_ng;
    float4* vx_ns;
    uint32_t* film_frames;
    // ReSTIR DI state (allocated on the first RestirPrimary frame).
    float4* prim[2];              // GpuPrimarySurfaceV2 per pixel, ping-pong by frame parity
    Reservoir* rs_temporal;       // initial + temporal reservoirs of this frame
    Reservoir* rs_published[2];   // published reservoirs, ping-pong by frame parity
    uint32_t* rs_reasons;         // RestirRejectionReason per pixel
    float4* rs_direct;            // ReSTIR direct diffuse (first plane) and specular
};

// ReSTIR passes between the bounce loop and Resolve (restir.cu); grid-stride
// over the batch's paths with `blocks` CTAs of 128 threads.
void launch_restir(const WfDevice& d, uint32_t blocks, bool deep_stack, bool wide, cudaStream_t s);
// RestirDebugV3 records (4 x uint4 per pixel) and view (float4 per pixel) of
// `n` published reservoirs; either output may be null.
void launch_restir_debug(const void* published, uint32_t n, uint32_t mode, uint32_t max_m, uint32_t max_age,
                         void* records, void* image, cudaStream_t s);

}  // namespace re
