/*
 * re_b200.h -- C ABI of the B200 (sm_100a) wavefront path-tracing hot path.
 *
 * Every record below is byte-compatible with the RenderingEngine contract it
 * names, so a host that already fills those records (Wave2Runtime, the L4
 * software-GPU backend, the L6 megakernel bridge) can hand its buffers to this
 * library unchanged.  No CUDA or C++ types cross this boundary: streams are
 * passed as `void*` (a cudaStream_t or NULL for the legacy default stream) and
 * every entry point returns an `re_status` code.  Nothing throws across the
 * ABI; the message for the last failure on the calling thread is available
 * from re_last_error().
 *
 * Reference interfaces replaced (paths inside the RenderingEngine project):
 *   - IGpuTraversalBackend::BuildOrUpdateScene / RecordTraceClosestBatch /
 *     RecordTraceAnyBatch      include/rt/gpu/IGpuTraversalBackend.hpp:72-84
 *   - GpuTraversalStatusCode   include/rt/gpu/IGpuTraversalBackend.hpp:15-22
 *   - Wave2Runtime::SetScene / UpdateFrame / RecordFrame / CollectCompletedFrame
 *                              include/renderers/Wave2Runtime.hpp:95-131
 *   - ExecutionArchitecture    include/app/RuntimeConfig.hpp:45-51
 */
#ifndef RE_B200_H
#define RE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define RE_API __declspec(dllexport)
#else
#define RE_API __attribute__((visibility("default")))
#endif

/* ------------------------------------------------------------------------ */
/* Status codes.  0..4 carry the numeric values of GpuTraversalStatusCode    */
/* (IGpuTraversalBackend.hpp:15-22); 5.. are B200-specific failures.         */
/* ------------------------------------------------------------------------ */
typedef enum re_status {
    RE_SUCCESS = 0,
    RE_INVALID_ARGUMENT = 1,
    RE_UNSUPPORTED = 2,
    RE_MISSING_SCENE = 3,
    RE_RECORDING_FAILED = 4,
    RE_CUDA_ERROR = 5,
    RE_OUT_OF_MEMORY = 6,
    RE_FATAL_QUEUE = 7,      /* a wavefront queue overflowed (FatalFlags set) */
    RE_BUDGET_EXCEEDED = 8,  /* serving: request does not fit the HBM budget   */
    RE_NOT_READY = 9,        /* serving: request still in flight               */
    RE_TIMEOUT = 10          /* a bounded device wait gave up                  */
} re_status;

/* Where caller buffers live.  Host buffers are staged through pinned memory. */
typedef enum re_memory {
    RE_MEMORY_HOST = 0,
    RE_MEMORY_DEVICE = 1
} re_memory;

/* ------------------------------------------------------------------------ */
/* 16-byte lanes (AbiFloat4 / AbiUInt4, contracts/AbiTypesV0.hpp).           */
/* ------------------------------------------------------------------------ */
typedef struct re_float4 { float x, y, z, w; } re_float4;
typedef struct re_uint4 { uint32_t x, y, z, w; } re_uint4;

/* Geometry / instance / material flag bits (contracts/SceneAbiV0.hpp:16-44). */
#define RE_GEOMETRY_FLAG_OPAQUE        (1u << 0)
#define RE_GEOMETRY_FLAG_ALPHA_MASK    (1u << 1)
#define RE_GEOMETRY_FLAG_DOUBLE_SIDED  (1u << 2)
#define RE_INSTANCE_FLAG_VISIBLE       (1u << 0)
#define RE_INSTANCE_FLAG_CASTS_SHADOW  (1u << 1)
#define RE_MATERIAL_FLAG_DOUBLE_SIDED  (1u << 0)
#define RE_MATERIAL_FLAG_ALPHA_MASK    (1u << 1)
#define RE_MATERIAL_FLAG_EMISSIVE      (1u << 2)

/* HitKind / HitFlags (contracts/RayHitAbiV0.hpp:15-28). */
#define RE_HIT_KIND_MISS      0u
#define RE_HIT_KIND_TRIANGLE  1u
#define RE_HIT_KIND_INVALID   3u
#define RE_HIT_FLAG_FRONT_FACE (1u << 0)

/* CanonicalTraversalTriangle, 176 B (rt/gpu/CanonicalTraversalScene.hpp:15-25).
 * identity = (stable instance, primitive, geometry, material);
 * metadata = (geometry flags, material flags, traversal ID, instance flags). */
typedef struct re_canonical_triangle {
    re_float4 positions[3];
    re_float4 normals[3];
    re_float4 texcoords[3];
    re_uint4 identity;
    re_uint4 metadata;
} re_canonical_triangle;

/* Object-space scene records of SceneAbiV0 (contracts/SceneAbiV0.hpp:77-112),
 * the input of re_scene_expand_canonical. */
typedef struct re_mat4_rows {
    re_float4 row0, row1, row2, row3;
} re_mat4_rows;
typedef struct re_gpu_vertex_v0 {      /* GpuVertexV0, 64 B                  */
    re_float4 position;                /* object space, w = 1                */
    re_float4 normal;                  /* object space unit normal, w = 0    */
    re_float4 tangent;
    re_float4 texcoord0;
} re_gpu_vertex_v0;
typedef struct re_gpu_geometry_v0 {    /* GpuGeometryV0, 64 B                */
    re_uint4 index_range;              /* first index, count, vertex offset, first primitive ID */
    re_uint4 identity;                 /* geometry ID, mesh ID, material, GeometryFlags */
    re_float4 local_bounds_min;
    re_float4 local_bounds_max;
} re_gpu_geometry_v0;
typedef struct re_gpu_instance_v0 {    /* GpuInstanceV0, 224 B               */
    re_mat4_rows object_to_world;
    re_mat4_rows world_to_object;
    re_mat4_rows previous_object_to_world;
    re_uint4 metadata;                 /* first geometry, geometry count, stable instance ID, InstanceFlags */
    re_uint4 reserved0;
} re_gpu_instance_v0;
typedef struct re_gpu_material_v0 {    /* GpuMaterialV0, 128 B               */
    re_float4 base_color_factor;
    re_float4 emissive_factor_strength;
    re_float4 surface_params;
    re_float4 transmission_params;
    re_float4 attenuation_color_distance;
    re_uint4 texture_image_indices;
    re_uint4 texture_sampler_indices;
    re_uint4 metadata;                 /* MaterialModel, MaterialFlags, stable ID, reserved */
} re_gpu_material_v0;

/* SoftwareNodeRecord, 48 B (rt/software_gpu/SoftwareGpu.hpp:46-60).  Leaf iff
 * links.y != 0: links.x = first leaf-ordered primitive, links.y = count.
 * Interior: links.x / links.z = left / right child.  links.w = parent. */
typedef struct re_software_node {
    re_float4 bounds_min;
    re_float4 bounds_max;
    re_uint4 links;
} re_software_node;

/* GpuRayQueueRecordV1, 64 B (contracts/GpuRecordsAbiV1.hpp:80-86).
 * identity = (ray ID, path ID, bounce, visibility mask); tMin/tMax exclusive. */
typedef struct re_ray_record {
    re_float4 origin_tmin;
    re_float4 direction_tmax;
    re_uint4 identity;
    re_uint4 rng;
} re_ray_record;

/* GpuHitQueueRecordV1, 96 B (contracts/GpuRecordsAbiV1.hpp:90-97).
 * ids = (instance, primitive, geometry, material);
 * metadata = (ray ID, HitKind, HitFlags, path ID). */
typedef struct re_hit_record {
    re_float4 position_t;
    re_float4 geometric_normal_bary_u;
    re_float4 shading_normal_bary_v;
    re_uint4 ids;
    re_uint4 metadata;
    re_uint4 reserved0;
} re_hit_record;

/* PbrMaterialGpu, 128 B (integrators/megakernel/MegakernelBridge.hpp:259-269).
 * metadata = (BSDF model, allowed lobes, complex conductor Fresnel, flags). */
typedef struct re_material {
    re_float4 base_color_metallic;
    re_float4 emissive_roughness;
    re_float4 transmission_ior;
    re_float4 attenuation_color_distance;
    re_float4 f0;
    re_float4 conductor_eta;
    re_float4 conductor_k;
    re_uint4 metadata;
} re_material;

/* PbrLightGpu, 96 B (integrators/megakernel/MegakernelBridge.hpp:274-282).
 * identity = (LightType, LightFlags, stable light ID, primitive ID);
 * payload = (fixture geometry, texture, distribution offset, instance ID). */
typedef struct re_light {
    re_float4 position_range;
    re_float4 direction_cos_outer;
    re_float4 radiance_scale;
    re_float4 shape_params;
    re_uint4 identity;
    re_uint4 payload;
} re_light;

/* BSDF models (resources/shaders/include/bsdf/PbrBsdf.hlsli:75-80). */
#define RE_BSDF_LAMBERT                  0u
#define RE_BSDF_GGX_CONDUCTOR            1u
#define RE_BSDF_GGX_DIELECTRIC_REFLECTION 2u
#define RE_BSDF_SMOOTH_GLASS             3u
#define RE_BSDF_ROUGH_DIELECTRIC         4u
#define RE_BSDF_METALLIC_ROUGHNESS       5u
/* Lobe bits (PbrBsdf.hlsli:55-73). */
#define RE_LOBE_DIFFUSE      (1u << 0)
#define RE_LOBE_GLOSSY       (1u << 1)
#define RE_LOBE_SPECULAR     (1u << 2)
#define RE_LOBE_REFLECTION   (1u << 3)
#define RE_LOBE_TRANSMISSION (1u << 4)
#define RE_LOBE_ALL          0x1fu
/* Material flags in metadata.w (pbr_l6_types.hlsli:27-28). */
#define RE_MATERIAL_PURE_EMITTER (1u << 0)

/* Light types and flags (pbr_l6_types.hlsli:11-22). */
#define RE_LIGHT_POINT             0u
#define RE_LIGHT_DIRECTIONAL       1u
#define RE_LIGHT_SPOT              2u
#define RE_LIGHT_SPHERE_AREA       3u
#define RE_LIGHT_EMISSIVE_TRIANGLE 4u
#define RE_LIGHT_ENVIRONMENT       5u
#define RE_LIGHT_FLAG_ENABLED   (1u << 0)
#define RE_LIGHT_FLAG_TWO_SIDED (1u << 1)
#define RE_LIGHT_SELECTION_UNIFORM 0u
#define RE_LIGHT_SELECTION_POWER   1u

/* ------------------------------------------------------------------------ */
/* Library                                                                   */
/* ------------------------------------------------------------------------ */

/* Message of the last failure on the calling thread ("" after success). */
RE_API const char* re_last_error(void);

/* ---- Scene ingestion ---------------------------------------------------- */
/* Instance expansion on the GPU, as BuildCanonicalTraversalScene
 * (src/rt/gpu/CanonicalTraversalScene.cpp:69-187): every visible instance's
 * geometries' triangles, instance-major, transformed to world space
 * (positions by object_to_world, normals by world_to_object transposed and
 * renormalised in double precision), into CanonicalTraversalTriangle records
 * with the traversal ID = output index.  Inputs in host memory; `out` (room
 * for `out_capacity` records) in `memory`.  RE_INVALID_ARGUMENT with the
 * reference's messages for empty inputs, bad ranges, bad vertex indices,
 * non-finite results or no visible triangle; `*out_count` is the count. */
RE_API re_status re_scene_expand_canonical(const re_gpu_vertex_v0* vertices, uint32_t vertex_count,
                                           const uint32_t* indices, uint32_t index_count,
                                           const re_gpu_geometry_v0* geometries, uint32_t geometry_count,
                                           const re_gpu_instance_v0* instances, uint32_t instance_count,
                                           const re_gpu_material_v0* materials, uint32_t material_count,
                                           re_canonical_triangle* out, uint32_t out_capacity, uint32_t* out_count,
                                           uint32_t memory, uint32_t device, void* stream);

/* ---- Image outputs of a film (host code; read the film first) ---------- */
/* Linear-RGB identity hash of HashLinearRgbPixels
 * (src/rt/cpu/ImageOutput.cpp:343-380): 64-bit FNV-1a over the tag "RERGB"
 * 1 3 0, width and height (little-endian 32-bit), then each component's bits
 * with -0 folded to +0.  `rgb` holds width x height x 3 floats, row-major,
 * top row first; RE_INVALID_ARGUMENT for zero dimensions, another component
 * count or a non-finite component (ValidateLinearRgb, ImageOutput.cpp:28-79). */
RE_API re_status re_image_hash_linear_rgb(uint32_t width, uint32_t height, const float* rgb,
                                          uint64_t component_count, uint64_t* hash_out);
/* 32-bit float RGB OpenEXR file, as WriteLinearRgbExr (ImageOutput.cpp:156-216)
 * writes it: scanline, channels B, G, R, ZIP compression (16-line blocks).
 * Same validation as the hash. */
RE_API re_status re_image_write_exr(const char* path, uint32_t width, uint32_t height, const float* rgb,
                                    uint64_t component_count);
/* ABI version of this header (major << 16 | minor). */
RE_API uint32_t re_abi_version(void);
#define RE_ABI_VERSION ((1u << 16) | 0u)

/* ExecutionArchitecture value appended after {Staged, CpuReference, Megakernel,
 * Wavefront} (app/RuntimeConfig.hpp:45-51) and its CLI token. */
#define RE_EXECUTION_ARCHITECTURE_CUDA_WAVEFRONT 4u
RE_API const char* re_execution_architecture_token(void); /* "cuda-wavefront" */

/* CapabilityTable rule for the new architecture (app/CapabilityTable.cpp:100-180):
 * returns 1 when (transport, backend, estimator) is built, 0 otherwise, and
 * fills `reason` (may be NULL) with a fixed string explaining a rejection. */
#define RE_TRANSPORT_PBR 0u
#define RE_TRANSPORT_WHITTED 1u
#define RE_BACKEND_GPU_FLATTENED_SAH 1u
#define RE_BACKEND_GPU_LBVH 4u
RE_API int re_capability_is_built(uint32_t transport, uint32_t backend,
                                  uint32_t estimator, const char** reason);

/* ------------------------------------------------------------------------ */
/* Scene: IGpuTraversalBackend::BuildOrUpdateScene                           */
/* ------------------------------------------------------------------------ */
typedef struct re_scene re_scene;

#define RE_BUILD_FLATTENED_SAH 0u  /* BuildKind::FlattenedCpuSah (SoftwareGpu.hpp:130-134) */
#define RE_BUILD_LBVH          1u  /* BuildKind::KarrasLbvh, built on the GPU             */

typedef struct re_scene_desc {
    const re_canonical_triangle* triangles; /* host memory                       */
    uint32_t triangle_count;
    /* Optional caller-built flattened SAH (FlattenCanonicalL3BinnedSah).  When
     * non-NULL, `triangles` must already be in the nodes' leaf order. */
    const re_software_node* nodes;
    uint32_t node_count;
    uint32_t build_kind;        /* RE_BUILD_*                                     */
    uint32_t sah_bins;          /* 0 -> 16 (Bvh.hpp:68)                            */
    uint32_t max_leaf_size;     /* 0 -> 4  (Bvh.hpp:69)                            */
    uint64_t fingerprint;       /* scene identity, must be non-zero               */
    uint32_t generation;        /* must be non-zero                               */
    uint32_t device;            /* CUDA ordinal                                   */
} re_scene_desc;

typedef struct re_scene_info {
    uint32_t triangle_count;
    uint32_t node_count;        /* binary nodes (SoftwareNodeRecord count)       */
    uint32_t max_depth;
    uint32_t leaf_count;
    uint64_t device_bytes;      /* resident HBM bytes of this scene              */
    double build_ms;            /* host SAH build or GPU LBVH build time          */
    uint32_t node_bytes;        /* bytes per device node record                   */
    uint32_t triangle_bytes;    /* bytes per device triangle record               */
    double gpu_build_ms;        /* device time of the GPU LBVH passes (0 for SAH)  */
} re_scene_info;

RE_API re_status re_scene_create(const re_scene_desc* desc, re_scene** out_scene);
/* A scene from CanonicalTraversalTriangle records already in device memory
 * (desc->triangles is a device pointer, e.g. re_scene_expand_canonical's
 * output; build_kind RE_BUILD_LBVH, no caller nodes): the primitive checks
 * of re_scene_create run on the device, and traversal IDs must also be a
 * permutation of 0 .. triangle_count - 1 (as the expansion numbers them);
 * the records are read, never kept.  Same scene as re_scene_create on a host
 * copy of the records. */
RE_API re_status re_scene_create_from_device(const re_scene_desc* desc, re_scene** out_scene);
RE_API re_status re_scene_destroy(re_scene* scene);
RE_API re_status re_scene_info_get(const re_scene* scene, re_scene_info* out);
/* Alpha-masked geometry (pbr_software_traversal.hlsli:207-240, 430-470):   */
/* triangles whose geometry or material flags carry ALPHA_MASK are tested  */
/* for coverage before closest- and any-hit acceptance.  A candidate's     */
/* material (identity.w) indexes `materials` (GpuMaterialV0): alpha =       */
/* base_color_factor.w, times, when texture_image_indices.x names a layer,  */
/* the atlas texel at the interpolated texture coordinate (nearest texel,   */
/* clamped to the edge); below surface_params.w the candidate is skipped.   */
/* A material index beyond material_count, a layer >= layers, a sampler id  */
/* other than sampler_id with a layer, or a sampler id without a layer ends */
/* that ray's traversal as invalid, as in the reference.  atlas_alpha:      */
/* layers x height x width floats (the alpha channel in [0, 1]).  Set it    */
/* before binding the scene to renderers; it may be reset.                  */
RE_API re_status re_scene_set_alpha_masks(re_scene* scene, const re_gpu_material_v0* materials,
                                          uint32_t material_count, const float* atlas_alpha, uint32_t width,
                                          uint32_t height, uint32_t layers, uint32_t sampler_id);
/* Copy the scene's flattened 48 B node records (node order of the build) and
 * the leaf-ordered triangle permutation (source index per leaf slot) to host. */
RE_API re_status re_scene_export_flat(const re_scene* scene, re_software_node* nodes,
                                      uint32_t node_capacity, uint32_t* leaf_order,
                                      uint32_t order_capacity);

/* Host-only binned-SAH build + flatten (no GPU needed): the replacement of
 * Rt::Cpu::Bvh<float>(BinnedSah) + SoftwareGpu::FlattenCanonicalL3BinnedSah
 * (rt/cpu/Bvh.hpp:82-133, src/rt/software_gpu/SoftwareGpu.cpp:1109-1247).
 * Writes pre-order 48 B node records and the source triangle index of every
 * leaf slot.  node_capacity must be >= 2 * count - 1. */
RE_API re_status re_sah_build_host(const re_canonical_triangle* triangles, uint32_t count,
                                   uint32_t sah_bins, uint32_t max_leaf_size,
                                   re_software_node* nodes_out, uint32_t node_capacity,
                                   uint32_t* node_count_out, uint32_t* leaf_order_out,
                                   uint32_t* max_depth_out);

/* ------------------------------------------------------------------------ */
/* Trace batches: RecordTraceClosestBatch / RecordTraceAnyBatch              */
/* Offsets are record indices, never bytes (IGpuTraversalBackend.hpp:56-70). */
/* The batch is rejected with RE_MISSING_SCENE unless fingerprint+generation */
/* match the scene.  The call is asynchronous on `stream` for device memory  */
/* and synchronous for host memory.                                          */
/* ------------------------------------------------------------------------ */
typedef struct re_trace_batch {
    const re_ray_record* rays;
    re_hit_record* hits;
    uint32_t ray_offset;
    uint32_t hit_offset;
    uint32_t ray_count;
    uint32_t memory;            /* re_memory of rays and hits                      */
    uint64_t fingerprint;
    uint32_t generation;
    uint32_t reserved;
    void* stream;
} re_trace_batch;

/* Traversal counters (GpuTraversalCounterSlot, SoftwareGpu.hpp:206-221). */
typedef struct re_traversal_counters {
    uint64_t node_tests;
    uint64_t triangle_tests;
    uint64_t stack_overflows;
    uint64_t invalid_rays;
    uint64_t invalid_hits;
    uint64_t max_stack_depth;
    uint64_t leaf_visits;
    uint64_t leaf_primitives;
    uint64_t max_leaf_occupancy;
} re_traversal_counters;

RE_API re_status re_trace_closest(re_scene* scene, const re_trace_batch* batch);
RE_API re_status re_trace_any(re_scene* scene, const re_trace_batch* batch);
/* Same traversal with per-batch counters accumulated into *counters (slower). */
RE_API re_status re_trace_counted(re_scene* scene, const re_trace_batch* batch,
                                  uint32_t any_hit, re_traversal_counters* counters);

/* ------------------------------------------------------------------------ */
/* Wavefront renderer: Wave2Runtime::SetScene / UpdateFrame / RecordFrame /  */
/* CollectCompletedFrame (renderers/Wave2Runtime.hpp:95-131) for the         */
/* cuda-wavefront execution architecture.                                    */
/* ------------------------------------------------------------------------ */
typedef struct re_renderer re_renderer;

/* MegakernelFrameConstantsGpu, 304 B (MegakernelBridge.hpp:300-322).  The
 * renderer reads the camera, image (width, height, sample index, maximum
 * depth), sampling (seed low/high, light selection, direct estimator),
 * russianRoulette (start depth, min, max, ray epsilon) and output (stream tag,
 * -, transport, shadow method) lanes; it fills the trace/distribution counts
 * from the scene it holds. */
typedef struct re_frame_constants {
    re_float4 camera_position_tan_half_fov;
    re_float4 camera_forward_aspect;
    re_float4 camera_right_lens_radius;
    re_float4 camera_up_exposure;
    re_uint4 image;
    re_uint4 trace;
    re_uint4 sampling;
    re_uint4 environment;
    re_uint4 distribution;
    re_float4 russian_roulette;
    re_float4 scene_center_radius;
    re_float4 environment_to_world[3];
    re_float4 world_to_environment[3];
    re_uint4 traversal;
    re_uint4 output;
} re_frame_constants;

/* Direct-light estimator values of the frame's sampling.w lane
 * (pbr_l6_types.hlsli:36-39). */
#define RE_ESTIMATOR_BSDF_ONLY 0u
#define RE_ESTIMATOR_NEE 1u
#define RE_ESTIMATOR_MIS 2u
#define RE_ESTIMATOR_RESTIR_PRIMARY 3u
#define RE_SHADOW_PHYSICAL 2u

/* FatalFlags (integrators/wavefront/include/WavefrontTypes.hpp:68-92). */
#define RE_FATAL_RAY_OVERFLOW        (1u << 0)
#define RE_FATAL_NEXT_OVERFLOW       (1u << 2)
#define RE_FATAL_SHADOW_OVERFLOW     (1u << 3)
#define RE_FATAL_INVALID_CAPACITY    (1u << 6)
#define RE_FATAL_RAYGEN_PBR_FRAME    (1u << 9)
#define RE_FATAL_SHADOW_METHOD       (1u << 20)

typedef struct re_renderer_desc {
    uint32_t max_width;         /* path capacity = max_width * max_height     */
    uint32_t max_height;
    uint32_t max_depth;         /* <= 16                                      */
    uint32_t device;
} re_renderer_desc;

/* Autotuned launch configuration (block size, persistent grid, fused
 * intersect+shade split point, CUDA-graph capture of the bounce sequence). */
typedef struct re_renderer_tuning {
    uint32_t block_size;        /* 128, 256 or 512                             */
    uint32_t blocks_per_sm;     /* persistent CTAs per SM, 0 = occupancy max   */
    uint32_t fuse_intersect_shade; /* 1: intersect and shade in one kernel     */
    uint32_t use_graph;         /* 1: replay the frame as one CUDA graph       */
    uint32_t shade_variant;     /* 0: out-of-line BSDF calls, 1: inlined <=128
                                   registers, 2: inlined <=168 registers; split
                                   in two kernels (NEE | BSDF sampling): 3
                                   out-of-line, 4 inlined (the default); 5:
                                   three kernels (hit and emission | NEE |
                                   BSDF sampling), inlined; 6 / 7: variant 5
                                   with registers capped for 6 / 5 CTAs of
                                   128 per SM                                  */
    uint32_t traversal_refill;  /* 0: packet fetch; k in 1..32: a warp refills
                                   idle lanes once k lanes are idle, stepping
                                   one node or leaf at a time: four-wide nodes
                                   in modes 2-4, child pairs in modes 0-1      */
    uint32_t traversal_mode;    /* split Intersect and TraceShadow with refill 0:
                                   0: one child-pair node or leaf per step (the
                                   reference's loop); 1: while-while with
                                   postponed leaves; 2: four-wide 128 B nodes
                                   (built on first use), postponed leaves; 3
                                   (default): per launch, 4 when a scene of
                                   the launch is an LBVH (one triangle per
                                   leaf), else 2; 4: four-wide, one node or
                                   leaf per step; 5: eight-wide 256 B nodes;
                                   6: eight-wide nodes compressed to 96 B
                                   (8-bit child boxes, decoded outward);
                                   7 / 8: modes 4 / 2 with a conservative
                                   one-fma slab test (enters every box the
                                   reference's test enters).  Same closest
                                   hits and visibility in every mode, except
                                   where the reference's own slab rounding
                                   rejects the box of the triangle a ray
                                   hits (modes 6-8 enter it)                  */
} re_renderer_tuning;

/* Film read-back selectors. */
#define RE_FILM_MEAN              0u  /* progressive mean over frames          */
#define RE_FILM_SAMPLE            1u  /* last frame's per-pixel sample value    */
#define RE_FILM_CAMERA_EMISSION   2u
#define RE_FILM_DIRECT_DIFFUSE    3u
#define RE_FILM_DIRECT_SPECULAR   4u
#define RE_FILM_INDIRECT_DIFFUSE  5u
#define RE_FILM_INDIRECT_SPECULAR 6u
#define RE_FILM_PRIMARY_POSITION  7u  /* xyz position, w view depth (0: miss)   */
#define RE_FILM_PRIMARY_NORMAL    8u  /* xyz shading normal, w material index   */
#define RE_FILM_PRIMARY_ALBEDO    9u  /* xyz base color, w roughness            */
#define RE_FILM_PRIMARY_IDENTITY 10u  /* uint32 instance, primitive, material,
                                         front face (instance 0xffffffff: miss) */

typedef struct re_frame_telemetry {
    uint64_t path_rays;         /* closest-hit rays traced (all bounces)       */
    uint64_t shadow_rays;       /* any-hit rays traced                          */
    uint32_t fatal_mask;        /* FatalFlags of the last frame (0 = ok)        */
    uint32_t non_finite;
    uint32_t negative_pdf;
    uint32_t frames_accumulated;
    uint32_t active_per_bounce[16];
    uint32_t shadow_per_bounce[16];
    double gpu_ms;              /* device time of the last frame               */
    uint64_t total_path_rays;   /* since the film was last reset               */
    uint64_t total_shadow_rays;
} re_frame_telemetry;

RE_API re_status re_renderer_create(const re_renderer_desc* desc, re_renderer** out);
RE_API re_status re_renderer_destroy(re_renderer* r);
RE_API re_status re_renderer_set_tuning(re_renderer* r, const re_renderer_tuning* tuning);
/* Binds a resident scene plus its PbrMaterialGpu / PbrLightGpu records and the
 * FixtureTriangleGpu records emissive-triangle lights point at
 * (payload.x); builds the light alias table (uniform or power weighted) and
 * the per-triangle emitter map.  Copies everything into HBM. */
RE_API re_status re_renderer_set_scene(re_renderer* r, re_scene* scene,
                                       const re_material* materials, uint32_t material_count,
                                       const re_light* lights, uint32_t light_count,
                                       const re_float4* fixture_triangles /* 4 lanes each */,
                                       uint32_t fixture_count, uint32_t light_selection,
                                       float scene_radius);
/* Renders one sample per pixel.  accumulate = 0 resets the progressive film
 * first.  Asynchronous on `stream`; fails with RE_FATAL_QUEUE / RE_INVALID_ARGUMENT
 * when the frame contract is violated (FatalFlags are also reported by
 * re_renderer_collect). */
RE_API re_status re_renderer_render(re_renderer* r, const re_frame_constants* frame,
                                    uint32_t accumulate, void* stream);
/* Copies one film plane (re_float4 per pixel, row-major) to `out`. */
RE_API re_status re_renderer_read_film(re_renderer* r, uint32_t plane, re_float4* out,
                                       uint32_t pixel_count, uint32_t memory, void* stream);
/* Starts reading one film plane of a view (pixels [path_offset, path_offset +
 * pixel_count)) into host memory, ordered after the work queued on `stream`,
 * and returns without waiting.  The plane is first copied on the device into
 * one of two renderer-owned staging buffers (used in turn), then to
 * `host_out` on the renderer's own copy stream, so the next frame queued on
 * `stream` overlaps the transfer: two frames in flight, as the reference
 * keeps two frame slots and reads a slot only after its fence
 * (Wave2Runtime.hpp:24, CollectCompletedFrame Wave2Runtime.hpp:95-131).
 * `host_out` should be pinned (page-locked) for the copy to overlap; it must
 * stay valid until re_renderer_wait_reads returns.  A third read in flight
 * waits, on the device, for the host copy of the first. */
RE_API re_status re_renderer_read_view_async(re_renderer* r, uint32_t plane, uint32_t path_offset,
                                             uint32_t pixel_count, re_float4* host_out, void* stream);
/* Blocks until every read started by re_renderer_read_view_async has landed. */
RE_API re_status re_renderer_wait_reads(re_renderer* r);
/* Synchronizes and returns the last frame's counters (CollectCompletedFrame). */
RE_API re_status re_renderer_collect(re_renderer* r, re_frame_telemetry* out);
/* Device pointer of a film plane (valid until the renderer is destroyed). */
RE_API re_status re_renderer_film_pointer(re_renderer* r, uint32_t plane, void** out);

/* ------------------------------------------------------------------------ */
/* Batched views: many cameras over many resident scenes in one launch.     */
/* Every bound scene occupies a slot; every view names its slot, a range of */
/* the renderer's path pool (path_offset .. + width * height) and a key     */
/* that identifies it across launches (its ReSTIR history).  One launch     */
/* renders one sample of every view: one persistent wavefront (RayGen ->    */
/* Intersect / Shade / Shadow per bounce -> ReSTIR -> Resolve) over the     */
/* union of the views' paths, replayed from one CUDA graph for every batch  */
/* of the same depth.  Results are independent of the batch: the random    */
/* streams are keyed by (pixel within the view, sample).                    */
/* The single-view calls above are the batch of one view in slot 0 at path  */
/* offset 0 with key 0.                                                      */
/* ------------------------------------------------------------------------ */
#define RE_MAX_SCENE_SLOTS 32u
#define RE_MAX_BATCH_VIEWS 256u

typedef struct re_view_desc {
    const re_frame_constants* frame;  /* camera, extent, sample index, depth, estimator */
    uint32_t scene_slot;
    uint32_t path_offset;             /* first path of the view in the path pool        */
    uint32_t accumulate;              /* 0: this sample restarts the view's film         */
    uint32_t reserved;
    uint64_t view_key;                /* the view's identity across launches             */
} re_view_desc;

/* Binds a resident scene with its materials / lights to a slot (the tables of
 * re_renderer_set_scene).  Synchronises the device. */
RE_API re_status re_renderer_bind_scene(re_renderer* r, uint32_t slot, re_scene* scene,
                                        const re_material* materials, uint32_t material_count,
                                        const re_light* lights, uint32_t light_count,
                                        const re_float4* fixture_triangles, uint32_t fixture_count,
                                        uint32_t light_selection, float scene_radius);
RE_API re_status re_renderer_unbind_scene(re_renderer* r, uint32_t slot);
/* Environment map of a scene slot (the environment variant of              */
/* Wave2Runtime's scene build, Wave2Runtime.cpp:560-612): width x height     */
/* linear-RGBA texels, equirectangular, row 0 at theta = 0 (+y of           */
/* environment space), u = atan2(z, x) / 2 pi, v = acos(y) / pi, read with  */
/* nearest texels, u wrapping and v clamped (Wave2Runtime.cpp:2568-2579).   */
/* Builds the importance tables (BuildEnvironmentDistribution,              */
/* MegakernelBridge.cpp:191-273) from the texels' luminance                  */
/* 0.2126 r + 0.7152 g + 0.0722 b; the slot's enabled RE_LIGHT_ENVIRONMENT   */
/* light (one at most) then radiates it, scaled by its radiance_scale, with  */
/* pi R^2 scale x integrated luminance as its power weight.  Call before     */
/* binding the slot's scene (unbind first to change it); NULL texels clears  */
/* it.  Frames rotate the map with their environment_to_world /              */
/* world_to_environment rows (all zero = identity).  ReSTIR DI frames over a */
/* scene with an environment light are rejected (RE_UNSUPPORTED).           */
RE_API re_status re_renderer_set_environment(re_renderer* r, uint32_t slot, const re_float4* texels,
                                             uint32_t width, uint32_t height);
/* The slot's environment importance tables as built: row alias entries     */
/* (height), column alias entries (height x width; AliasEntryGpu records     */
/* q, pmf, alias, item) and the integrated luminance.  NULL outputs skip.   */
RE_API re_status re_renderer_environment_tables(re_renderer* r, uint32_t slot, re_float4* rows_out,
                                                re_float4* columns_out, double* integrated_luminance);
/* One sample of every view (path ranges must not overlap). Asynchronous. */
RE_API re_status re_renderer_render_views(re_renderer* r, const re_view_desc* views, uint32_t view_count,
                                          void* stream);
/* Copies a film plane of the paths [path_offset, path_offset + pixel_count). */
RE_API re_status re_renderer_read_view(re_renderer* r, uint32_t plane, uint32_t path_offset,
                                       uint32_t pixel_count, re_float4* out, uint32_t memory, void* stream);
/* Forgets a view's ReSTIR history bookkeeping. */
RE_API re_status re_renderer_release_view(re_renderer* r, uint64_t view_key);
RE_API re_status re_renderer_path_capacity(const re_renderer* r, uint32_t* out);
/* Launch plan of one batch step (the render server's policy): the views of
 * each scene are cut, in their given order, into chunks of at most
 * `launch_paths` paths (a larger view is a chunk of its own), and the chunks
 * are placed first-fit into launches of at most `launch_paths` paths.  A
 * large scene fills launches of its own, so its hierarchy stays hot in L2,
 * while small scenes share launches.  Scenes keep the order of their first
 * view.  launch_of_view[i] receives view i's launch index and *launch_count
 * the number of launches.  Host only. */
RE_API re_status re_plan_launches(const uint32_t* scene_slots, const uint32_t* pixel_counts, uint32_t view_count,
                                  uint32_t launch_paths, uint32_t* launch_of_view, uint32_t* launch_count);

/* Per-stage profile of one frame (the reference's per-pass timestamp queries,
 * WavefrontSchedule.hpp:119-132, plus the traversal counters of
 * SoftwareGpu.hpp:206-221).  The frame is rendered twice without touching the
 * film: once with counting traversal kernels (node / triangle tests), once
 * with CUDA events between the split stage launches (times). */
typedef struct re_stage_profile {
    float raygen_ms;
    float resolve_ms;
    float intersect_ms[16];
    float shade_ms[16];
    float shadow_ms[16];
    uint32_t rays[16];
    uint32_t shadows[16];
    uint64_t intersect_node_tests[16];
    uint64_t intersect_triangle_tests[16];
    uint64_t shadow_node_tests[16];
    uint64_t shadow_triangle_tests[16];
    float restir_ms;            /* ReSTIR passes (RestirPrimary frames)       */
    /* Node records fetched by the traversal that ran (64 B child pairs, or
     * 128 B four-wide nodes under traversal_mode 2), bytes per bounce. */
    uint64_t intersect_node_bytes[16];
    uint64_t shadow_node_bytes[16];
} re_stage_profile;
RE_API re_status re_renderer_profile(re_renderer* r, const re_frame_constants* frame,
                                     re_stage_profile* out);

/* ------------------------------------------------------------------------ */
/* ReSTIR DI on the primary surface (estimator RE_ESTIMATOR_RESTIR_PRIMARY). */
/* Frames whose frame constants select that estimator run, after the bounce  */
/* loop, the reference's production passes (resources/shaders/restir/       */
/* Restir*V3.comp.hlsl): streamed initial RIS over light candidates,        */
/* temporal reuse of the previous frame's published reservoir (reprojected  */
/* through the previous frame's camera), spatial reuse, one winner shadow   */
/* ray, resolve, and the direct term added to the film's direct planes.     */
/* Reservoirs are GpuRestirReservoirV3 records (RestirAbiV3.hpp:149-157),   */
/* surfaces GpuPrimarySurfaceV2 (ReconstructionAbiV2.hpp:44-52).            */
/* ------------------------------------------------------------------------ */
typedef struct re_restir_config {
    uint32_t candidates;          /* RIS candidates per pixel (<= 1024)          */
    uint32_t spatial_neighbors;   /* <= 30 (kMaxSpatialNeighbors)               */
    uint32_t max_m;               /* M cap after every merge                    */
    uint32_t max_history_age;
    uint32_t temporal;            /* 1: temporal reuse                          */
    uint32_t neighbor_mode;       /* 0: 8-direction rings (the reference's      */
                                  /*    table), 1: seeded disk of disk_radius   */
    float disk_radius;            /* pixels                                     */
    float normal_cos;             /* validation (ReSTIRFrameParameters.hpp:19)  */
    float relative_depth;
    float position_distance;
    uint32_t estimator;           /* 0: biased, 1: reference correction        */
                                  /*    (EstimatorMode, restir/RestirTypes.hpp: */
                                  /*    67-71): after spatial reuse, the        */
                                  /*    winner is re-weighted with visibility   */
                                  /*    at the centre and every neighbour       */
                                  /*    (RestirReference*V3.comp.hlsl)          */
} re_restir_config;

/* GpuRestirStatisticsV3 counts of the last frame (RestirAbiV3.hpp:172-178). */
typedef struct re_restir_statistics {
    uint32_t candidates_generated, candidates_valid, candidates_rejected, m_clamped;
    uint32_t temporal_attempts, temporal_accepted, spatial_attempts, spatial_accepted;
    uint32_t visibility_submitted, visibility_evaluated, visibility_visible, visibility_duplicate;
} re_restir_statistics;

/* Planes for re_renderer_restir_pointer (device pointers, last frame). */
#define RE_RESTIR_PUBLISHED   0u  /* GpuRestirReservoirV3 per pixel (final)        */
#define RE_RESTIR_TEMPORAL    1u  /* GpuRestirReservoirV3 per pixel (after temporal) */
#define RE_RESTIR_SURFACES    2u  /* GpuPrimarySurfaceV2 per pixel                 */
#define RE_RESTIR_DIRECT      3u  /* float4 diffuse[pixels] then float4 specular[pixels] */
#define RE_RESTIR_REASONS     4u  /* uint32 RestirRejectionReason per pixel        */

RE_API re_status re_restir_default_config(re_restir_config* out);
RE_API re_status re_renderer_set_restir(re_renderer* r, const re_restir_config* config);
/* Camera cut: the next RestirPrimary frame rejects all temporal history. */
RE_API re_status re_renderer_restir_reset(re_renderer* r);
RE_API re_status re_renderer_restir_statistics(re_renderer* r, re_restir_statistics* out);
RE_API re_status re_renderer_restir_pointer(re_renderer* r, uint32_t plane, void** out);
/* Copies `bytes` of a plane (last frame's pixel count x record size). */
/* Debug view of the last frame's published reservoirs, as RestirDebugV3
 * (resources/shaders/restir/RestirDebugV3.comp.hlsl) writes it: per pixel a
 * GpuRestirDebugV3 record (64 B: light / primitive / provenance IDs, sample
 * generation, weight sum / W / target / final weight with non-finite values
 * as 0, M / age / flags / rejection) to `records_out`, and a float4 view to
 * `image_out`, `mode` as the reference's debug mode: 0 M and age over their
 * caps, 1 the weights as w / (1 + w), 2-5 IDs, provenance, reuse flags and
 * rejection reasons as golden-ratio hues, 6+ final visibility.  Either
 * output may be null; `memory` says where both live. */
RE_API re_status re_renderer_restir_debug(re_renderer* r, uint32_t mode, uint32_t pixel_count, void* records_out,
                                          re_float4* image_out, uint32_t memory, void* stream);
RE_API re_status re_renderer_restir_read(re_renderer* r, uint32_t plane, void* dst, uint64_t bytes,
                                         uint32_t memory, void* stream);

/* ------------------------------------------------------------------------ */
/* Render server: continuous batching of render requests on one GPU.        */
/* Requests (scene, camera, extent, depth, estimator incl. ReSTIR, samples) */
/* arrive over time; every step renders one sample of every admitted        */
/* request in batched launches (re_renderer_render_views; requests grouped  */
/* by scene under a path budget, re_plan_launches), so requests             */
/* that arrive while others are on the GPU join at the next step as path    */
/* ranges and memory free up.  Scenes are registered once (host copies) and */
/* made resident on demand with a GPU LBVH build; resident scenes, the path */
/* pool and the ReSTIR history stay in HBM, admitted against a byte budget, */
/* and the least recently used unpinned scenes are evicted to make room.    */
/* A scene is charged, before its build, 260 B per triangle (two 64 B nodes, */
/* a 64 B triangle, a 64 B attribute record, a 4 B index) plus its material, */
/* light (+24 B each) and fixture records and 1 MiB; once built, its        */
/* measured bytes.  A request's film equals the same request rendered alone.*/
/* ------------------------------------------------------------------------ */
typedef struct re_server re_server;

typedef struct re_server_desc {
    uint64_t hbm_budget_bytes;   /* scenes + path pool + ReSTIR state          */
    uint32_t path_capacity;      /* paths rendered concurrently (<= 2^27 - 1)  */
    uint32_t max_depth;          /* <= 16                                      */
    uint32_t device;
    uint32_t max_batch_views;    /* requests per launch, <= RE_MAX_BATCH_VIEWS */
    uint32_t build_kind;         /* RE_BUILD_LBVH or RE_BUILD_FLATTENED_SAH    */
    uint32_t restir;             /* 1: reserve ReSTIR state for RestirPrimary requests */
    re_restir_config restir_config;
    uint32_t launch_paths;       /* paths per launch of one step (0: 16 Mi); see re_plan_launches */
    uint32_t backfill_window;    /* admission: how many later requests that fit
                                    now may start ahead of one that waits for
                                    budget or a path range (0: strict arrival
                                    order; RE_BACKFILL_DEFAULT: 64)            */
} re_server_desc;
#define RE_BACKFILL_DEFAULT 0xffffffffu

typedef struct re_render_request {
    uint64_t scene_key;
    re_frame_constants frame;    /* image.z = first sample index; image.w = depth */
    uint32_t spp;                /* samples = server steps the request takes    */
    uint32_t reserved;
    double arrival_time;         /* seconds on the server clock (<= now: now)   */
} re_render_request;

#define RE_REQUEST_WAITING  0u
#define RE_REQUEST_RUNNING  1u
#define RE_REQUEST_DONE     2u
#define RE_REQUEST_FAILED   3u

typedef struct re_request_status {
    uint32_t state;              /* RE_REQUEST_*                                */
    uint32_t samples_done;
    uint32_t error;              /* re_status of a failed request               */
    uint32_t reserved;
    double arrival_time, admit_time, completion_time;  /* server clock, seconds */
} re_request_status;

typedef struct re_server_stats {
    uint64_t submitted, completed, failed, launches;
    uint64_t samples;            /* pixels x samples of completed requests      */
    uint64_t path_rays, shadow_rays;
    uint64_t scene_builds, evictions;
    uint64_t resident_bytes, budget_bytes;
    double latency_p50, latency_p99, latency_mean;   /* seconds, completed     */
    double first_arrival, last_completion;           /* server clock, seconds  */
    uint64_t backfilled;         /* requests admitted ahead of a waiting one    */
} re_server_stats;

RE_API re_status re_server_create(const re_server_desc* desc, re_server** out);
RE_API re_status re_server_destroy(re_server* s);
/* Seconds since the server was created (the clock of arrival times). */
RE_API double re_server_clock(const re_server* s);
/* Registers a scene's records (copied); fails if the key is taken. */
RE_API re_status re_server_register_scene(re_server* s, uint64_t scene_key, const re_canonical_triangle* triangles,
                                          uint32_t triangle_count, const re_material* materials,
                                          uint32_t material_count, const re_light* lights, uint32_t light_count,
                                          const re_float4* fixture_triangles, uint32_t fixture_count,
                                          uint32_t light_selection, float scene_radius);
RE_API re_status re_server_submit(re_server* s, const re_render_request* request, uint64_t* request_id);
/* Runs the scheduling loop: admits arrived requests, launches, retires.
 * Returns after `max_steps` launches, or when nothing is admitted or in
 * flight and no request arrives within `max_wait_seconds`. */
RE_API re_status re_server_pump(re_server* s, uint32_t max_steps, double max_wait_seconds, uint32_t* steps);
/* Runs until every submitted request is done or failed. */
RE_API re_status re_server_drain(re_server* s);
RE_API re_status re_server_poll(re_server* s, uint64_t request_id, re_request_status* out);
/* The finished request's film (progressive mean, re_float4 per pixel). */
RE_API re_status re_server_read_result(re_server* s, uint64_t request_id, re_float4* out, uint32_t pixel_count);
/* Forgets a finished request and its result. */
RE_API re_status re_server_release(re_server* s, uint64_t request_id);
RE_API re_status re_server_stats_get(re_server* s, re_server_stats* out);

/* ------------------------------------------------------------------------ */
/* BSDF readback probe: the device BSDF (Lambert, GGX conductor, GGX        */
/* dielectric reflection, smooth glass, rough dielectric, metallic-         */
/* roughness; PbrBsdf.hlsli:82-1679) evaluated and sampled on a batch of    */
/* queries, one thread per query, with the same functions the Shade kernels  */
/* call.  Replaces the reference's compile/readback probe                   */
/* resources/shaders/integrators/pbr_sampling_probe.hlsl:9-102 (fixed        */
/* context, one material per probe) with caller-chosen contexts, parameters  */
/* (BsdfContextL6 / BsdfParamsL6, PbrBsdf.hlsli:15-80), directions and       */
/* random triples, so the device arithmetic can be checked against the      */
/* reference's FP64 twin (integrators/megakernel/include/ReferenceBsdf.hpp:  */
/* EvaluateBsdfL6 :922, PdfBsdfL6 :980, SampleBsdfL6 :1242) and sampled     */
/* statistically.  Per query: EvaluateBsdfL6(wo, wi), SampleBsdfL6(wo,      */
/* random), and PdfBsdfL6(wo, sampled direction) for a non-delta sample.     */
/* `memory` says where queries and results live (RE_MEMORY_HOST: staged     */
/* through device memory and synchronised before return; RE_MEMORY_DEVICE:  */
/* asynchronous on `stream`).  Both pointers 16-byte aligned.               */
/* ------------------------------------------------------------------------ */
typedef struct re_bsdf_query {
    float geometric_normal[3]; float eta_incident;
    float shading_normal[3]; float eta_transmitted;
    float tangent[3]; uint32_t transport_mode;       /* 0 radiance, 1 importance */
    float base_color[3]; float metallic;
    float f0[3]; float perceptual_roughness;
    float conductor_eta[3]; float transmission;
    float conductor_k[3]; uint32_t model;            /* 0..5 as BsdfParamsL6.model */
    float wo[3]; uint32_t allowed_lobes;
    float wi[3]; uint32_t use_complex_conductor_fresnel;
    float random[3]; uint32_t reserved;               /* lobe, u, v in [0, 1) */
} re_bsdf_query;
typedef struct re_bsdf_probe_result {
    float eval_value[3]; float eval_pdf;
    float eval_diffuse[3]; uint32_t eval_measure;    /* 0 invalid, 1 solid angle, 2 discrete */
    float eval_specular[3]; uint32_t eval_lobe;
    float sample_direction[3]; float sample_pdf;
    float sample_value[3]; float sample_eta;
    float sample_diffuse[3]; uint32_t sample_measure;
    float sample_specular[3]; uint32_t sample_lobe;
    uint32_t eval_valid; uint32_t sample_delta; uint32_t sample_valid;
    float pdf_at_sample;                              /* PdfBsdfL6(wo, sample_direction), 0 for delta */
} re_bsdf_probe_result;
RE_API re_status re_bsdf_probe(const re_bsdf_query* queries, uint32_t count, re_bsdf_probe_result* results,
                               uint32_t memory, void* stream);

/* ------------------------------------------------------------------------ */
/* Allocation-free GPU LBVH build.  No counterpart in the reference: it is   */
/* the GPU LBVH of re_scene_create(RE_BUILD_LBVH) (bounds, 30-bit Morton     */
/* codes, stable radix sort on (code, stable ID), Karras hierarchy, refit)  */
/* for callers that cannot allocate device memory where they build, e.g. a  */
/* renderer rebuilding small dynamic meshes between launches of a frame     */
/* under a fixed memory budget, where a cudaMalloc would synchronise the    */
/* device.  Every intermediate array lives in one static device array of    */
/* about 9.3 MB; the call makes no allocation of any kind.                  */
/*   - At most RE_LBVH_STATIC_MAX_TRIANGLES triangles; larger counts fail   */
/*     with RE_INVALID_ARGUMENT before anything is launched.                */
/*   - All calls on one device share the scratch: calls that overlap (on    */
/*     any streams or threads) race and must be serialised by the caller.   */
/*   - The first call on a device, with that device current, resolves the   */
/*     scratch address (cudaGetSymbolAddress); make it before any stream     */
/*     capture.                                                             */
/*   - No buffer needs to start at zero: each call re-initialises its own   */
/*     bounds and refit counters.                                           */
/*   - The cached scratch address belongs to the device's context: a        */
/*     cudaDeviceReset between calls is not supported (the next call would  */
/*     launch on a stale address).                                          */
/*   - A CUDA error still pending from the caller's earlier work is         */
/*     returned as RE_CUDA_ERROR, naming it, before anything is launched.   */
/* Inputs (device, current device): positions as 3 re_float4 per triangle   */
/* (w ignored) and the stable IDs the sort breaks ties on.  The IDs should  */
/* be unique, as every other scene build requires (it rejects duplicates);  */
/* this call cannot check without a read-back, so triangles whose Morton    */
/* codes and IDs are both equal are split by their sorted position (source  */
/* order), which still gives a well-formed hierarchy.                       */
/* Outputs (device): order_out[count] = source index of each leaf in sorted */
/* order; nodes_out[count - 1] = the Karras internal nodes (node 0 is the   */
/* root) with their bounds; with count == 1 only order_out is written and   */
/* nodes_out may be NULL.  Alignment, checked (RE_INVALID_ARGUMENT):         */
/* positions and nodes_out 16 bytes, stable_ids and order_out 4 bytes.      */
/* Asynchronous on `stream` (NULL = the legacy default stream).             */
/* ------------------------------------------------------------------------ */
#define RE_LBVH_STATIC_MAX_TRIANGLES 65536u
#define RE_LBVH_CHILD_LEAF (1u << 31)  /* child is a leaf: low bits = sorted position */
typedef struct re_lbvh_node {
    float bounds_min[3];
    uint32_t left;
    float bounds_max[3];
    uint32_t right;
} re_lbvh_node;
RE_API re_status re_lbvh_build_static(const re_float4* positions, const uint32_t* stable_ids, uint32_t count,
                                      uint32_t* order_out, re_lbvh_node* nodes_out, void* stream);

/* ------------------------------------------------------------------------ */
/* SVGF / A-Trous reconstruction: SvgfReconstruction (reconstruction/       */
/* include/reconstruction/Svgf.hpp:30-75, src/Svgf.cpp:393-752) on the GPU.  */
/* Temporal reprojection with per-tap history validation and a 3x3 nearest  */
/* fallback, luminance moments, 7x7 variance bootstrap, N x 5x5 B3 A-Trous   */
/* with depth / normal / luminance edge stopping, demodulation by albedo.   */
/* History (HistoryPingPong, History.hpp:24-61) stays resident in HBM.      */
/* ------------------------------------------------------------------------ */
typedef struct re_svgf re_svgf;

/* GBufferPixel (reconstruction/include/reconstruction/Types.hpp:72-90) with
 * the two bools folded into `flags`; 64 bytes. */
#define RE_GBUFFER_VALID         (1u << 0)
#define RE_GBUFFER_MOTION_VALID  (1u << 1)
typedef struct re_gbuffer_pixel {
    float linear_depth;
    float world_normal[3];
    float diffuse_albedo[3];
    float specular_albedo[3];
    float expected_previous_linear_depth;
    float motion[2];               /* previous UV - current UV               */
    uint32_t material_id;
    uint32_t object_id;
    uint32_t flags;                /* RE_GBUFFER_VALID | RE_GBUFFER_MOTION_VALID */
} re_gbuffer_pixel;

/* SignalPixel (Types.hpp:92-95), byte-identical: diffuse then specular. */
typedef struct re_signal_pixel {
    float diffuse[3];
    float specular[3];
} re_signal_pixel;

/* SvgfConfig and its parts (Types.hpp:164-202), flattened.  Field defaults
 * come from re_svgf_default_config(). */
typedef struct re_svgf_config {
    float relative_depth_threshold;    /* ValidationConfig                  */
    float absolute_depth_threshold;
    float normal_cosine_threshold;
    uint32_t require_material_id;
    uint32_t require_object_id;
    uint32_t max_history_length;       /* TemporalConfig, <= 2^31 - 1       */
    float minimum_color_alpha;
    float minimum_moments_alpha;
    uint32_t short_history_length;     /* VarianceConfig                    */
    uint32_t spatial_radius;           /* <= 64                             */
    float minimum_variance;
    uint32_t atrous_iterations;        /* ATrousConfig, <= 16               */
    float phi_depth;
    float phi_normal;
    float phi_luminance;
    float minimum_albedo;              /* SvgfConfig                        */
    uint32_t demodulate_specular;
} re_svgf_config;

/* ResetTrigger bits (Types.hpp:130-140). */
#define RE_RESET_CAMERA_CUT            (1u << 0)
#define RE_RESET_FIELD_OF_VIEW         (1u << 1)
#define RE_RESET_RESOLUTION            (1u << 2)
#define RE_RESET_SCENE                 (1u << 3)
#define RE_RESET_BACKEND               (1u << 4)
#define RE_RESET_TRANSPORT             (1u << 5)
#define RE_RESET_RECONSTRUCTION_PARAMS (1u << 6)
#define RE_RESET_SHADER_RELOAD         (1u << 7)

/* RejectReason bits (Types.hpp:100-113). */
#define RE_REJECT_NO_HISTORY      (1u << 0)
#define RE_REJECT_RESET           (1u << 1)
#define RE_REJECT_SCREEN_BOUNDS   (1u << 2)
#define RE_REJECT_INVALID_CURRENT (1u << 3)
#define RE_REJECT_INVALID_HISTORY (1u << 4)
#define RE_REJECT_NON_FINITE      (1u << 5)
#define RE_REJECT_DEPTH           (1u << 6)
#define RE_REJECT_NORMAL          (1u << 7)
#define RE_REJECT_MATERIAL_ID     (1u << 8)
#define RE_REJECT_OBJECT_ID       (1u << 9)
#define RE_REJECT_INVALID_MOTION  (1u << 10)

/* FrameInputs (Svgf.hpp:12-17).  Both arrays are width*height records,
 * row-major, in `memory`; device arrays must be 16-byte aligned. */
typedef struct re_svgf_frame_inputs {
    const re_gbuffer_pixel* gbuffer;
    const re_signal_pixel* raw_signal;
    uint32_t width;
    uint32_t height;
    uint32_t memory;               /* re_memory                               */
    uint32_t reset_trigger;        /* RE_RESET_* bits                         */
    uint64_t frame_index;
} re_svgf_frame_inputs;

/* ReconstructionFrame planes (Svgf.hpp:19-29) for re_svgf_read; per pixel:
 * RAW/TEMPORAL/ATROUS/SVGF re_signal_pixel, HISTORY_LENGTH uint32, MOMENTS
 * 2 floats, VARIANCE float, ACCEPTED uint32 (0/1), REJECT_REASONS uint32. */
#define RE_SVGF_PLANE_RAW            0u
#define RE_SVGF_PLANE_TEMPORAL       1u
#define RE_SVGF_PLANE_ATROUS         2u
#define RE_SVGF_PLANE_SVGF           3u
#define RE_SVGF_PLANE_HISTORY_LENGTH 4u
#define RE_SVGF_PLANE_MOMENTS        5u
#define RE_SVGF_PLANE_VARIANCE       6u
#define RE_SVGF_PLANE_ACCEPTED       7u
#define RE_SVGF_PLANE_REJECT_REASONS 8u

/* ReconstructionOutput (Types.hpp:155-166) for re_svgf_select_output. */
#define RE_SVGF_OUTPUT_RAW               0u
#define RE_SVGF_OUTPUT_TEMPORAL          1u
#define RE_SVGF_OUTPUT_ATROUS            2u
#define RE_SVGF_OUTPUT_SVGF              3u
#define RE_SVGF_OUTPUT_MOTION            4u
#define RE_SVGF_OUTPUT_HISTORY_LENGTH    5u
#define RE_SVGF_OUTPUT_MOMENTS           6u
#define RE_SVGF_OUTPUT_VARIANCE          7u
#define RE_SVGF_OUTPUT_HISTORY_ACCEPTANCE 8u
#define RE_SVGF_OUTPUT_REJECT_REASONS    9u

RE_API re_status re_svgf_default_config(re_svgf_config* out);
/* SvgfReconstruction(extent, framesInFlight, config): validates the config
 * like ValidateConfigOrThrow (Svgf.cpp:52-80) and allocates the history
 * surfaces (2 x frames_in_flight) and per-frame planes in HBM. */
RE_API re_status re_svgf_create(uint32_t width, uint32_t height, uint32_t frames_in_flight,
                                const re_svgf_config* config, uint32_t device, re_svgf** out);
RE_API re_status re_svgf_destroy(re_svgf* s);
/* SetConfig: the next process() applies ResetTrigger::ReconstructionParameters. */
RE_API re_status re_svgf_set_config(re_svgf* s, const re_svgf_config* config);
RE_API re_status re_svgf_get_config(const re_svgf* s, re_svgf_config* out);
/* Reset(extent): drops every history generation. */
RE_API re_status re_svgf_reset(re_svgf* s, uint32_t width, uint32_t height);
/* Process(inputs): asynchronous on `stream`; the frame's planes stay valid
 * until the next process() call. */
RE_API re_status re_svgf_process(re_svgf* s, const re_svgf_frame_inputs* inputs, void* stream);
/* Copies one ReconstructionFrame plane of the last processed frame. */
RE_API re_status re_svgf_read(re_svgf* s, uint32_t plane, void* dst, uint64_t bytes,
                              uint32_t memory, void* stream);
/* Device pointer of a plane of the last processed frame. */
RE_API re_status re_svgf_plane_pointer(re_svgf* s, uint32_t plane, void** out);
/* SelectOutput (Svgf.cpp:754-822): 3 floats per pixel into `dst`.  `gbuffer`
 * (width*height records in `gbuffer_memory`) is read only for MOTION and may
 * be NULL otherwise. */
RE_API re_status re_svgf_select_output(re_svgf* s, const re_gbuffer_pixel* gbuffer,
                                       uint32_t gbuffer_memory, uint32_t output, float* dst,
                                       uint32_t dst_memory, void* stream);
/* ComputeRmse (Svgf.cpp:824-833) of two 3-float-per-pixel device images;
 * double accumulation, synchronous. */
RE_API re_status re_image_rmse(const float* candidate, const float* reference, uint64_t pixel_count,
                               float* out_rmse, void* stream);

/* ------------------------------------------------------------------------ */
/* Renderer -> reconstruction.  No counterpart in the reference, whose      */
/* SVGF runs on G-buffers it is handed (reconstruction/Svgf.hpp:52-75): this*/
/* forms them from a rendered view.                                          */
/* ------------------------------------------------------------------------ */
/* Camera matrices of a frame in the reconstruction conventions of
 * reconstruction/Math.hpp:110-129 and MotionVectors.hpp:7-18 (row-major,
 * column vectors, right-handed view space looking down -Z): the
 * view-projection whose clip w is the view depth and whose UV is the
 * renderer's image position, and the world-to-view matrix.  Host only. */
RE_API re_status re_camera_matrices(const re_frame_constants* frame, float view_projection[16],
                                    float world_to_view[16]);
/* SVGF inputs of one rendered view (width x height of `current`, paths from
 * `path_offset`, scene in `scene_slot`), from the last launch that rendered
 * it: per pixel a re_gbuffer_pixel of the primary hit (view linear depth,
 * shading normal, diffuse / specular albedo of the hit material, material
 * and instance IDs, motion to the `previous` frame's camera as
 * ComputeMotionVector, MotionVectors.cpp:37-74, computes it; `previous` NULL:
 * no motion) and a re_signal_pixel of that frame's radiance (diffuse:
 * camera-visible emission + direct + indirect diffuse; specular: direct +
 * indirect specular).  Albedos: Lambert, diffuse = base color;
 * metallic-roughness, diffuse = base * (1 - metallic) * (1 - transmission),
 * specular = f0 * (1 - metallic) + base * metallic; conductor, specular =
 * base; dielectric reflection, specular = f0; glass, specular = 1. */
RE_API re_status re_renderer_export_reconstruction(re_renderer* r, uint32_t scene_slot, uint32_t path_offset,
                                                   const re_frame_constants* current,
                                                   const re_frame_constants* previous, re_gbuffer_pixel* gbuffer,
                                                   re_signal_pixel* signal, uint32_t memory, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RE_B200_H */
