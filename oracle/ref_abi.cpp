// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// Compiles the C ABI header (include/re_b200.h) beside the reference's own
// contract headers and checks, field by field, that every record the library
// reads or writes as-is has the reference layout: size, alignment and the
// offset of every member.  A mismatch fails the oracle/_ref build; the
// exported count lets a test see that the check was built.
#include <cstddef>
#include <cstdint>

#include "MegakernelBridge.hpp"
#include "contracts/GpuRecordsAbiV1.hpp"
#include "contracts/RestirAbiV3.hpp"
#include "contracts/SceneAbiV0.hpp"
#include "re_b200.h"
#include "rt/gpu/CanonicalTraversalScene.hpp"
#include "rt/software_gpu/SoftwareGpu.hpp"

namespace mk = RenderingEngine::Integrators::Megakernel;
namespace gpu = RenderingEngine::Rt::Gpu;
namespace sg = RenderingEngine::Rt::SoftwareGpu;
namespace v0 = RenderingEngine::Contracts::AbiV0;
namespace v1 = RenderingEngine::Contracts::AbiV1;

namespace {

int g_checked = 0;

#define RE_SAME_RECORD(OURS, THEIRS)                                                     \
    static_assert(sizeof(OURS) == sizeof(THEIRS), #OURS " and " #THEIRS " differ in size"); \
    static_assert(alignof(THEIRS) == 16 && sizeof(OURS) % 16 == 0, #OURS " lanes");        \
    static const int OURS##_size_checked = (++g_checked, 0)
#define RE_SAME_FIELD(OURS, A, THEIRS, B)                                                 \
    static_assert(offsetof(OURS, A) == offsetof(THEIRS, B), #OURS "." #A " is not at " #THEIRS "." #B); \
    static const int OURS##_##A##_checked = (++g_checked, 0)

// CanonicalTraversalTriangle (rt/gpu/CanonicalTraversalScene.hpp:15-25).
RE_SAME_RECORD(re_canonical_triangle, gpu::CanonicalTraversalTriangle);
RE_SAME_FIELD(re_canonical_triangle, positions, gpu::CanonicalTraversalTriangle, positions);
RE_SAME_FIELD(re_canonical_triangle, normals, gpu::CanonicalTraversalTriangle, normals);
RE_SAME_FIELD(re_canonical_triangle, texcoords, gpu::CanonicalTraversalTriangle, texcoords);
RE_SAME_FIELD(re_canonical_triangle, identity, gpu::CanonicalTraversalTriangle, identity);
RE_SAME_FIELD(re_canonical_triangle, metadata, gpu::CanonicalTraversalTriangle, metadata);

// SoftwareNodeRecord (rt/software_gpu/SoftwareGpu.hpp:50-60).
RE_SAME_RECORD(re_software_node, sg::SoftwareNodeRecord);
RE_SAME_FIELD(re_software_node, bounds_min, sg::SoftwareNodeRecord, boundsMin);
RE_SAME_FIELD(re_software_node, bounds_max, sg::SoftwareNodeRecord, boundsMax);
RE_SAME_FIELD(re_software_node, links, sg::SoftwareNodeRecord, links);

// GpuRayQueueRecordV1 / GpuHitQueueRecordV1 (contracts/GpuRecordsAbiV1.hpp:76-94).
RE_SAME_RECORD(re_ray_record, v1::GpuRayQueueRecordV1);
RE_SAME_FIELD(re_ray_record, origin_tmin, v1::GpuRayQueueRecordV1, originTMin);
RE_SAME_FIELD(re_ray_record, direction_tmax, v1::GpuRayQueueRecordV1, directionTMax);
RE_SAME_FIELD(re_ray_record, identity, v1::GpuRayQueueRecordV1, identity);
RE_SAME_FIELD(re_ray_record, rng, v1::GpuRayQueueRecordV1, rng);
RE_SAME_RECORD(re_hit_record, v1::GpuHitQueueRecordV1);
RE_SAME_FIELD(re_hit_record, position_t, v1::GpuHitQueueRecordV1, positionT);
RE_SAME_FIELD(re_hit_record, geometric_normal_bary_u, v1::GpuHitQueueRecordV1, geometricNormalBaryU);
RE_SAME_FIELD(re_hit_record, shading_normal_bary_v, v1::GpuHitQueueRecordV1, shadingNormalBaryV);
RE_SAME_FIELD(re_hit_record, ids, v1::GpuHitQueueRecordV1, ids);
RE_SAME_FIELD(re_hit_record, metadata, v1::GpuHitQueueRecordV1, metadata);
RE_SAME_FIELD(re_hit_record, reserved0, v1::GpuHitQueueRecordV1, reserved0);

// PbrMaterialGpu / PbrLightGpu / MegakernelFrameConstantsGpu
// (integrators/megakernel/MegakernelBridge.hpp:259-338).
RE_SAME_RECORD(re_material, mk::PbrMaterialGpu);
RE_SAME_FIELD(re_material, base_color_metallic, mk::PbrMaterialGpu, baseColorMetallic);
RE_SAME_FIELD(re_material, emissive_roughness, mk::PbrMaterialGpu, emissiveRoughness);
RE_SAME_FIELD(re_material, transmission_ior, mk::PbrMaterialGpu, transmissionIor);
RE_SAME_FIELD(re_material, attenuation_color_distance, mk::PbrMaterialGpu, attenuationColorDistance);
RE_SAME_FIELD(re_material, f0, mk::PbrMaterialGpu, f0);
RE_SAME_FIELD(re_material, conductor_eta, mk::PbrMaterialGpu, conductorEta);
RE_SAME_FIELD(re_material, conductor_k, mk::PbrMaterialGpu, conductorK);
RE_SAME_FIELD(re_material, metadata, mk::PbrMaterialGpu, metadata);
RE_SAME_RECORD(re_light, mk::PbrLightGpu);
RE_SAME_FIELD(re_light, position_range, mk::PbrLightGpu, positionRange);
RE_SAME_FIELD(re_light, direction_cos_outer, mk::PbrLightGpu, directionCosOuter);
RE_SAME_FIELD(re_light, radiance_scale, mk::PbrLightGpu, radianceScale);
RE_SAME_FIELD(re_light, shape_params, mk::PbrLightGpu, shapeParams);
RE_SAME_FIELD(re_light, identity, mk::PbrLightGpu, identity);
RE_SAME_FIELD(re_light, payload, mk::PbrLightGpu, payload);
RE_SAME_RECORD(re_frame_constants, mk::MegakernelFrameConstantsGpu);
RE_SAME_FIELD(re_frame_constants, camera_position_tan_half_fov, mk::MegakernelFrameConstantsGpu,
              cameraPositionTanHalfFov);
RE_SAME_FIELD(re_frame_constants, camera_forward_aspect, mk::MegakernelFrameConstantsGpu, cameraForwardAspect);
RE_SAME_FIELD(re_frame_constants, camera_right_lens_radius, mk::MegakernelFrameConstantsGpu, cameraRightLensRadius);
RE_SAME_FIELD(re_frame_constants, camera_up_exposure, mk::MegakernelFrameConstantsGpu, cameraUpExposure);
RE_SAME_FIELD(re_frame_constants, image, mk::MegakernelFrameConstantsGpu, image);
RE_SAME_FIELD(re_frame_constants, trace, mk::MegakernelFrameConstantsGpu, trace);
RE_SAME_FIELD(re_frame_constants, sampling, mk::MegakernelFrameConstantsGpu, sampling);
RE_SAME_FIELD(re_frame_constants, environment, mk::MegakernelFrameConstantsGpu, environment);
RE_SAME_FIELD(re_frame_constants, distribution, mk::MegakernelFrameConstantsGpu, distribution);
RE_SAME_FIELD(re_frame_constants, russian_roulette, mk::MegakernelFrameConstantsGpu, russianRoulette);
RE_SAME_FIELD(re_frame_constants, scene_center_radius, mk::MegakernelFrameConstantsGpu, sceneCenterRadius);
RE_SAME_FIELD(re_frame_constants, environment_to_world, mk::MegakernelFrameConstantsGpu, environmentToWorld0);
RE_SAME_FIELD(re_frame_constants, world_to_environment, mk::MegakernelFrameConstantsGpu, worldToEnvironment0);
RE_SAME_FIELD(re_frame_constants, traversal, mk::MegakernelFrameConstantsGpu, traversal);
RE_SAME_FIELD(re_frame_constants, output, mk::MegakernelFrameConstantsGpu, output);
static_assert(offsetof(mk::MegakernelFrameConstantsGpu, environmentToWorld2) -
                      offsetof(mk::MegakernelFrameConstantsGpu, environmentToWorld0) ==
                  2 * sizeof(re_float4),
              "environment rows are consecutive");

// SceneAbiV0 object-space records (contracts/SceneAbiV0.hpp:76-111).
RE_SAME_RECORD(re_gpu_vertex_v0, v0::GpuVertexV0);
RE_SAME_FIELD(re_gpu_vertex_v0, position, v0::GpuVertexV0, position);
RE_SAME_FIELD(re_gpu_vertex_v0, normal, v0::GpuVertexV0, normal);
RE_SAME_FIELD(re_gpu_vertex_v0, tangent, v0::GpuVertexV0, tangent);
RE_SAME_FIELD(re_gpu_vertex_v0, texcoord0, v0::GpuVertexV0, texcoord0);
RE_SAME_RECORD(re_gpu_geometry_v0, v0::GpuGeometryV0);
RE_SAME_FIELD(re_gpu_geometry_v0, index_range, v0::GpuGeometryV0, indexRange);
RE_SAME_FIELD(re_gpu_geometry_v0, identity, v0::GpuGeometryV0, identity);
RE_SAME_FIELD(re_gpu_geometry_v0, local_bounds_min, v0::GpuGeometryV0, localBoundsMin);
RE_SAME_FIELD(re_gpu_geometry_v0, local_bounds_max, v0::GpuGeometryV0, localBoundsMax);
RE_SAME_RECORD(re_gpu_instance_v0, v0::GpuInstanceV0);
RE_SAME_FIELD(re_gpu_instance_v0, object_to_world, v0::GpuInstanceV0, objectToWorld);
RE_SAME_FIELD(re_gpu_instance_v0, world_to_object, v0::GpuInstanceV0, worldToObject);
RE_SAME_FIELD(re_gpu_instance_v0, previous_object_to_world, v0::GpuInstanceV0, previousObjectToWorld);
RE_SAME_FIELD(re_gpu_instance_v0, metadata, v0::GpuInstanceV0, metadata);
RE_SAME_RECORD(re_gpu_material_v0, v0::GpuMaterialV0);
RE_SAME_FIELD(re_gpu_material_v0, base_color_factor, v0::GpuMaterialV0, baseColorFactor);
RE_SAME_FIELD(re_gpu_material_v0, emissive_factor_strength, v0::GpuMaterialV0, emissiveFactorStrength);
RE_SAME_FIELD(re_gpu_material_v0, surface_params, v0::GpuMaterialV0, surfaceParams);
RE_SAME_FIELD(re_gpu_material_v0, transmission_params, v0::GpuMaterialV0, transmissionParams);
RE_SAME_FIELD(re_gpu_material_v0, attenuation_color_distance, v0::GpuMaterialV0, attenuationColorDistance);
RE_SAME_FIELD(re_gpu_material_v0, texture_image_indices, v0::GpuMaterialV0, textureImageIndices);
RE_SAME_FIELD(re_gpu_material_v0, texture_sampler_indices, v0::GpuMaterialV0, textureSamplerIndices);
RE_SAME_FIELD(re_gpu_material_v0, metadata, v0::GpuMaterialV0, metadata);

// Enumerations the header mirrors.
static_assert(RE_LIGHT_EMISSIVE_TRIANGLE == static_cast<uint32_t>(mk::LightType::EmissiveTriangle), "light type");
static_assert(RE_LIGHT_ENVIRONMENT == static_cast<uint32_t>(mk::LightType::Environment), "light type");
static_assert(RE_GEOMETRY_FLAG_ALPHA_MASK == v0::GeometryFlagAlphaMask, "geometry flag");
static_assert(RE_GEOMETRY_FLAG_DOUBLE_SIDED == v0::GeometryFlagDoubleSided, "geometry flag");
static_assert(RE_MATERIAL_FLAG_ALPHA_MASK == v0::MaterialFlagAlphaMask, "material flag");
static_assert(RE_MATERIAL_FLAG_DOUBLE_SIDED == v0::MaterialFlagDoubleSided, "material flag");
static_assert(RE_INSTANCE_FLAG_CASTS_SHADOW == v0::InstanceFlagCastsShadow, "instance flag");

}  // namespace

extern "C" int ref_abi_checked_fields() { return g_checked; }
