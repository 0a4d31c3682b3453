// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// A thin extern "C" shim over the reference's own CPU code, compiled from the
// unmodified reference sources by oracle/Makefile into oracle/_ref/.  Tests
// load it with ctypes to pin the oracle restatement and to check the CUDA
// kernels against the reference implementation itself:
//   - Rt::Cpu::Bvh<float> binned-SAH build      include/rt/cpu/Bvh.hpp:82-133
//   - SoftwareGpu::FlattenCanonicalL3BinnedSah  src/rt/software_gpu/SoftwareGpu.cpp:1109
//   - SoftwareGpu::Trace (closest / any)        src/rt/software_gpu/SoftwareGpu.cpp:1529
//   - SoftwareGpu::BuildKarrasLbvh              src/rt/software_gpu/SoftwareGpu.cpp:1265
//   - RenderCornellReference                    src/integrators/reference_cpu/CornellReference.cpp:734
//   - Megakernel::CounterRandomFloat / BuildVoseAliasTable / BuildTopLevelLightDistribution
//                                               integrators/megakernel/MegakernelBridge.cpp:40-589
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "MegakernelBridge.hpp"
#include "integrators/reference_cpu/CornellReference.hpp"
#include "rt/cpu/Bvh.hpp"
#include "rt/cpu/Random.hpp"
#include "rt/software_gpu/SoftwareGpu.hpp"

namespace sg = RenderingEngine::Rt::SoftwareGpu;
namespace cpu = RenderingEngine::Rt::Cpu;
namespace mk = RenderingEngine::Integrators::Megakernel;

namespace {

std::vector<sg::SoftwarePrimitiveRecord> make_prims(const float* v, const uint32_t* ids, uint32_t n) {
    std::vector<sg::SoftwarePrimitiveRecord> prims(n);
    for (uint32_t i = 0; i < n; ++i) {
        const float* t = v + size_t(i) * 9u;
        prims[i] = sg::MakeTriangle({t[0], t[1], t[2]}, {t[3], t[4], t[5]}, {t[6], t[7], t[8]}, ids[i]);
    }
    return prims;
}

void export_bvh(const sg::FlatBvh& bvh, float* nodes_out, uint32_t* order_ids_out) {
    for (size_t i = 0; i < bvh.nodes.size(); ++i) {
        std::memcpy(nodes_out + i * 12u, &bvh.nodes[i], 48);
    }
    for (size_t i = 0; i < bvh.primitives.size(); ++i) order_ids_out[i] = bvh.primitives[i].identity.x;
}

}  // namespace

extern "C" {

// Bvh<float>(BinnedSah, leaf) + FlattenCanonicalL3BinnedSah.  Writes node
// records (12 words each), the primitive order (source indices) and depth.
// Returns the node count, or -1 with the status code in *status.
int ref_sah_build(const float* v, const uint32_t* ids, uint32_t n, uint32_t max_leaf,
                  float* nodes_out, uint32_t node_capacity, uint32_t* order_out,
                  uint32_t* depth_out, int* status) {
    std::vector<cpu::Triangle<float>> tris(n);
    for (uint32_t i = 0; i < n; ++i) {
        const float* t = v + size_t(i) * 9u;
        tris[i] = cpu::Triangle<float>({t[0], t[1], t[2]}, {t[3], t[4], t[5]}, {t[6], t[7], t[8]}, ids[i]);
    }
    try {
        cpu::Bvh<float> bvh(std::span<const cpu::Triangle<float>>(tris), cpu::BvhBuildMethod::BinnedSah, max_leaf);
        const auto prims = make_prims(v, ids, n);
        const sg::FlatBuildResult flat = sg::FlattenCanonicalL3BinnedSah(bvh, prims);
        *status = int(flat.status);
        if (!flat.Succeeded()) return -1;
        if (flat.bvh.nodes.size() > node_capacity) { *status = 100; return -1; }
        for (size_t i = 0; i < flat.bvh.nodes.size(); ++i) std::memcpy(nodes_out + i * 12u, &flat.bvh.nodes[i], 48);
        const auto order = bvh.PrimitiveOrder();
        for (size_t i = 0; i < order.size(); ++i) order_out[i] = uint32_t(order[i]);
        *depth_out = flat.bvh.maximumDepth;
        return int(flat.bvh.nodes.size());
    } catch (const std::exception&) {
        *status = 200;
        return -1;
    }
}

// SoftwareGpu::Trace over caller-supplied flattened nodes and leaf-ordered
// primitives.  rays: n x 12 floats (originTMin, directionTMax, query as bits).
// hits_out: n x 8 words (tBary, identity).  counters_out: 11 u64 values.
void ref_trace(const float* nodes, uint32_t node_count, const float* prim_v, const uint32_t* prim_ids,
               uint32_t prim_count, const float* rays, uint32_t ray_count, uint32_t mode,
               uint32_t stack_capacity, uint32_t threads, uint32_t* hits_out, uint64_t* counters_out) {
    sg::FlatBvh bvh;
    bvh.nodes.resize(node_count);
    for (uint32_t i = 0; i < node_count; ++i) std::memcpy(&bvh.nodes[i], nodes + size_t(i) * 12u, 48);
    bvh.primitives = make_prims(prim_v, prim_ids, prim_count);
    // Harness thread pool over interleaved rays; Trace is const and noexcept.
    const uint32_t nt = threads == 0 ? 1u : threads;
    std::vector<sg::TraversalCounters> part(nt);
    auto work = [&](uint32_t tid) {
        for (uint32_t r = tid; r < ray_count; r += nt) {
            sg::SoftwareRayRecord ray;
            std::memcpy(&ray, rays + size_t(r) * 12u, 48);
            const sg::TraceResult res = sg::Trace(bvh, ray, sg::QueryMode(mode), stack_capacity);
            std::memcpy(hits_out + size_t(r) * 8u, &res.hit, 32);
            part[tid].Accumulate(res.counters);
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < nt; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    sg::TraversalCounters total{};
    for (const auto& c : part) total.Accumulate(c);
    const uint64_t c[11] = {total.nodeTests, total.triangleTests, total.rays, total.hits,
                            total.stackOverflows, total.invalidRays, total.invalidHits,
                            total.leafVisits, total.accumulatedLeafPrimitives,
                            total.maximumStackDepth, total.maximumLeafOccupancy};
    std::memcpy(counters_out, c, sizeof(c));
}

// SoftwareGpu::BuildKarrasLbvh.  Returns node count or -1 (status in *status).
int ref_lbvh_build(const float* v, const uint32_t* ids, uint32_t n, float* nodes_out,
                   uint32_t node_capacity, uint32_t* prim_ids_out, uint32_t* morton_out,
                   uint32_t* depth_out, int* status) {
    const auto prims = make_prims(v, ids, n);
    const sg::FlatBuildResult r = sg::BuildKarrasLbvh(prims);
    *status = int(r.status);
    if (!r.Succeeded()) return -1;
    if (r.bvh.nodes.size() > node_capacity) { *status = 100; return -1; }
    export_bvh(r.bvh, nodes_out, prim_ids_out);
    for (size_t i = 0; i < r.bvh.mortonOrder.size(); ++i) {
        morton_out[i * 2 + 0] = r.bvh.mortonOrder[i].code;
        morton_out[i * 2 + 1] = r.bvh.mortonOrder[i].sourceIndex;
    }
    *depth_out = r.bvh.maximumDepth;
    return int(r.bvh.nodes.size());
}

// RenderCornellReference.  pixels_out: w*h*3 floats.  stats_out: scene hash,
// ray count, shadow-ray count, non-finite count.  Returns elapsed ms or -1.
double ref_cornell(uint32_t width, uint32_t height, uint32_t spp, uint32_t max_bounces, uint64_t seed,
                   uint32_t threads, float* pixels_out, uint64_t* stats_out) {
    RenderingEngine::Integrators::ReferenceCpu::CornellReferenceOptions o;
    o.width = width;
    o.height = height;
    o.spp = spp;
    o.maxBounces = max_bounces;
    o.seed = seed;
    o.threads = threads;
    RenderingEngine::Integrators::ReferenceCpu::CornellReferenceResult r;
    std::string err;
    if (!RenderingEngine::Integrators::ReferenceCpu::RenderCornellReference(o, r, err)) return -1.0;
    std::memcpy(pixels_out, r.pixels.data(), r.pixels.size() * sizeof(float));
    stats_out[0] = r.sceneHash;
    stats_out[1] = r.rayCount;
    stats_out[2] = r.shadowRayCount;
    stats_out[3] = r.nonFiniteCount;
    return r.elapsedMilliseconds;
}

float ref_counter_random(uint32_t pixel, uint32_t sample, uint32_t dim, uint32_t stream, uint64_t seed) {
    return mk::CounterRandomFloat(pixel, sample, dim, stream, seed);
}

void ref_philox(const uint32_t* counter, const uint32_t* key, uint32_t* out) {
    const auto r = mk::Philox4x32TenRounds({counter[0], counter[1], counter[2], counter[3]}, {key[0], key[1]});
    for (int i = 0; i < 4; ++i) out[i] = r[i];
}

// BuildVoseAliasTable: entries_out n x 4 words (q, pmf as float bits, alias, item).
int ref_alias_table(const double* weights, uint32_t n, uint32_t* entries_out) {
    try {
        const mk::AliasTable t = mk::BuildVoseAliasTable(std::span<const double>(weights, n));
        std::memcpy(entries_out, t.entries.data(), t.entries.size() * 16u);
        return int(t.entries.size());
    } catch (const std::exception&) {
        return -1;
    }
}

// BuildTopLevelLightDistribution over PbrLightGpu records (96 B each).
int ref_light_distribution(const void* lights, uint32_t n, uint32_t selection, float scene_radius,
                           uint32_t* alias_out, float* pmf_by_light_out) {
    try {
        std::vector<mk::PbrLightGpu> ls(n);
        std::memcpy(ls.data(), lights, size_t(n) * sizeof(mk::PbrLightGpu));
        const auto d = mk::BuildTopLevelLightDistribution(ls, mk::LightSelection(selection), scene_radius, 0.0);
        std::memcpy(alias_out, d.alias.data(), d.alias.size() * 16u);
        std::memcpy(pmf_by_light_out, d.selectionPmfByLight.data(), d.selectionPmfByLight.size() * 4u);
        return int(d.alias.size());
    } catch (const std::exception&) {
        return -1;
    }
}

}  // extern "C"

extern "C" {

// The seeded 18-triangle scene and ray corpus of the reference's statistical
// traversal parity test (tests/statistical/L3/TraversalParityTests.cpp:18-43,
// :62-84), generated with the reference's own Pcg32.  Triangles are returned
// as float (9 per triangle) with their stable IDs; rays as float
// (origin.xyz, tMin, direction.xyz, tMax).  The FP64 brute-force closest hit
// of every ray (TraceClosestBruteForce<double>) is returned as the golden
// answer: id (0xffffffff for a miss) and t.
void ref_l3_parity_corpus(uint32_t ray_count, float* tris_out, uint32_t* ids_out, float* rays_out,
                          uint32_t* brute_id_out, double* brute_t_out) {
    std::vector<cpu::Triangle<double>> triangles;
    uint32_t pid = 100u;
    for (uint32_t layer = 0u; layer < 3u; ++layer) {
        const double z = -2.0 - double(layer) * 1.5;
        for (uint32_t cell = 0u; cell < 3u; ++cell) {
            const double x = -2.2 + double(cell) * 2.2;
            const double y = -0.8 + double(layer) * 0.7;
            triangles.emplace_back(cpu::Vec3<double>{x - 0.55, y - 0.45, z}, cpu::Vec3<double>{x + 0.55, y - 0.45, z},
                                   cpu::Vec3<double>{x + 0.35, y + 0.55, z - 0.05}, pid++);
            triangles.emplace_back(cpu::Vec3<double>{x - 0.45, y - 0.35, z - 0.35},
                                   cpu::Vec3<double>{x + 0.30, y + 0.50, z - 0.40},
                                   cpu::Vec3<double>{x - 0.60, y + 0.40, z - 0.50}, pid++);
        }
    }
    for (size_t i = 0; i < triangles.size(); ++i) {
        const auto& t = triangles[i];
        const double v[9] = {t.v0.x, t.v0.y, t.v0.z, t.v1.x, t.v1.y, t.v1.z, t.v2.x, t.v2.y, t.v2.z};
        for (int k = 0; k < 9; ++k) tris_out[i * 9 + k] = float(v[k]);
        ids_out[i] = t.primitiveId;
    }
    cpu::Pcg32 rng(0x4c33504152495459ull, 0x524159434f525055ull);
    for (uint32_t r = 0; r < ray_count; ++r) {
        const cpu::Vec3<double> origin{rng.Uniform<double>() * 10.0 - 5.0, rng.Uniform<double>() * 7.0 - 3.5,
                                       rng.Uniform<double>() * 3.0 + 0.25};
        const cpu::Vec3<double> target{rng.Uniform<double>() * 7.0 - 3.5, rng.Uniform<double>() * 4.0 - 2.0,
                                       -(rng.Uniform<double>() * 6.0 + 1.0)};
        const cpu::Ray<double> ray{origin, cpu::NormalizeOrZero(target - origin), 1.0e-8, 1.0e6};
        const cpu::Hit<double> brute = cpu::TraceClosestBruteForce<double>(triangles, ray);
        float* o = rays_out + size_t(r) * 8u;
        o[0] = float(ray.origin.x); o[1] = float(ray.origin.y); o[2] = float(ray.origin.z); o[3] = float(ray.tMin);
        o[4] = float(ray.direction.x); o[5] = float(ray.direction.y); o[6] = float(ray.direction.z); o[7] = float(ray.tMax);
        brute_id_out[r] = brute.IsHit() ? brute.primitiveId : 0xffffffffu;
        brute_t_out[r] = brute.IsHit() ? brute.t : 0.0;
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// BuildCanonicalTraversalScene (src/rt/gpu/CanonicalTraversalScene.cpp:69):
// instance expansion of flat SceneAbiV0 arrays into CanonicalTraversalTriangle
// records.  Returns the triangle count, or -1 with the reference's error
// message copied to `error` (capacity `error_cap`).
// ---------------------------------------------------------------------------
#include "rt/gpu/CanonicalTraversalScene.hpp"

extern "C" {

int ref_canonical_expand(const void* vertices, uint32_t vertex_count, const uint32_t* indices, uint32_t index_count,
                         const void* geometries, uint32_t geometry_count, const void* instances,
                         uint32_t instance_count, const void* materials, uint32_t material_count, void* out,
                         uint32_t out_capacity, char* error, uint32_t error_cap) {
    namespace abi = RenderingEngine::Contracts::AbiV0;
    namespace scn = RenderingEngine::Scene;
    namespace gpu = RenderingEngine::Rt::Gpu;
    abi::GpuSceneConstantsV0 constants{};
    scn::CanonicalSceneView view;
    view.stableId = "oracle";
    view.fingerprint = 1u;
    view.generation = 1u;
    view.constants = &constants;
    view.vertices = {static_cast<const abi::GpuVertexV0*>(vertices), vertex_count};
    view.indices = {indices, index_count};
    view.geometries = {static_cast<const abi::GpuGeometryV0*>(geometries), geometry_count};
    view.instances = {static_cast<const abi::GpuInstanceV0*>(instances), instance_count};
    view.materials = {static_cast<const abi::GpuMaterialV0*>(materials), material_count};
    const gpu::CanonicalTraversalSceneBuild build = gpu::BuildCanonicalTraversalScene(view);
    if (!build) {
        if (error != nullptr && error_cap > 0u) {
            const size_t n = std::min<size_t>(build.error.size(), error_cap - 1u);
            std::memcpy(error, build.error.data(), n);
            error[n] = '\0';
        }
        return -1;
    }
    const size_t n = build.scene.triangles.size();
    if (n > out_capacity) return -2;
    std::memcpy(out, build.scene.triangles.data(), n * sizeof(gpu::CanonicalTraversalTriangle));
    return int(n);
}

}  // extern "C"

extern "C" {

// BuildEnvironmentDistribution (MegakernelBridge.cpp:191-273) over per-texel
// luminance: row entries (height), column entries (height x width), the
// integrated luminance and the uniform-sphere fallback flag.  Returns 0, or
// -1 when the reference rejects the input.
int ref_env_distribution(uint32_t width, uint32_t height, const float* luminance, uint32_t* rows_out,
                         uint32_t* cols_out, double* integrated_out, int* fallback_out) {
    try {
        const auto d = mk::BuildEnvironmentDistribution(
            width, height, std::span<const float>(luminance, size_t(width) * height));
        std::memcpy(rows_out, d.rowAlias.data(), d.rowAlias.size() * 16u);
        std::memcpy(cols_out, d.columnAlias.data(), d.columnAlias.size() * 16u);
        *integrated_out = d.integratedLuminance;
        *fallback_out = d.usedUniformSphereFallback ? 1 : 0;
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// BuildTopLevelLightDistribution with an environment's integrated luminance.
int ref_light_distribution_env(const void* lights, uint32_t n, uint32_t selection, float scene_radius,
                               double env_integrated, uint32_t* alias_out, float* pmf_by_light_out) {
    try {
        std::vector<mk::PbrLightGpu> ls(n);
        std::memcpy(ls.data(), lights, size_t(n) * sizeof(mk::PbrLightGpu));
        const auto d =
            mk::BuildTopLevelLightDistribution(ls, mk::LightSelection(selection), scene_radius, env_integrated);
        std::memcpy(alias_out, d.alias.data(), d.alias.size() * 16u);
        std::memcpy(pmf_by_light_out, d.selectionPmfByLight.data(), d.selectionPmfByLight.size() * 4u);
        return int(d.alias.size());
    } catch (const std::exception&) {
        return -1;
    }
}

}  // extern "C"
